"""fjb_render_batch: mixed frames (three capture stocks on two print papers, four
frame sizes, every spatial stage) in one call.

* the batch's outputs are bit-identical to the same frames rendered one by one
  through fj_cuda_render (same kernels, same parameters, same order), eagerly and
  through a captured CUDA graph;
* a replay of the captured graph renders new pixel contents of the same buffers (the
  outputs follow the new sources) without any host-side kernel launch of the library;
* per-frame outcomes equal fj_cuda_render's;
* diffusion-form autotuning records a decision per frame size and radius, and its
  output agrees with the fixed rule's within the two forms' difference;
* a frame that fails its checks fails the batch before any work is enqueued."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(320, 180), (256, 256), (384, 216), (200, 150)]
RECIPES = [("print", 0x1001), ("vision3_500t_2383", 0x1002), ("ektar100_endura", 0x1003)]


@pytest.fixture(scope="module")
def batch_recipes(prepare):
    import os

    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    return {name: prepare.PreparedRecipe.load(os.path.join(golden, f"recipe_{name}.npz")) for name, _ in RECIPES}


def _records(batch_recipes, n=6):
    from film_juicer_b200 import frame_records, grain_plan

    noise = grain_plan.synthetic_noise()
    recs = []
    for i in range(n):
        name, rh = RECIPES[i % len(RECIPES)]
        w, h = SIZES[i % len(SIZES)]
        recs.append(frame_records.FrameRecord(batch_recipes[name], w, h, recipe_hash=rh, noise=noise,
                                              descriptor_width=w * 8))
    return recs


def _sources(torch, prepare, recs, seed):
    return [torch.from_numpy(np.ascontiguousarray(prepare.synthetic_frame(r.width, r.height, seed=seed + i))).cuda()
            for i, r in enumerate(recs)]


def _single(torch, owner, recs, srcs):
    """The frames one by one through fj_cuda_render on `owner`."""
    outs, res = [], []
    for r, s in zip(recs, srcs):
        d = torch.full_like(s, -1.0)
        res.append(owner.render(r, s, d))
        outs.append(d.cpu().numpy())
    return outs, res


def test_batch_matches_single_frames_eager_and_graph(torch_cuda, batch_recipes, prepare):
    from film_juicer_b200 import load_library, runtime

    torch = torch_cuda
    recs = _records(batch_recipes)
    srcs = _sources(torch, prepare, recs, 20261211)
    stream = torch.cuda.Stream()
    lib = load_library()
    with runtime.Owner() as single:
        want, want_res = _single(torch, single, recs, srcs)
    with runtime.Owner() as owner:
        dsts = [torch.full_like(s, -1.0) for s in srcs]
        outs = owner.render_batch(recs, srcs, dsts, stream)  # eager
        stream.synchronize()
        for i, d in enumerate(dsts):
            assert np.array_equal(d.cpu().numpy(), want[i]), i
            assert outs[i].flags == want_res[i].flags and outs[i].status.category == 0
        # graph: the first call with a token renders eagerly and captures
        for d in dsts:
            d.fill_(-1.0)
        torch.cuda.synchronize()
        owner.render_batch(recs, srcs, dsts, stream, graph_token=7)
        assert owner.last_batch_text == ""  # the graph was captured
        stream.synchronize()
        for i, d in enumerate(dsts):
            assert np.array_equal(d.cpu().numpy(), want[i]), i
        # new pixel contents in the same buffers; the replay launches nothing from the host
        new = _sources(torch, prepare, recs, 20261299)
        for s, n in zip(srcs, new):
            s.copy_(n)
        torch.cuda.synchronize()
        # per-frame renders on the same owner leave its caches and the graph alone
        want2, _ = _single(torch, owner, recs, [n.clone() for n in new])
        for d in dsts:
            d.fill_(-1.0)
        torch.cuda.synchronize()
        before = int(lib.fjb_kernel_launches())
        outs = owner.render_batch(recs, srcs, dsts, stream, graph_token=7)
        after = int(lib.fjb_kernel_launches())
        assert after == before
        stream.synchronize()
        for i, d in enumerate(dsts):
            assert np.array_equal(d.cpu().numpy(), want2[i]), i
            assert outs[i].status.category == 0
        assert any(float(np.abs(a - b).max()) > 1e-3 for a, b in zip(want, want2))


def test_autotuned_diffusion_form(torch_cuda, batch_recipes, prepare):
    from film_juicer_b200 import abi, runtime

    torch = torch_cuda
    recs = _records(batch_recipes, n=2)
    srcs = _sources(torch, prepare, recs, 20261212)
    with runtime.Owner() as single:
        want, _ = _single(torch, single, recs, srcs)
    stream = torch.cuda.Stream()
    with runtime.Owner() as owner:
        owner.set_autotune(True)
        for r in recs:
            assert owner.diffusion_form(r.width, r.height, r.host.h.optics.camera.radius_px) == -1
        dsts = [torch.full_like(s, -1.0) for s in srcs]
        owner.render_batch(recs, srcs, dsts, stream)
        stream.synchronize()
        for i, r in enumerate(recs):
            form = owner.diffusion_form(r.width, r.height, r.host.h.optics.camera.radius_px)
            assert form in (abi.FJB_DIFFUSION_DIRECT, abi.FJB_DIFFUSION_FFT)
            got = dsts[i].cpu().numpy()
            assert np.all(np.isfinite(got))
            assert float(np.abs(got - want[i]).max()) <= 2e-3


def test_batch_rejects_before_any_work(torch_cuda, batch_recipes, recipes, prepare):
    from film_juicer_b200 import abi, frame_records, runtime

    torch = torch_cuda
    recs = _records(batch_recipes, n=2)
    # enlarger diffusion on a direct route: rejected as fj_cuda_render rejects it
    recs.append(frame_records.FrameRecord(recipes["direct"], 160, 90, recipe_hash=0x1004, enlarger=True,
                                          descriptor_width=1280))
    srcs = _sources(torch, prepare, recs, 20261213)
    dsts = [torch.full_like(s, -1.0) for s in srcs]
    stream = torch.cuda.Stream()
    with runtime.Owner() as owner:
        with pytest.raises(runtime.FjError) as e:
            owner.render_batch(recs, srcs, dsts, stream)
        assert e.value.status.category == abi.FJ_STATUS_UNSUPPORTED_INPUT
        stream.synchronize()
        for d in dsts:
            assert float(d.max()) == -1.0  # nothing ran
