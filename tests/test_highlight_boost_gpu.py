"""Highlight reconstruction (the second of the path's next rows) on the camera carrier:
the frame maximum over the three planes, then the normalised-exponential lift of every
sample above the protection level so that the maximum lands on maximum * peak_gain.

Against the reference's own CUDA launcher (launch_highlight_boost, compiled for sm_100a):
bit-identical planes and the same disposition on every case, both branches of the curve
(shape below and above 0.5), bypass, peak overflow and invalid carriers. Against the
oracle's restatement: 2 ulp-scale relative bound (it rounds without fused multiply-adds
and uses the host libm's exp/expm1). Through fj_cuda_render: a frame with the boost
against the oracle's stage chain."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = {
    # name: (protection, sharpness, peak_gain, disposition)
    "applied_soft": (0.8, 0.3, 1.5, 1),
    "applied_sharp": (0.5, 6.0, 3.0, 1),
    "applied_high_protection": (3.5, 2.0, 1.2, 1),
    "bypass": (100.0, 2.0, 2.0, 0),
    "peak_overflow": (0.5, 2.0, 1e38, 3),
}


def carrier(seed, w=131, h=77, bad=None):
    rng = np.random.default_rng(seed)
    planes = [rng.gamma(2.0, 0.35, size=(h, w)).astype(np.float32) for _ in range(3)]
    planes[1][h // 3, w // 2] = 6.5  # the frame maximum
    planes[0][5, 7] = 4.0
    if bad is not None:
        planes[2][2, 3] = bad
    return planes


@pytest.fixture(scope="module")
def ref_lib(oracle):
    lib = oracle.load_reference()
    if lib is None or not hasattr(lib, "ref_highlight_boost"):
        pytest.skip("reference CUDA harness not built with the highlight boost")
    return lib


@pytest.mark.parametrize("name", list(CASES))
def test_matches_reference_cuda(torch_cuda, ref_lib, name):
    torch = torch_cuda
    from film_juicer_b200 import descriptors, runtime
    from oracle import optics

    prot, sharp, gain, want = CASES[name]
    d = descriptors.highlight_boost_record(prot, sharp, gain)
    host = carrier(1)
    mine = [torch.from_numpy(p).cuda() for p in host]
    ref = [torch.from_numpy(p).cuda() for p in host]
    rd = optics.reference_highlight_boost(torch, d, ref)
    assert rd == want
    if want in (0, 1):
        assert runtime.highlight_boost(d, mine) == want
    else:
        with pytest.raises(runtime.FjError, match="PeakOverflow"):
            runtime.highlight_boost(d, mine)
    torch.cuda.synchronize()
    for a, b in zip(mine, ref):
        assert torch.equal(a, b), name


@pytest.mark.parametrize("bad", [-0.25, float("nan"), float("inf")])
def test_invalid_carrier_matches_reference(torch_cuda, ref_lib, bad):
    torch = torch_cuda
    from film_juicer_b200 import descriptors, runtime
    from oracle import optics

    d = descriptors.highlight_boost_record(0.8, 2.0, 2.0)
    host = carrier(2, bad=bad)
    ref = [torch.from_numpy(p).cuda() for p in host]
    assert optics.reference_highlight_boost(torch, d, ref) == 2
    mine = [torch.from_numpy(p).cuda() for p in host]
    with pytest.raises(runtime.FjError, match="InvalidCarrier"):
        runtime.highlight_boost(d, mine)


@pytest.mark.parametrize("name", ["applied_soft", "applied_sharp", "applied_high_protection", "bypass"])
def test_matches_oracle(torch_cuda, name):
    torch = torch_cuda
    from film_juicer_b200 import descriptors, runtime
    from oracle import optics

    prot, sharp, gain, want = CASES[name]
    d = descriptors.highlight_boost_record(prot, sharp, gain)
    host = carrier(3)
    mine = [torch.from_numpy(p).cuda() for p in host]
    assert runtime.highlight_boost(d, mine) == want
    ref, disp = optics.highlight_boost(d, host)
    assert disp == want
    for a, b in zip(mine, ref):
        a = a.cpu().numpy()
        assert np.all(np.abs(a - b) <= 4e-7 * np.maximum(1.0, np.abs(b))), (name, float(np.abs(a - b).max()))


def test_frame_schedule_with_boost_matches_oracle_chain(torch_cuda, recipes, prepare):
    from film_juicer_b200 import descriptors, frame_records, runtime
    from oracle import frame as oframe

    torch = torch_cuda
    w, h = 120, 72
    rec = frame_records.FrameRecord(recipes["print"], w, h, grain=False,
                                    highlight_boost=descriptors.highlight_boost_record(0.05, 3.0, 1.8))
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=20261205))
    s = torch.from_numpy(src).cuda()
    d = torch.full_like(s, -1.0)
    with runtime.Owner() as owner:
        owner.render(rec, s, d)
    got = d.cpu().numpy()
    want, _ = oframe.render_frame(rec, recipes["print"], src)
    plain, _ = oframe.render_frame(frame_records.FrameRecord(recipes["print"], w, h, grain=False), recipes["print"], src)
    assert float(np.abs(want - plain).max()) > 1e-3  # the boost changes the frame
    err = np.abs(got - want)
    assert np.all(err <= 2e-4 + 3e-4 * np.abs(want)), float(err.max())
