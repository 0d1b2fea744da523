"""The print exposure's 81-wavelength contraction on the tensor cores (tcgen05 BF16
tiles with FP32 accumulation, fjb_print_tc.cu) against the FP32 form (the reference's
arithmetic, src/Cuda/JuicerCudaDeviceHelpers.cuh:866-935) and the oracle.

Bounds (stated per output, as the precision target asks):
* spectral integral raw_c (fjb_print_raw) per pixel and channel, relative to the FP32
  form: <= 2.5e-3 with one BF16 transmittance per wavelength (its rounding, 2^-9, is
  the largest term), <= 2e-4 with hi + lo transmittances (exponent carried to ~2^-17
  by the hi + lo density and spectrum pairs);
* encoded output: CIEDE2000 against the FP32 form and against the oracle p99 <= 0.5
  (the path's precision target);
* pixels with a non-finite density take the FP32 cold path: bit-identical raw;
* frames that are not a multiple of the 128-pixel tile, and the owner path
  (fjb_owner_set_print_form + fj_cuda_render)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FORMS = {"tensor": (1, 2.5e-3), "tensor_split": (2, 2e-4)}


@pytest.fixture(scope="module")
def print_recipe(torch_cuda, recipes, prepare):
    from film_juicer_b200 import runtime

    rec = prepare.HostRecord(recipes["print"])
    dr = runtime.DeviceRecipe(rec)
    yield rec, dr
    dr.close()


def _density(torch, dr, prepare, w, h, seed=20261205):
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=seed))
    s = torch.from_numpy(src).cuda()
    planes = [torch.empty((h, w), device="cuda") for _ in range(3)]
    dr.set_print_form(0)
    dr.capture_density(s, planes)
    return src, planes


def _raw(torch, dr, density, form):
    h, w = density[0].shape
    out = [torch.full((h, w), float("nan"), device="cuda") for _ in range(3)]
    dr.set_print_form(form)
    dr.print_raw(density, out)
    dr.set_print_form(0)
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in out]


@pytest.mark.parametrize("form", list(FORMS))
@pytest.mark.parametrize("size", [(1920, 1080), (61, 45), (1, 1), (127, 3)])
def test_spectral_integral_against_fp32_form(torch_cuda, print_recipe, prepare, form, size):
    torch = torch_cuda
    rec, dr = print_recipe
    w, h = size
    _, dens = _density(torch, dr, prepare, w, h)
    code, bound = FORMS[form]
    want = _raw(torch, dr, dens, 0)
    got = _raw(torch, dr, dens, code)
    for g, r in zip(got, want):
        assert np.all(np.isfinite(g))
        rel = np.abs(g - r) / np.maximum(np.abs(r), 1e-30)
        assert float(rel.max()) <= bound, (form, float(rel.max()), float(np.percentile(rel, 99)))


def test_non_finite_density_takes_the_fp32_path(torch_cuda, print_recipe, prepare):
    torch = torch_cuda
    rec, dr = print_recipe
    _, dens = _density(torch, dr, prepare, 300, 7)
    dens[0][2, 5] = float("nan")
    dens[1][4, 299] = float("inf")
    dens[2][0, 0] = float("-inf")
    want = _raw(torch, dr, dens, 0)
    for code in (1, 2):
        got = _raw(torch, dr, dens, code)
        for g, r in zip(got, want):
            for (y, x) in ((2, 5), (4, 299), (0, 0)):
                same = np.float32(g[y, x]).view(np.uint32) == np.float32(r[y, x]).view(np.uint32)
                assert same or (np.isnan(g[y, x]) and np.isnan(r[y, x]))


@pytest.mark.parametrize("form", list(FORMS))
def test_encoded_output_delta_e(torch_cuda, print_recipe, prepare, oracle, form):
    from oracle import color

    torch = torch_cuda
    rec, dr = print_recipe
    w, h = 480, 270
    src, dens = _density(torch, dr, prepare, w, h)
    outs = {}
    for name, code in (("fp32", 0), (form, FORMS[form][0])):
        d = torch.full((h, w, 3), -1.0, device="cuda")
        dr.set_print_form(code)
        dr.render_from_density(dens, None, d)
        outs[name] = d.cpu().numpy()
    dr.set_print_form(0)
    st = color.delta_e_stats(outs[form], outs["fp32"])
    assert st["p99"] <= 0.5, st
    ref, _ = oracle.render(rec, src, stage=2, planes=[p.cpu().numpy() for p in dens])
    st = color.delta_e_stats(outs[form], ref)
    assert st["p99"] <= 0.5, st


def test_owner_renders_the_frame_in_the_tensor_form(torch_cuda, recipes, prepare):
    from film_juicer_b200 import frame_records, runtime
    from oracle import color

    torch = torch_cuda
    w, h = 640, 360
    rec = frame_records.FrameRecord(recipes["print"], w, h)
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=20261205))
    s = torch.from_numpy(src).cuda()
    outs = []
    for form in (0, 1, 2):
        d = torch.full_like(s, -1.0)
        with runtime.Owner() as owner:
            owner.set_print_form(form)
            owner.render(rec, s, d)
        outs.append(d.cpu().numpy())
    for k in (1, 2):
        assert np.all(np.isfinite(outs[k]))
        st = color.delta_e_stats(outs[k], outs[0])
        assert st["p99"] <= 0.5, (k, st)
    # the split form is closer to the FP32 form than the single-BF16 one
    assert color.delta_e_stats(outs[2], outs[0])["p99"] <= color.delta_e_stats(outs[1], outs[0])["p99"] + 1e-6
