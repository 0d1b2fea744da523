"""Enlarger diffusion (FJ_OPTICS_ENLARGER_DIFFUSION): the print-linear exposure of the
capture density, the enlarger's diffusion on it, print development from the diffused
exposure, then the scan of print density (src/Cuda/JuicerCudaExecutor.cpp:2292-2365).

* stage by stage against the reference's own kernels
  (src/Cuda/Scan/JuicerCudaScanPipeline.cu:2924 build_enlarger_print_linear_exposure,
  :2943 develop_print_density_from_enlarger_linear) and the oracle: the linear
  exposure (with and without a film-dust plane) within 1e-9 + 1e-4 |ref| (FP32 spectral
  sums in different orders), the print density within 1e-4 + 1e-4 |ref|;
* the whole frame through fj_cuda_render with enlarger diffusion, alone and with every
  other stage, against the oracle's chain, with the frame-schedule bound
  (2e-4 + 3e-4 |oracle| on at least 99 % of the pixels, mean below 1e-4), and it
  differs from the same frame without enlarger diffusion;
* FFT-form enlarger diffusion (radius 12 at 4K-scale pixels) through the frame."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ATOL, RTOL = 2e-4, 3e-4


def _density(torch, dr, prepare, w, h, seed=20261205):
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=seed))
    planes = [torch.empty((h, w), device="cuda") for _ in range(3)]
    dr.capture_density(torch.from_numpy(src).cuda(), planes)
    torch.cuda.synchronize()
    return planes


@pytest.mark.parametrize("with_dust", [False, True])
def test_enlarger_stages_match_reference_and_oracle(torch_cuda, recipes, prepare, oracle, with_dust):
    from film_juicer_b200 import runtime
    from oracle import optics

    torch = torch_cuda
    w, h = 240, 135
    rec = prepare.HostRecord(recipes["print"])
    dr = runtime.DeviceRecipe(rec)
    dens = _density(torch, dr, prepare, w, h)
    dust = None
    if with_dust:
        rng = np.random.default_rng(3)
        dust = torch.from_numpy(rng.uniform(0.6, 1.0, size=(h, w)).astype(np.float32)).cuda()
    lin = [torch.empty((h, w), device="cuda") for _ in range(3)]
    dr.enlarger_linear_exposure(dens, lin, dust=dust)
    torch.cuda.synchronize()
    got_lin = [t.cpu().numpy() for t in lin]
    dens_h = [t.cpu().numpy() for t in dens]
    dust_h = dust.cpu().numpy() if dust is not None else None
    want = optics.enlarger_linear(rec, dens_h, dust_h)
    ref = optics.reference_enlarger(torch, rec, 0, dens_h, dust_h)
    for k in range(3):
        assert np.all(np.isfinite(got_lin[k])) and float(got_lin[k].min()) > 0.0
        assert np.all(np.abs(got_lin[k] - want[k]) <= 1e-9 + 1e-4 * np.abs(want[k]))
        if ref is not None:
            assert np.all(np.abs(got_lin[k] - ref[k]) <= 1e-9 + 1e-4 * np.abs(ref[k])), float(
                np.abs(got_lin[k] - ref[k]).max())
    # development from (a blurred copy of) the linear exposure, in place
    blurred = [0.5 * p + 0.25 * np.roll(p, 1, axis=1) + 0.25 * np.roll(p, -1, axis=0) for p in got_lin]
    dev = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.float32)).cuda() for p in blurred]
    dr.enlarger_develop(dev, dev)
    torch.cuda.synchronize()
    got_d = [t.cpu().numpy() for t in dev]
    want_d = optics.enlarger_develop(rec, blurred)
    ref_d = optics.reference_enlarger(torch, rec, 1, blurred)
    for k in range(3):
        assert np.all(np.abs(got_d[k] - want_d[k]) <= 1e-4 + 1e-4 * np.abs(want_d[k]))
        if ref_d is not None:
            assert np.all(np.abs(got_d[k] - ref_d[k]) <= 1e-4 + 1e-4 * np.abs(ref_d[k]))
    dr.close()


@pytest.mark.parametrize("config", ["enlarger_only", "all_stages", "all_stages_and_post"])
def test_frame_with_enlarger_matches_oracle_chain(torch_cuda, recipes, prepare, config):
    from film_juicer_b200 import descriptors, frame_records, runtime
    from oracle import frame as oframe

    torch = torch_cuda
    w, h = 120, 72
    kw = dict(enlarger=True)
    if config == "enlarger_only":
        kw.update(diffusion=False, halation=False, spatial_dir=False, grain=False)
    if config == "all_stages_and_post":
        kw["post"] = descriptors.scanner_post_record(lens_blur_sigma_px=0.8, unsharp_sigma_px=0.7, unsharp_amount=0.7)
    # 4 um pixels so that the enlarger radius (0.3 % of a 3840-px gate) is 12 px: the FFT form
    rec = frame_records.FrameRecord(recipes["print"], w, h, descriptor_width=3840, **kw)
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=20261205))
    s = torch.from_numpy(src).cuda()
    d = torch.full_like(s, -1.0)
    with runtime.Owner() as owner:
        owner.render(rec, s, d)
    got = d.cpu().numpy()
    want, _ = oframe.render_frame(rec, recipes["print"], src)
    assert np.all(np.isfinite(got))
    err = np.abs(got - want)
    bad = err > ATOL + RTOL * np.abs(want)
    assert float(bad.mean()) <= 0.01, (config, float(bad.mean()), float(err.max()))
    assert float(err.mean()) <= 1e-4, (config, float(err.mean()))
    assert rec.host.h.optics.enlarger.radius_px == 12
    rec.host.h.optics.flags &= ~2
    d2 = torch.full_like(s, -1.0)
    with runtime.Owner() as owner:
        owner.render(rec, s, d2)
    assert float(np.abs(d2.cpu().numpy() - got).max()) > 1e-3
