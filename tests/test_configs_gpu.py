"""Parity at the sizes of the path's benchmark configurations, against the reference's
own CUDA kernels (compiled from its sources into oracle/_ref/libjuicer_ref.so).

* Configuration 1: 512 x 512, kodak_portra_400 direct scan (Hanatos TC LUT, scanner
  LUT r = 17, sRGB, no spatial stage): the fused per-pixel chain
  (fjb_render_pixels) against juicer_cuda_negative_pipeline
  (src/Cuda/Scan/JuicerCudaScanPipeline.cu:2244), with error flags equal.
* Configuration 2: 1920 x 1080, kodak_portra_400 -> kodak_portra_endura, stage by
  stage with the frame's own descriptors (35 mm gate, 18.23 um pixels):
  - visual grain (35 mm, fixed seeds, production-shaped noise): bit-identical to
    juicer_cuda_apply_visual_grain (:3141) on the capture density of the frame;
  - scatter / halation on the frame's camera exposure: launch_scatter_halation
    (src/Cuda/Film/JuicerCudaScatterHalation.cu:690);
  - spatial DIR, 200 um tail at weight 0.03: juicer_cuda_build_print_spatial_dir
    (src/Cuda/Film/JuicerCudaFilmPipeline.cu:1479);
  - capture density and the print / scan / output chain: the reference's focused
    capture density (:2894) and print pipeline (:3759).
Bounds are the ones the stage tests state: the reference's processor-pixel bound
2e-4 + 3e-4 |ref| on encoded output, 1e-4 + 1e-4 |ref| on density, 2e-5 + 2e-5 |ref|
on halation planes, 1e-6 + 1e-5 |ref| on DIR corrections."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
W2, H2 = 1920, 1080


@pytest.fixture(scope="module")
def ref_lib(oracle):
    lib = oracle.load_reference()
    if lib is None:
        pytest.skip("reference CUDA harness not built (needs the reference sources at build time)")
    return lib


@pytest.fixture(scope="module")
def frame2(recipes, prepare):
    from film_juicer_b200 import frame_records

    rec = frame_records.FrameRecord(recipes["print"], W2, H2)
    src = np.ascontiguousarray(prepare.synthetic_frame(W2, H2, seed=20261203 + 1))
    return rec, src


def _ref_render(torch, ref_lib, oracle, rec, src):
    lut = oracle.scanner_lut_for(rec)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    s = torch.from_numpy(src).cuda()
    d = torch.zeros_like(s)
    flags = C.c_uint32()
    h, w, comps = src.shape
    rc = ref_lib.ref_render(rec.pointer(), ptrs, C.c_void_p(s.data_ptr()), w * comps * 4, C.c_void_p(d.data_ptr()),
                            w * comps * 4, w, h, comps, C.byref(flags))
    assert rc == 0, f"reference launcher returned cudaError {rc}"
    return d.cpu().numpy(), int(flags.value)


def _within(a, b, atol, rtol):
    err = np.abs(a - b)
    return bool(np.all(err <= atol + rtol * np.abs(b))), float(err.max())


@pytest.mark.parametrize("route", ["direct", "print"])
def test_config1_512_fused_chain_matches_reference(torch_cuda, ref_lib, oracle, recipes, prepare, route):
    torch = torch_cuda
    from film_juicer_b200 import runtime

    rec = prepare.HostRecord(recipes[route])
    assert rec.h.scanner_lut.resolution == 17
    src = np.ascontiguousarray(prepare.synthetic_frame(512, 512, seed=20261203))
    ref, rflags = _ref_render(torch, ref_lib, oracle, rec, src)
    dr = runtime.DeviceRecipe(rec)
    s = torch.from_numpy(src).cuda()
    d = torch.empty_like(s)
    dr.clear_flags()
    dr.render(s, d)
    flags = dr.read_flags()
    dr.close()
    assert flags == rflags
    ok, worst = _within(d.cpu().numpy(), ref, 2e-4, 3e-4)
    assert ok, worst


def test_config2_print_chain_at_1080p_matches_reference(torch_cuda, ref_lib, oracle, recipes, prepare, frame2):
    torch = torch_cuda
    from film_juicer_b200 import runtime

    _, src = frame2
    rec = prepare.HostRecord(recipes["print"])
    ref, rflags = _ref_render(torch, ref_lib, oracle, rec, src)
    dr = runtime.DeviceRecipe(rec)
    s = torch.from_numpy(src).cuda()
    d = torch.empty_like(s)
    dr.clear_flags()
    dr.render(s, d)
    assert dr.read_flags() == rflags
    dr.close()
    ok, worst = _within(d.cpu().numpy(), ref, 2e-4, 3e-4)
    assert ok, worst


def test_config2_capture_density_at_1080p_matches_reference(torch_cuda, ref_lib, oracle, recipes, prepare, frame2):
    torch = torch_cuda
    from film_juicer_b200 import runtime

    _, src = frame2
    rec = prepare.HostRecord(recipes["print"])
    lut = oracle.scanner_lut_for(rec)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    s = torch.from_numpy(src).cuda()
    ref_planes = [torch.zeros((H2, W2), device="cuda") for _ in range(3)]
    rc = ref_lib.ref_capture_density(rec.pointer(), ptrs, C.c_void_p(s.data_ptr()), W2 * 12, W2, H2, 3,
                                     *[C.c_void_p(p.data_ptr()) for p in ref_planes])
    assert rc == 0
    dr = runtime.DeviceRecipe(rec)
    mine = [torch.empty((H2, W2), device="cuda") for _ in range(3)]
    dr.capture_density(s, mine)
    torch.cuda.synchronize()
    dr.close()
    for a, b in zip(mine, ref_planes):
        ok, worst = _within(a.cpu().numpy(), b.cpu().numpy(), 1e-4, 1e-4)
        assert ok, worst


def test_config2_grain_at_1080p_is_bit_identical(torch_cuda, recipes, prepare, oracle, frame2):
    """The 35 mm grain of the 1080p frame, on the frame's capture density, with the
    production-shaped noise: every float of the three planes equal."""
    torch = torch_cuda
    from film_juicer_b200 import runtime
    from oracle import grain as og

    rec, src = frame2
    recipe = recipes["print"]
    a = recipe.arrays
    layers = [[a["density_layers"][:, l, c] for c in range(3)] for l in range(3)]
    base = [a["density_rgb"][:, c] for c in range(3)]
    dr = runtime.DeviceRecipe(prepare.HostRecord(recipe))
    s = torch.from_numpy(src).cuda()
    dens = [torch.empty((H2, W2), device="cuda") for _ in range(3)]
    dr.capture_density(s, dens)
    torch.cuda.synchronize()
    planes = [t.cpu().numpy() for t in dens]
    grain = rec.host.h.grain
    ref = og.reference_visual_grain(torch, grain, rec.noise.record, base, layers, False, planes)
    if ref is None:
        pytest.skip("reference CUDA harness not built")
    dnoise = runtime.DeviceNoise(rec.noise.record)
    runtime.visual_grain(dr, grain, dens, dnoise)
    torch.cuda.synchronize()
    dr.close()
    for c in range(3):
        got = dens[c].cpu().numpy()
        assert float(np.abs(got - planes[c]).max()) > 1e-3  # grain was applied
        diff = got.view(np.uint32) != ref[c].view(np.uint32)
        assert not diff.any(), (c, int(diff.sum()), float(np.abs(got - ref[c]).max()))


def test_config2_halation_at_1080p_matches_reference(torch_cuda, recipes, prepare, oracle, frame2):
    torch = torch_cuda
    from film_juicer_b200 import runtime
    from oracle import optics

    rec, src = frame2
    d = rec.host.h.optics.scatter_halation
    dr = runtime.DeviceRecipe(prepare.HostRecord(recipes["print"]))
    s = torch.from_numpy(src).cuda()
    carrier = [torch.empty((H2, W2), device="cuda") for _ in range(3)]  # B, G, R
    dr.camera_exposure(s, carrier)
    torch.cuda.synchronize()
    dr.close()
    rgb = [carrier[2].cpu().numpy(), carrier[1].cpu().numpy(), carrier[0].cpu().numpy()]
    ref = optics.reference_scatter_halation(torch, d, rgb)
    if ref is None:
        pytest.skip("reference CUDA harness not built")
    dev = [torch.from_numpy(p).cuda() for p in rgb]
    runtime.scatter_halation(d, dev)
    torch.cuda.synchronize()
    for g, r in zip(dev, ref):
        ok, worst = _within(g.cpu().numpy(), r, 2e-5, 2e-5)
        assert ok, worst


def test_config2_spatial_dir_at_1080p_matches_reference(torch_cuda, recipes, prepare, oracle, frame2):
    torch = torch_cuda
    from film_juicer_b200 import runtime
    from oracle import dir as odir

    rec, src = frame2
    sd = rec.host.h.spatial_dir
    host = prepare.HostRecord(recipes["print"])
    ref = odir.reference_spatial_dir(torch, host, sd, src)
    if ref is None:
        pytest.skip("reference CUDA harness not built")
    ref_f, ref_l = ref
    dr = runtime.DeviceRecipe(host)
    s = torch.from_numpy(src).cuda()
    filt = [torch.empty((H2, W2), device="cuda") for _ in range(3)]
    lraw = [torch.empty((H2, W2), device="cuda") for _ in range(3)]
    dr.spatial_dir_build(sd, filt, lraw, src=s)
    torch.cuda.synchronize()
    dr.close()
    for g, r in zip(filt, ref_f):
        ok, worst = _within(g.cpu().numpy(), r, 1e-6, 1e-5)
        assert ok, worst
    for g, r in zip(lraw, ref_l):
        ok, worst = _within(g.cpu().numpy(), r, 1e-6, 1e-6)
        assert ok, worst
