"""The positive route: a reversal stock (fujifilm_provia_100f) scanned directly
(FJ_ROUTE_POSITIVE_DIRECT, tests/golden/recipe_positive.npz), whose DIR couplers run in
the receiver-Langmuir mode (the receivers' references and knees, the donors as the
density maximum minus the layer density).

* the fused per-pixel chain (fjb_render_pixels) against the reference's CUDA
  (juicer_cuda_negative_pipeline, src/Cuda/Scan/JuicerCudaScanPipeline.cu:2244, which
  scans every direct route) at 512 x 512: error flags equal, encoded output within the
  reference's processor-pixel bound 2e-4 + 3e-4 |ref|, and against the oracle;
* capture density (fjb_capture_density) against the reference's focused capture
  density (:2894), 1e-4 + 1e-4 |ref|;
* spatial DIR of a 35 mm frame (source + filter) against the reference's launcher
  (src/Cuda/Film/JuicerCudaFilmPipeline.cu:1479), 1e-6 + 1e-5 |ref|, and the whole staged
  frame (fj_cuda_render: spatial DIR with the receiver finalisation, grain) finite."""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
W, H = 512, 512


@pytest.fixture(scope="module")
def positive(prepare):
    here = os.path.dirname(os.path.abspath(__file__))
    r = prepare.PreparedRecipe.load(os.path.join(here, "golden", "recipe_positive.npz"))
    from film_juicer_b200 import abi

    assert r.route == abi.FJ_ROUTE_POSITIVE_DIRECT
    assert r.scalars["dir_mode"] == abi.FJ_DIR_POSITIVE_RECEIVER_LANGMUIR
    return r


@pytest.fixture(scope="module")
def ref_lib(oracle):
    lib = oracle.load_reference()
    if lib is None:
        pytest.skip("reference CUDA harness not built (needs the reference sources at build time)")
    return lib


def _within(a, b, atol, rtol):
    err = np.abs(a - b)
    return bool(np.all(err <= atol + rtol * np.abs(b))), float(err.max())


def test_positive_fused_chain_matches_reference_and_oracle(torch_cuda, ref_lib, oracle, positive, prepare):
    from film_juicer_b200 import runtime

    torch = torch_cuda
    rec = prepare.HostRecord(positive)
    src = np.ascontiguousarray(prepare.synthetic_frame(W, H, seed=20261207))
    lut = oracle.scanner_lut_for(rec)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    s = torch.from_numpy(src).cuda()
    ref_d = torch.zeros_like(s)
    rflags = C.c_uint32()
    rc = ref_lib.ref_render(rec.pointer(), ptrs, C.c_void_p(s.data_ptr()), W * 12, C.c_void_p(ref_d.data_ptr()),
                            W * 12, W, H, 3, C.byref(rflags))
    assert rc == 0
    dr = runtime.DeviceRecipe(rec)
    d = torch.empty_like(s)
    dr.clear_flags()
    dr.render(s, d)
    flags = dr.read_flags()
    dr.close()
    got = d.cpu().numpy()
    assert flags == int(rflags.value)
    ok, worst = _within(got, ref_d.cpu().numpy(), 2e-4, 3e-4)
    assert ok, worst
    want, oflags = oracle.render(rec, src[:192, :256].copy())
    ok, worst = _within(got[:192, :256], want, 2e-4, 3e-4)
    assert ok, worst
    assert np.all(np.isfinite(got))


def test_positive_capture_density_matches_reference(torch_cuda, ref_lib, oracle, positive, prepare):
    from film_juicer_b200 import runtime

    torch = torch_cuda
    rec = prepare.HostRecord(positive)
    src = np.ascontiguousarray(prepare.synthetic_frame(W, H, seed=20261208))
    lut = oracle.scanner_lut_for(rec)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    s = torch.from_numpy(src).cuda()
    ref_planes = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    rc = ref_lib.ref_capture_density(rec.pointer(), ptrs, C.c_void_p(s.data_ptr()), W * 12, W, H, 3,
                                     *[C.c_void_p(p.data_ptr()) for p in ref_planes])
    assert rc == 0
    dr = runtime.DeviceRecipe(rec)
    mine = [torch.empty((H, W), device="cuda") for _ in range(3)]
    dr.capture_density(s, mine)
    torch.cuda.synchronize()
    dr.close()
    for a, b in zip(mine, ref_planes):
        ok, worst = _within(a.cpu().numpy(), b.cpu().numpy(), 1e-4, 1e-4)
        assert ok, worst


def test_positive_spatial_dir_and_frame(torch_cuda, positive, prepare, oracle):
    from film_juicer_b200 import frame_records, runtime
    from oracle import dir as odir

    torch = torch_cuda
    fw, fh = 640, 426
    rec = frame_records.FrameRecord(positive, fw, fh, recipe_hash=0x3001, descriptor_width=fw * 6)
    sd = rec.host.h.spatial_dir
    assert sd.component_count > 0
    src = np.ascontiguousarray(prepare.synthetic_frame(fw, fh, seed=20261209))
    host = prepare.HostRecord(positive)
    ref = odir.reference_spatial_dir(torch, host, sd, src)
    if ref is None:
        pytest.skip("reference CUDA harness not built")
    ref_f, ref_l = ref
    dr = runtime.DeviceRecipe(host)
    s = torch.from_numpy(src).cuda()
    filt = [torch.empty((fh, fw), device="cuda") for _ in range(3)]
    lraw = [torch.empty((fh, fw), device="cuda") for _ in range(3)]
    dr.spatial_dir_build(sd, filt, lraw, src=s)
    torch.cuda.synchronize()
    dr.close()
    for g, r in zip(filt, ref_f):
        ok, worst = _within(g.cpu().numpy(), r, 1e-6, 1e-5)
        assert ok, worst
    # the whole staged frame on the positive route
    with runtime.Owner() as owner:
        dst = torch.full_like(s, -1.0)
        out = owner.render(rec, s, dst)
        assert out.status.category == 0
        torch.cuda.synchronize()
        assert bool(torch.isfinite(dst).all())
        assert float(dst.min()) >= 0.0
