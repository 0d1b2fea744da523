"""GPU parity of the fused per-pixel chain (a1..a13) against the CPU oracle.

Tolerance: the reference's own bound for CUDA processor pixels,
|gpu - oracle| <= 2e-4 + 3e-4 |oracle| per encoded output channel
(tests/README.md:937 of the reference), and 1e-4 + 1e-4 |oracle| on dye density.
The GPU uses CUDA's exp2f/log10f/powf/cbrtf and fused multiply-adds, the oracle
glibc's and separately rounded operations, so results agree to FP32 rounding, not
bit for bit; interval/LUT-cell selection is exact for identical inputs.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OUT_ATOL, OUT_RTOL = 2e-4, 3e-4
DENS_ATOL, DENS_RTOL = 1e-4, 1e-4
SIZES = [(1, 1), (7, 5), (17, 19), (1, 64), (64, 1), (256, 192)]


def close(got, ref, atol, rtol):
    bad = np.abs(got - ref) > atol + rtol * np.abs(ref)
    return int(bad.sum()), float(np.max(np.abs(got - ref))) if got.size else 0.0


@pytest.fixture(scope="module")
def device_recipes(torch_cuda, recipes, prepare):
    from film_juicer_b200 import runtime

    out = {}
    for name, r in recipes.items():
        rec = prepare.HostRecord(r)
        out[name] = (rec, runtime.DeviceRecipe(rec))
    yield out
    for _, dr in out.values():
        dr.close()


def frame(prepare, w, h, comps, seed=20261203):
    src = prepare.synthetic_frame(w, h, seed=seed)
    if comps == 4:
        alpha = np.linspace(0, 1, w * h, dtype=np.float32).reshape(h, w, 1)
        src = np.concatenate([src, alpha], axis=2)
    return np.ascontiguousarray(src)


@pytest.mark.parametrize("route", ["direct", "print"])
@pytest.mark.parametrize("comps", [3, 4])
@pytest.mark.parametrize("size", SIZES, ids=[f"{w}x{h}" for w, h in SIZES])
def test_render_pixels_matches_oracle(torch_cuda, device_recipes, prepare, oracle, route, comps, size):
    torch = torch_cuda
    rec, dr = device_recipes[route]
    w, h = size
    src = frame(prepare, w, h, comps)
    s = torch.from_numpy(src).cuda()
    d = torch.full_like(s, -7.0)
    dr.clear_flags()
    dr.render(s, d)
    flags = dr.read_flags()
    got = d.cpu().numpy()
    ref, rflags = oracle.render(rec, src)
    assert flags == rflags
    nbad, worst = close(got[..., :3], ref[..., :3], OUT_ATOL, OUT_RTOL)
    assert nbad == 0, f"{nbad} channels outside tolerance, worst {worst}"
    if comps == 4:
        assert np.array_equal(got[..., 3], src[..., 3])


@pytest.mark.parametrize("route", ["direct", "print"])
def test_capture_density_matches_oracle(torch_cuda, device_recipes, prepare, oracle, route):
    torch = torch_cuda
    rec, dr = device_recipes[route]
    src = frame(prepare, 160, 90, 3)
    s = torch.from_numpy(src).cuda()
    planes = [torch.empty((90, 160), device="cuda") for _ in range(3)]
    dr.capture_density(s, planes)
    got = [p.cpu().numpy() for p in planes]
    ref, _ = oracle.render(rec, src, stage=1)
    for g, r in zip(got, ref):
        nbad, worst = close(g, r, DENS_ATOL, DENS_RTOL)
        assert nbad == 0, worst


@pytest.mark.parametrize("route", ["direct", "print"])
def test_staged_equals_fused_bitwise(torch_cuda, device_recipes, prepare, route):
    """capture density -> planes -> scan is the fused chain split at a plane boundary."""
    torch = torch_cuda
    _, dr = device_recipes[route]
    src = frame(prepare, 123, 77, 4)
    s = torch.from_numpy(src).cuda()
    fused = torch.empty_like(s)
    dr.render(s, fused)
    planes = [torch.empty((77, 123), device="cuda") for _ in range(3)]
    dr.capture_density(s, planes)
    staged = torch.empty_like(s)
    dr.render_from_density(planes, s, staged)
    torch.cuda.synchronize()
    assert torch.equal(fused, staged)


@pytest.mark.parametrize("route", ["direct", "print"])
def test_carrier_path_matches_oracle(torch_cuda, device_recipes, prepare, oracle, route):
    torch = torch_cuda
    rec, dr = device_recipes[route]
    src = frame(prepare, 64, 48, 3)
    s = torch.from_numpy(src).cuda()
    carrier = [torch.empty((48, 64), device="cuda") for _ in range(3)]
    dr.camera_exposure(s, carrier)
    got_e = [c.cpu().numpy() for c in carrier]
    ref_e, _ = oracle.render(rec, src, stage=3)
    for g, r in zip(got_e, ref_e):
        assert close(g, r, 1e-6, 2e-5)[0] == 0
    out = torch.empty_like(s)
    dr.render_carrier(carrier, s, out)
    ref, _ = oracle.render(rec, None, stage=4, planes=ref_e)
    nbad, worst = close(out.cpu().numpy(), ref, OUT_ATOL, OUT_RTOL)
    assert nbad == 0, worst


def test_dir_failure_sets_deferred_flag(torch_cuda, recipes, prepare, oracle):
    """An invalid donor knee on the green layer makes its Langmuir term fail; the NaN
    donor then reaches every receiver through the coupler matrix, so bit 8 plus the
    full B,G,R channel mask is raised (src/Cuda/JuicerCudaDeviceHelpers.cuh:1125-1204),
    the pixel's density becomes NaN and the scan reports failure (bit 0), writing
    black."""
    torch = torch_cuda
    from film_juicer_b200 import runtime

    rec = prepare.HostRecord(recipes["direct"])
    rec.h.dir_couplers.donor_k_rgb[1] = -1.0
    dr = runtime.DeviceRecipe(rec)
    src = frame(prepare, 16, 8, 3)
    s = torch.from_numpy(src).cuda()
    d = torch.empty_like(s)
    dr.clear_flags()
    dr.render(s, d)
    flags = dr.read_flags()
    ref, rflags = oracle.render(rec, src)
    assert flags == rflags
    assert flags & (1 << 8) and (flags >> 9) & 7 == 0b111 and flags & 1
    assert np.array_equal(d.cpu().numpy(), ref)
    dr.close()


def test_zero_sized_frame_is_a_no_op(torch_cuda, device_recipes):
    torch = torch_cuda
    _, dr = device_recipes["print"]
    s = torch.zeros((1, 1, 3), device="cuda")
    d = torch.full_like(s, 5.0)
    from film_juicer_b200 import abi

    err = abi.ErrorText()
    st = dr.lib.fjb_render_pixels(dr.handle, C.c_void_p(s.data_ptr()), 12, C.c_void_p(d.data_ptr()), 12, 0, 0, 3,
                                  None, C.byref(err.buf))
    assert st.category == 0
    torch.cuda.synchronize()
    assert float(d.item() if d.numel() == 1 else d[0, 0, 0]) == 5.0 or True
    assert torch.all(d == 5.0)


def test_fj_cuda_render_whole_frame(torch_cuda, recipes, prepare, oracle):
    """The drop-in entry point: create -> inspect -> render (sub-window) -> destroy."""
    torch = torch_cuda
    from film_juicer_b200 import abi, load_library

    lib = load_library()
    rec = prepare.HostRecord(recipes["print"], recipe_hash=0x1234)
    H, W = 40, 56
    src = frame(prepare, W, H, 4)
    s = torch.from_numpy(src).cuda()
    d = torch.full_like(s, -1.0)
    err = abi.ErrorText()
    owner = C.c_void_p()
    assert lib.fj_cuda_create(C.byref(owner), C.byref(err.buf)).category == 0
    second = C.c_void_p()
    assert lib.fj_cuda_create(C.byref(second), C.byref(err.buf)).category != 0  # one live owner
    fr = abi.FjFrame()
    for im, t in ((fr.source, s), (fr.destination, d)):
        im.address = t.data_ptr()
        im.bounds = abi.FjRect(0, 0, W, H)
        im.row_bytes = t.stride(0) * 4
        im.components = 4
        im.depth = abi.FJ_DEPTH_FLOAT32
    fr.render_window = abi.FjRect(3, 2, W - 5, H - 1)
    fr.full_frame_extent = abi.FjRect(0, 0, W, H)
    ctx = abi.FjCudaContext()
    assert lib.fj_cuda_inspect(owner, C.byref(fr), C.byref(ctx), C.byref(err.buf)).category == 0
    sub = abi.FjSubmission()
    cb = abi.FjAbortCallback(abi.FjAbortQuery(lambda user: abi.FJ_ABORT_CONTINUE), None)
    out = lib.fj_cuda_render(owner, C.byref(ctx), C.byref(fr), C.byref(sub), rec.pointer(), cb, C.byref(err.buf))
    assert out.status.category == 0, err.text
    got = d.cpu().numpy()
    ref, _ = oracle.render(rec, src)
    win = (slice(2, H - 1), slice(3, W - 5))
    assert close(got[win][..., :3], ref[win][..., :3], OUT_ATOL, OUT_RTOL)[0] == 0
    outside = np.ones((H, W), bool)
    outside[win] = False
    assert np.all(got[outside] == -1.0)
    # abort requested before any launch -> CANCELLED
    cb2 = abi.FjAbortCallback(abi.FjAbortQuery(lambda user: abi.FJ_ABORT_REQUESTED), None)
    out2 = lib.fj_cuda_render(owner, C.byref(ctx), C.byref(fr), C.byref(sub), rec.pointer(), cb2, C.byref(err.buf))
    assert out2.status.category == abi.FJ_STATUS_CANCELLED
    assert lib.fj_cuda_shutdown(owner, C.byref(err.buf)).category == 0
    assert lib.fj_cuda_check_terminal(owner, C.byref(err.buf)).category != 0
    assert lib.fj_cuda_destroy(owner, C.byref(err.buf)).category == 0
