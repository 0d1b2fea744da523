"""Device time of each stage against the reference's own CUDA kernels on the same 4K
frame (the reference compiled for sm_100a into the test harness; its launchers timed
with CUDA events after every upload). Guards against regressions: no stage may be
slower than the reference's. Set FJB_SPEED_REPORT to a path to keep
the table as JSON."""
import ctypes as C
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H = 3840, 2160


def test_stage_times_against_reference_cuda(torch_cuda, recipes, prepare, oracle):
    torch = torch_cuda
    from film_juicer_b200 import abi, frame_records, load_library, runtime
    from oracle import dir as odir
    from oracle import grain as ograin
    from oracle import optics as ooptics

    ref = oracle.load_reference()
    if ref is None:
        pytest.skip("reference CUDA harness not built")
    ref.ref_last_ms.restype = C.c_float
    lib = load_library()
    recipe = recipes["print"]
    rec = frame_records.FrameRecord(recipe, W, H)
    src = np.ascontiguousarray(prepare.synthetic_frame(W, H, seed=20261205))
    s = torch.from_numpy(src).cuda()
    d = torch.empty_like(s)
    err = abi.ErrorText()
    ours = {}
    with runtime.Owner() as owner:
        owner.render(rec, s, d)
        lib.fjb_owner_stage_timing(owner.handle, 1, C.byref(err.buf))
        for _ in range(5):
            owner.render(rec, s, d)
        t = abi.FjbStageTimes()
        lib.fjb_owner_stage_times(owner.handle, C.byref(t), C.byref(err.buf))
        for i, name in enumerate(abi.FJB_STAGE_NAMES):
            if t.frames[i]:
                ours[name] = t.total_ms[i] / t.frames[i]
    # the fused per-pixel chain alone (no spatial stages)
    host = prepare.HostRecord(recipe)
    dr = runtime.DeviceRecipe(host)
    for _ in range(3):
        dr.render(s, d)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        dr.render(s, d)
    e1.record()
    e1.synchronize()
    ours["monolithic"] = e0.elapsed_time(e1) / 10
    dr.close()

    theirs = {}
    lut = oracle.scanner_lut_for(host)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    flags = C.c_uint32()
    for _ in range(2):
        assert ref.ref_render(host.pointer(), ptrs, C.c_void_p(s.data_ptr()), W * 12, C.c_void_p(d.data_ptr()),
                              W * 12, W, H, 3, C.byref(flags)) == 0
    theirs["monolithic"] = ref.ref_last_ms()
    planes = [np.ascontiguousarray(prepare.synthetic_frame(W, H, seed=c)[..., 0]) for c in range(3)]
    for _ in range(2):
        ooptics.reference_scatter_halation(torch, rec.host.h.optics.scatter_halation, planes)
    theirs["scatter_halation"] = ref.ref_last_ms()
    for _ in range(2):
        odir.reference_spatial_dir(torch, rec.host, rec.host.h.spatial_dir, src)
    theirs["spatial_dir"] = ref.ref_last_ms()
    a = recipe.arrays
    layers = [[a["density_layers"][:, l, c] for c in range(3)] for l in range(3)]
    base = [a["density_rgb"][:, c] for c in range(3)]
    dens = [np.ascontiguousarray(np.clip(p * 2.0, 0.05, 2.5)) for p in planes]
    for _ in range(2):
        ograin.reference_visual_grain(torch, rec.host.h.grain, rec.noise.record, base, layers, False, dens)
    theirs["grain"] = ref.ref_last_ms()

    # film defects and the gate mask at 4K (the bench's next-rows record)
    if hasattr(ref, "ref_defects_timed"):
        from film_juicer_b200 import descriptors

        fx = descriptors.default_film_effects(W, H)
        fdens = [torch.from_numpy(p).cuda() for p in dens]
        dust = torch.empty((H, W), device="cuda")
        mask = torch.empty((fx.gate_height, fx.gate_width), device="cuda")
        need = max(int(lib.fjb_film_defects_scratch_bytes(C.byref(fx), W, H)),
                   int(lib.fjb_gate_mask_scratch_bytes(C.byref(fx), fx.gate_width, fx.gate_height)))
        table = torch.empty(need // 4 + 1, device="cuda")
        calls = {
            "film_defects": lambda: lib.fjb_film_defects(C.byref(fx), W, H, *[C.c_void_p(p.data_ptr()) for p in fdens],
                                                         C.c_void_p(dust.data_ptr()), C.c_void_p(table.data_ptr()),
                                                         need, None, C.byref(err.buf)),
            "gate_mask": lambda: lib.fjb_gate_mask(C.byref(fx), C.c_void_p(mask.data_ptr()), fx.gate_width,
                                                   fx.gate_height, C.c_void_p(table.data_ptr()), need, None,
                                                   C.byref(err.buf)),
        }
        for k, call in calls.items():
            call()
            e0.record()
            for _ in range(5):
                assert call().category == abi.FJ_STATUS_SUCCESS
            e1.record()
            e1.synchronize()
            ours[k] = e0.elapsed_time(e1) / 5
        for which, k, w, h in ((0, "film_defects", W, H), (1, "gate_mask", fx.gate_width, fx.gate_height)):
            for _ in range(2):
                assert ref.ref_defects_timed(C.byref(fx), which, w, h, *[C.c_void_p(p.data_ptr()) for p in fdens],
                                             C.c_void_p((dust if which == 0 else mask).data_ptr())) == 0
            theirs[k] = ref.ref_last_ms()

    table = {k: {"ours_ms": round(ours[k], 4), "reference_ms": round(theirs[k], 4),
                 "speedup": round(theirs[k] / ours[k], 2)} for k in theirs}
    print(json.dumps(table, indent=1))
    path = os.environ.get("FJB_SPEED_REPORT")
    if path:
        with open(path, "w") as fh:
            json.dump(table, fh, indent=1)
    for k, v in table.items():
        assert v["ours_ms"] <= v["reference_ms"], (k, v)


def test_camera_diffusion_against_reference_cufft(torch_cuda, recipes, prepare):
    """The reference's cuFFT camera diffusion (src/Cuda/Diffusion/JuicerCudaDiffusion.cu,
    driven through its execution planner by oracle/ref_fft_shim.cu) against this
    library's FFT form on the 4K carrier at radius 19: outputs within 2e-5 of the
    frame's scale (both FP32 transforms of the same PSF), and device time no longer than
    the reference's (its stage launch alone, mean of 5 after the first; ours the owner's
    camera-diffusion stage time in fj_cuda_render frames)."""
    import ctypes as C

    torch = torch_cuda
    from film_juicer_b200 import abi, frame_records, load_library, runtime

    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                        "libjuicer_ref_fft.so")
    if not os.path.exists(path):
        pytest.skip("reference cuFFT diffusion harness not built")
    ref = C.CDLL(path)
    ref.ref_fft_diffusion.restype = C.c_int
    ref.ref_fft_diffusion.argtypes = [C.POINTER(C.c_double)] * 4 + [C.c_int, C.c_double] + [C.c_void_p] * 6 + \
        [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float)]
    lib = load_library()
    rec = frame_records.FrameRecord(recipes["print"], W, H)
    desc = rec.host.h.optics.camera
    assert desc.radius_px == 19
    comps = runtime.diffusion_components(desc)
    src = torch.from_numpy(np.ascontiguousarray(prepare.synthetic_frame(W, H, seed=20261205))).cuda()
    dr = runtime.DeviceRecipe(rec.host)
    bgr = [torch.empty((H, W), device="cuda") for _ in range(3)]
    dr.camera_exposure(src, bgr)
    rgb = [bgr[2], bgr[1], bgr[0]]
    ours = [torch.empty_like(p) for p in rgb]
    runtime.diffusion(comps, desc.radius_px, desc.scatter_fraction, rgb, ours)
    theirs = [torch.empty_like(p) for p in rgb]
    ms = C.c_float()
    arr = lambda v: (C.c_double * 9)(*list(v))  # noqa: E731
    rc = ref.ref_fft_diffusion(arr(comps.lambda_px), arr(comps.red_weights), arr(comps.green_weights),
                               arr(comps.blue_weights), desc.radius_px, desc.scatter_fraction,
                               *[C.c_void_p(p.data_ptr()) for p in rgb], *[C.c_void_p(p.data_ptr()) for p in theirs],
                               W, H, 5, C.byref(ms))
    assert rc == 0, rc
    torch.cuda.synchronize()
    for a, b in zip(ours, theirs):
        scale = float(b.abs().max())
        assert float((a - b).abs().max()) <= 2e-5 * scale, float((a - b).abs().max()) / scale
    err = abi.ErrorText()
    d = torch.empty_like(src)
    with runtime.Owner() as owner:
        owner.render(rec, src, d)
        lib.fjb_owner_stage_timing(owner.handle, 1, C.byref(err.buf))
        for _ in range(5):
            owner.render(rec, src, d)
        t = abi.FjbStageTimes()
        lib.fjb_owner_stage_times(owner.handle, C.byref(t), C.byref(err.buf))
        i = abi.FJB_STAGE_NAMES.index("camera_diffusion")
        ours_ms = t.total_ms[i] / t.frames[i]
    row = {"ours_ms": round(ours_ms, 4), "reference_ms": round(ms.value, 4), "speedup": round(ms.value / ours_ms, 2)}
    print(json.dumps({"camera_diffusion": row}))
    path = os.environ.get("FJB_SPEED_REPORT")
    if path:
        table = json.load(open(path)) if os.path.exists(path) else {}
        table["camera_diffusion"] = row
        with open(path, "w") as fh:
            json.dump(table, fh, indent=1)
    dr.close()
    assert ours_ms <= ms.value, row
