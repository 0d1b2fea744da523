"""Scanner post effects (the first of the path's next rows): glare, lens blur and unsharp
on the linear output-RGB planes between the scan and the output encoding.

Against the reference's own CUDA launchers (juicer_cuda_print_focused_scan_linear_density_rgb
and juicer_cuda_print_focused_scanner_post_output, compiled for sm_100a) on the same
density planes: within 1e-6 on the direct route (glare noise, FP64 blur sums, scan and
encode); the print route adds the print development, where the builds differ by float
rounding (2e-5).
Against the oracle's restatement: the reference's CUDA pixel bound 2e-4 + 3e-4 |oracle|
(its glare uses the host libm's log/cos/exp). Through fj_cuda_render: the frame schedule
with post effects against the oracle's stage chain, as for the other stage combinations."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_lib(oracle):
    lib = oracle.load_reference()
    if lib is None:
        pytest.skip("reference CUDA harness not built (needs the reference sources at build time)")
    return lib

POSTS = {
    "glare": dict(glare_percent=0.6, glare_roughness=0.5, glare_blur_sigma_px=2.0),
    "glare_unblurred": dict(glare_percent=0.3, glare_roughness=0.8),
    "lens": dict(lens_blur_sigma_px=1.5),
    "unsharp": dict(unsharp_sigma_px=0.7, unsharp_amount=0.7),
    "all": dict(glare_percent=0.4, glare_roughness=0.4, glare_blur_sigma_px=3.0, lens_blur_sigma_px=0.9,
                unsharp_sigma_px=1.2, unsharp_amount=0.5),
}


def density_planes(torch, dr, src):
    planes = [torch.empty(src.shape[:2], device="cuda") for _ in range(3)]
    dr.capture_density(torch.from_numpy(src).cuda(), planes)
    torch.cuda.synchronize()
    return planes


@pytest.mark.parametrize("name", list(POSTS))
@pytest.mark.parametrize("route", ["print", "direct"])
def test_post_matches_reference_cuda(torch_cuda, ref_lib, oracle, recipes, prepare, route, name):
    torch = torch_cuda
    from film_juicer_b200 import descriptors, runtime

    if not hasattr(ref_lib, "ref_scanner_post"):
        pytest.skip("reference harness built without the post-effects entry")
    w, h = 96, 70
    rec = prepare.HostRecord(recipes[route])
    post = descriptors.scanner_post_record(**POSTS[name])
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=13))
    s = torch.from_numpy(src).cuda()
    dr = runtime.DeviceRecipe(rec)
    dens = density_planes(torch, dr, src)
    seed = oracle.glare_seed(rec.h.recipe_hash, 41, 3, -2)
    mine = torch.full_like(s, -1.0)
    runtime.render_from_density_post(dr, post, seed, (3, -2), dens, mine, src=s)
    lut = oracle.scanner_lut_for(rec)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    ref = torch.full_like(s, -1.0)
    rc = ref_lib.ref_scanner_post(rec.pointer(), ptrs, C.byref(post), seed, 3, -2,
                                  *[C.c_void_p(p.data_ptr()) for p in dens], C.c_void_p(s.data_ptr()), w * 12,
                                  C.c_void_p(ref.data_ptr()), w * 12, w, h, 3)
    assert rc == 0
    torch.cuda.synchronize()
    a, b = mine.cpu().numpy(), ref.cpu().numpy()
    assert np.all(np.isfinite(a))
    err = np.abs(a - b)
    # the direct route scans the capture density as is; the print route develops the
    # print first, where the two builds differ by float rounding of the spectral sums
    bound = 1e-6 if route == "direct" else 2e-5
    assert float(err.max()) <= bound, (name, float(err.max()), float((err > 0).mean()))
    dr.close()


# Frame shapes for the blur kernels: single pixel, frames narrower and shorter than one
# run of outputs, radii wider than the frame (reflection repeated), and a row too long
# for a shared-memory tile (the per-output fallback).
SHAPES = [
    (1, 1, dict(lens_blur_sigma_px=1.5, unsharp_sigma_px=0.7, unsharp_amount=0.7)),
    (5, 3, dict(glare_percent=0.4, glare_roughness=0.4, glare_blur_sigma_px=3.0, lens_blur_sigma_px=2.0)),
    (13, 40, dict(lens_blur_sigma_px=12.0, lens_blur_radius=50, unsharp_sigma_px=1.2, unsharp_amount=0.5)),
    (257, 11, dict(glare_percent=0.5, glare_roughness=0.3, glare_blur_sigma_px=4.0, lens_blur_sigma_px=0.8)),
    (24600, 2, dict(lens_blur_sigma_px=0.8, unsharp_sigma_px=0.7, unsharp_amount=0.7)),
]


@pytest.mark.parametrize("w,h,kw", SHAPES, ids=[f"{w}x{h}" for w, h, _ in SHAPES])
def test_post_shapes_match_reference_cuda(torch_cuda, ref_lib, oracle, recipes, prepare, w, h, kw):
    torch = torch_cuda
    from film_juicer_b200 import descriptors, runtime

    if not hasattr(ref_lib, "ref_scanner_post"):
        pytest.skip("reference harness built without the post-effects entry")
    rec = prepare.HostRecord(recipes["direct"])
    post = descriptors.scanner_post_record(**kw)
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=29))
    s = torch.from_numpy(src).cuda()
    dr = runtime.DeviceRecipe(rec)
    dens = density_planes(torch, dr, src)
    seed = oracle.glare_seed(rec.h.recipe_hash, 7, 1, 2)
    mine = torch.full_like(s, -1.0)
    runtime.render_from_density_post(dr, post, seed, (1, 2), dens, mine, src=s)
    lut = oracle.scanner_lut_for(rec)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    ref = torch.full_like(s, -1.0)
    rc = ref_lib.ref_scanner_post(rec.pointer(), ptrs, C.byref(post), seed, 1, 2,
                                  *[C.c_void_p(p.data_ptr()) for p in dens], C.c_void_p(s.data_ptr()), w * 12,
                                  C.c_void_p(ref.data_ptr()), w * 12, w, h, 3)
    assert rc == 0
    torch.cuda.synchronize()
    a, b = mine.cpu().numpy(), ref.cpu().numpy()
    assert np.all(np.isfinite(a))
    err = np.abs(a - b)
    assert float(err.max()) <= 1e-6, (w, h, float(err.max()), float((err > 0).mean()))
    dr.close()


@pytest.mark.parametrize("name", list(POSTS))
def test_post_matches_oracle(torch_cuda, oracle, recipes, prepare, name):
    torch = torch_cuda
    from film_juicer_b200 import descriptors, runtime

    w, h = 120, 64
    rec = prepare.HostRecord(recipes["print"])
    post = descriptors.scanner_post_record(**POSTS[name])
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=17))
    s = torch.from_numpy(src).cuda()
    dr = runtime.DeviceRecipe(rec)
    dens = density_planes(torch, dr, src)
    seed = oracle.glare_seed(rec.h.recipe_hash, 5, 0, 0)
    mine = torch.empty_like(s)
    runtime.render_from_density_post(dr, post, seed, (0, 0), dens, mine, src=s)
    want, _ = oracle.render_post(rec, post, seed, 0, 0, [d.cpu().numpy() for d in dens], src=src)
    got = mine.cpu().numpy()
    err = np.abs(got - want)
    assert np.all(err <= 2e-4 + 3e-4 * np.abs(want)), (name, float(err.max()))
    dr.close()


def test_post_changes_the_frame_and_hash_zero_is_inactive(torch_cuda, oracle, recipes, prepare):
    torch = torch_cuda
    from film_juicer_b200 import descriptors, runtime

    w, h = 64, 48
    rec = prepare.HostRecord(recipes["print"])
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=3))
    s = torch.from_numpy(src).cuda()
    dr = runtime.DeviceRecipe(rec)
    dens = density_planes(torch, dr, src)
    plain = torch.empty_like(s)
    dr.render_from_density(dens, s, plain)
    off = torch.empty_like(s)
    runtime.render_from_density_post(dr, descriptors.scanner_post_record(unsharp_sigma_px=1.0, unsharp_amount=0.7,
                                                                         hash=0), 1, (0, 0), dens, off, src=s)
    on = torch.empty_like(s)
    runtime.render_from_density_post(dr, descriptors.scanner_post_record(unsharp_sigma_px=1.0, unsharp_amount=0.7),
                                     1, (0, 0), dens, on, src=s)
    torch.cuda.synchronize()
    assert torch.equal(off, plain)
    assert float((on - plain).abs().max()) > 1e-4
    dr.close()


def test_post_rejects_malformed_records(torch_cuda, recipes, prepare):
    torch = torch_cuda
    from film_juicer_b200 import descriptors, runtime

    rec = prepare.HostRecord(recipes["print"])
    dr = runtime.DeviceRecipe(rec)
    dens = [torch.zeros((8, 8), device="cuda") for _ in range(3)]
    out = torch.empty((8, 8, 3), device="cuda")
    bad = descriptors.scanner_post_record(lens_blur_sigma_px=1.0, lens_blur_radius=4000)
    with pytest.raises(runtime.FjError, match="radius"):
        runtime.render_from_density_post(dr, bad, 1, (0, 0), dens, out)
    bad = descriptors.scanner_post_record(unsharp_sigma_px=1.0, unsharp_amount=0.5)
    bad.flags = 6
    with pytest.raises(runtime.FjError, match="flags"):
        runtime.render_from_density_post(dr, bad, 1, (0, 0), dens, out)
    dr.close()


@pytest.mark.parametrize("name", ["unsharp", "all"])
def test_frame_schedule_with_post_matches_oracle_chain(torch_cuda, recipes, prepare, name):
    from film_juicer_b200 import descriptors, frame_records, runtime
    from oracle import frame as oframe

    torch = torch_cuda
    w, h = 120, 72
    post = descriptors.scanner_post_record(**POSTS[name])
    rec = frame_records.FrameRecord(recipes["print"], w, h, post=post)
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=20261205))
    s = torch.from_numpy(src).cuda()
    d = torch.full_like(s, -1.0)
    with runtime.Owner() as owner:
        owner.render(rec, s, d, frame_token=9)
    got = d.cpu().numpy()
    want, _ = oframe.render_frame(rec, recipes["print"], src, frame_token=9)
    err = np.abs(got - want)
    bad = err > 2e-4 + 3e-4 * np.abs(want)
    assert float(bad.mean()) <= 0.01, (name, float(bad.mean()), float(err.max()))
    assert float(err.mean()) <= 1e-4, (name, float(err.mean()))
