"""Parity against the reference's OWN CUDA kernels, compiled for sm_100a from the
reference sources (oracle/_ref/libjuicer_ref.so, built by oracle/build_ref.py) and
driven with the same FjPreparedHostData: juicer_cuda_negative_pipeline /
juicer_cuda_print_pipeline (src/Cuda/Scan/JuicerCudaScanPipeline.cu:2244, :3759) and
juicer_cuda_print_focused_capture_density (:2894).

This pins both the CPU oracle and the B200 kernels to the plug-in's current CUDA
path on identical inputs. Tolerances are the reference's processor-pixel bound
(2e-4 + 3e-4 |ref|) on encoded output and 1e-4 + 1e-4 |ref| on density.
"""
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


def run_reference(torch, ref_lib, oracle, rec, src):
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


@pytest.mark.parametrize("route", ["direct", "print"])
@pytest.mark.parametrize("comps", [3, 4])
def test_b200_and_oracle_match_reference_cuda(torch_cuda, ref_lib, oracle, recipes, prepare, route, comps):
    torch = torch_cuda
    from film_juicer_b200 import runtime

    rec = prepare.HostRecord(recipes[route])
    src = prepare.synthetic_frame(200, 120, seed=20261203)
    if comps == 4:
        src = np.ascontiguousarray(np.concatenate([src, np.full((120, 200, 1), 0.25, np.float32)], axis=2))
    ref, rflags = run_reference(torch, ref_lib, oracle, rec, src)
    dr = runtime.DeviceRecipe(rec)
    s = torch.from_numpy(src).cuda()
    d = torch.empty_like(s)
    dr.clear_flags()
    dr.render(s, d)
    mine = d.cpu().numpy()
    assert dr.read_flags() == rflags
    dr.close()
    orc, oflags = oracle.render(rec, src)
    assert oflags == rflags
    tol = 2e-4 + 3e-4 * np.abs(ref)
    assert np.all(np.abs(mine - ref) <= tol), float(np.max(np.abs(mine - ref)))
    assert np.all(np.abs(orc - ref) <= tol), float(np.max(np.abs(orc - ref)))


@pytest.mark.parametrize("route", ["direct", "print"])
def test_capture_density_matches_reference_cuda(torch_cuda, ref_lib, oracle, recipes, prepare, route):
    torch = torch_cuda
    from film_juicer_b200 import runtime

    rec = prepare.HostRecord(recipes[route])
    src = prepare.synthetic_frame(150, 100, seed=7)
    lut = oracle.scanner_lut_for(rec)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    s = torch.from_numpy(src).cuda()
    ref_planes = [torch.zeros((100, 150), device="cuda") for _ in range(3)]
    rc = ref_lib.ref_capture_density(rec.pointer(), ptrs, C.c_void_p(s.data_ptr()), 150 * 12, 150, 100, 3,
                                     *[C.c_void_p(p.data_ptr()) for p in ref_planes])
    assert rc == 0
    dr = runtime.DeviceRecipe(rec)
    mine = [torch.empty((100, 150), device="cuda") for _ in range(3)]
    dr.capture_density(s, mine)
    torch.cuda.synchronize()
    for a, b in zip(mine, ref_planes):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.all(np.abs(a - b) <= 1e-4 + 1e-4 * np.abs(b)), float(np.max(np.abs(a - b)))
    dr.close()
