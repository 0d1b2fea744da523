"""fjb_diffusion_no_alloc against fjb_diffusion through the C-ABI (GPU).

Two calls in a row on the same frames -- a large radius, then a smaller one, so the
second call reads rows that the first left behind in the shared static PSF array --
must each match the allocating entry point. The tables differ only in how the FP64
PSF sum is ordered (device vs host) and in the FP64 exp of each side, a float32
rounding step of the normalised taps: |d| <= 1e-6 max(1, max |input|).

Collected last so that it also runs after every other test in the session."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _call(lib, name, comps, radius, fraction, src, dst, stream=0):
    from film_juicer_b200 import abi

    err = abi.ErrorText()
    h, w = src[0].shape
    st = getattr(lib, name)(C.byref(comps), radius, fraction, *[C.c_void_p(t.data_ptr()) for t in src],
                            *[C.c_void_p(t.data_ptr()) for t in dst], src[0].stride(0), w, h, C.c_void_p(stream),
                            C.byref(err.buf))
    return st, err.text


def test_no_alloc_matches_allocating_entry(torch_cuda):
    torch = torch_cuda
    from film_juicer_b200 import abi, descriptors, load_library, runtime

    lib = load_library()
    comps = runtime.diffusion_components(descriptors.diffusion_record(3.2, 3840, family=3, warmth=-0.6))
    rng = np.random.default_rng(17)
    h, w = 150, 211
    planes = [torch.from_numpy(rng.uniform(0.0, 2.0, size=(h, w)).astype(np.float32)).cuda() for _ in range(3)]
    planes[1][h // 3, w // 4] += 30.0
    scale = max(1.0, float(max(p.abs().max() for p in planes)))
    for radius, fraction in ((64, 0.35), (9, 0.2), (80, 0.5)):
        want = [torch.empty_like(p) for p in planes]
        got = [torch.full_like(p, float("nan")) for p in planes]
        st, text = _call(lib, "fjb_diffusion", comps, radius, fraction, planes, want)
        assert st.category == abi.FJ_STATUS_SUCCESS, text
        st, text = _call(lib, "fjb_diffusion_no_alloc", comps, radius, fraction, planes, got)
        assert st.category == abi.FJ_STATUS_SUCCESS, text
        torch.cuda.synchronize()
        for g, r in zip(got, want):
            err = (g - r).abs().max().item()
            assert err <= TOL * scale, (radius, err)


def test_no_alloc_rejects_radius_beyond_static_scratch(torch_cuda):
    torch = torch_cuda
    from film_juicer_b200 import abi, descriptors, load_library, runtime

    lib = load_library()
    comps = runtime.diffusion_components(descriptors.diffusion_record(3.2, 3840))
    a = [torch.zeros((8, 8), device="cuda") for _ in range(3)]
    b = [torch.zeros((8, 8), device="cuda") for _ in range(3)]
    st, text = _call(lib, "fjb_diffusion_no_alloc", comps, 81, 0.5, a, b)
    assert st.category == abi.FJ_STATUS_UNSUPPORTED_INPUT
    assert "static PSF scratch" in text


def test_no_alloc_leaves_free_device_memory_unchanged_and_runs_on_a_stream(torch_cuda):
    """The property the entry exists for: after a first call (which sets up the device
    address of the static array), further calls change the device's free memory by
    nothing. One call is enqueued on a non-default stream and only that stream is
    synchronised before the comparison."""
    torch = torch_cuda
    from film_juicer_b200 import abi, descriptors, load_library, runtime

    lib = load_library()
    comps = runtime.diffusion_components(descriptors.diffusion_record(4.0, 1920))
    rng = np.random.default_rng(5)
    h, w = 96, 128
    planes = [torch.from_numpy(rng.uniform(0.0, 1.5, size=(h, w)).astype(np.float32)).cuda() for _ in range(3)]
    want = [torch.empty_like(p) for p in planes]
    got = [torch.full_like(p, float("nan")) for p in planes]
    st, text = _call(lib, "fjb_diffusion", comps, 12, 0.3, planes, want)
    assert st.category == abi.FJ_STATUS_SUCCESS, text
    st, text = _call(lib, "fjb_diffusion_no_alloc", comps, 12, 0.3, planes, got)
    assert st.category == abi.FJ_STATUS_SUCCESS, text
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(4):
        st, text = _call(lib, "fjb_diffusion_no_alloc", comps, 12, 0.3, planes, got)
        assert st.category == abi.FJ_STATUS_SUCCESS, text
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    for g in got:
        g.fill_(float("nan"))
    torch.cuda.current_stream().synchronize()
    st, text = _call(lib, "fjb_diffusion_no_alloc", comps, 12, 0.3, planes, got, stream=side.cuda_stream)
    assert st.category == abi.FJ_STATUS_SUCCESS, text
    side.synchronize()
    scale = max(1.0, float(max(p.abs().max() for p in planes)))
    for g, r in zip(got, want):
        assert (g - r).abs().max().item() <= TOL * scale


def test_no_alloc_rejects_negative_weights_that_the_allocating_entry_accepts(torch_cuda):
    """The documented difference between the two entries: fjb_diffusion normalises any
    PSF whose stored sum is finite and positive, the no-allocation entry needs
    non-negative weights (its device build cannot check the sum before it is used)."""
    torch = torch_cuda
    from film_juicer_b200 import abi, descriptors, load_library, runtime

    lib = load_library()
    comps = runtime.diffusion_components(descriptors.diffusion_record(4.0, 1920))
    comps.green_weights[8] = -0.01 * abs(comps.green_weights[0]) - 1e-6
    a = [torch.rand((16, 24), device="cuda") for _ in range(3)]
    b = [torch.zeros((16, 24), device="cuda") for _ in range(3)]
    st, text = _call(lib, "fjb_diffusion", comps, 6, 0.5, a, b)
    assert st.category == abi.FJ_STATUS_SUCCESS, text
    st, text = _call(lib, "fjb_diffusion_no_alloc", comps, 6, 0.5, a, b)
    assert st.category == abi.FJ_STATUS_PREPARATION_FAILURE
    assert "non-negative" in text
