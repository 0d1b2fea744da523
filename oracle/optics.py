"""Oracle wrappers for the optics stages (test infrastructure only)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import oracle as _o


def scatter_halation(descriptor, planes_rgb):
    """CPU restatement of the reference's scatter/halation schedule; returns new planes."""
    lib = _o.load()
    abi = _o._abi()
    fn = lib.oracle_scatter_halation
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.FjScatterHalation)] + [C.c_void_p] * 3 + [C.c_long, C.c_int, C.c_int]
    out = [np.ascontiguousarray(p, dtype=np.float32).copy() for p in planes_rgb]
    h, w = out[0].shape
    rc = fn(C.byref(descriptor), *[C.c_void_p(p.ctypes.data) for p in out], w, w, h)
    if rc != 0:
        raise RuntimeError("oracle_scatter_halation failed")
    return out


def reference_scatter_halation(torch, descriptor, planes_rgb):
    """The reference's own CUDA scatter/halation on copies of the planes (None if the
    harness is not built)."""
    lib = _o.load_reference()
    if lib is None:
        return None
    abi = _o._abi()
    fn = lib.ref_scatter_halation
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.FjScatterHalation)] + [C.c_void_p] * 3 + [C.c_long, C.c_int, C.c_int]
    dev = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.float32)).cuda() for p in planes_rgb]
    h, w = dev[0].shape
    rc = fn(C.byref(descriptor), *[C.c_void_p(t.data_ptr()) for t in dev], w, w, h)
    if rc != 0:
        raise RuntimeError(f"reference scatter/halation returned cudaError {rc}")
    return [t.cpu().numpy() for t in dev]


def diffusion(components, radius, fraction, planes_rgb):
    """CPU oracle of the diffusion stage; returns new planes (R, G, B)."""
    lib = _o.load()
    fn = lib.oracle_diffusion
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_double,
                   C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int, C.c_int]
    lam = (C.c_double * 9)(*components.lambda_px)
    w = (C.c_double * 27)(*components.red_weights, *components.green_weights, *components.blue_weights)
    src = [np.ascontiguousarray(p, dtype=np.float32) for p in planes_rgb]
    out = [np.zeros_like(p) for p in src]
    h, wd = src[0].shape
    sp = (C.c_void_p * 3)(*[p.ctypes.data for p in src])
    dp = (C.c_void_p * 3)(*[p.ctypes.data for p in out])
    if fn(lam, w, radius, fraction, sp, dp, wd, h) != 0:
        raise RuntimeError("oracle_diffusion failed")
    return out


def diffusion_psf(components, radius):
    """The three normalised (2r+1)^2 PSFs (R, G, B) as the oracle stores them (float32)."""
    lib = _o.load()
    fn = lib.oracle_diffusion_psf
    fn.restype = None
    fn.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_int, C.c_void_p]
    lam = (C.c_double * 9)(*components.lambda_px)
    w = (C.c_double * 27)(*components.red_weights, *components.green_weights, *components.blue_weights)
    out = []
    for c in range(3):
        psf = np.zeros((2 * radius + 1, 2 * radius + 1), np.float32)
        fn(lam, w, radius, c, C.c_void_p(psf.ctypes.data))
        out.append(psf)
    return out


def diffusion_fft(components, radius, fraction, planes_rgb, workers: int = 1):
    """The diffusion stage in the reference's own form (src/Cuda/Diffusion/
    JuicerCudaDiffusion.cu:510-625: reflect-padded frame, real FFT, product with the
    PSF spectrum, inverse FFT, crop, mix), in FP64 with scipy's FFT over `workers`
    threads. Same PSF and padding as diffusion(); the results agree with its direct
    FP64 sum to FP64 transform rounding (checked in tests/test_diffusion_golden.py).
    The CPU baseline times this form, the parity tests use the direct sum."""
    import scipy.fft as sfft

    psfs = diffusion_psf(components, radius)
    out = []
    f = np.float32(fraction)
    for p, psf in zip(planes_rgb, psfs):
        p = np.ascontiguousarray(p, dtype=np.float32)
        h, w = p.shape
        padded = np.pad(p.astype(np.float64), radius, mode="reflect") if radius > 0 else p.astype(np.float64)
        ny, nx = sfft.next_fast_len(padded.shape[0], real=True), sfft.next_fast_len(padded.shape[1], real=True)
        spec = sfft.rfft2(padded, s=(ny, nx), workers=workers)
        kern = np.zeros((ny, nx))
        kern[: 2 * radius + 1, : 2 * radius + 1] = psf.astype(np.float64)
        spec *= sfft.rfft2(kern, workers=workers)
        conv = sfft.irfft2(spec, s=(ny, nx), workers=workers)
        acc = conv[2 * radius: 2 * radius + h, 2 * radius: 2 * radius + w].astype(np.float32)
        out.append(((np.float32(1.0) - f) * p + f * acc).astype(np.float32))
    return out


def diffusion_components(family, group_weights, group_lambda_um, warmth, spatial_scale, pixel_size_um):
    """Pure-Python restatement of the reference's diffusion component expansion
    (rust/film-juicer-core/src/optics/diffusion_frame.rs:285-421: expand_group,
    halo_weights, Components::new). Returns (lambda_px[9], weights[3][9]) as lists."""
    import math

    def expand(center, spread, count, alpha):
        lo, hi = math.log(center / spread), math.log(center * spread)
        lam, w = [], []
        for i in range(count):
            if i + 1 == count:
                ll = hi
            elif i != 0:
                ll = lo + (hi - lo) * (i / (count - 1))
            else:
                ll = lo
            lam.append(math.exp(ll))
            w.append(lam[-1] ** (2.0 - alpha) if alpha is not None else 1.0)
        t = 0.0
        for v in w:
            t += v
        return lam, [v / t for v in w]

    core = expand(group_lambda_um[0], 1.5, 2, None)
    halo = expand(group_lambda_um[1], 2.0, 3, None)
    bloom = expand(group_lambda_um[2], 2.5, 4, (3.2, 3.5, 2.9, 2.5)[family])
    grad = [-1.0 + 2.0 * i / 2 for i in range(3)]
    target = 0.0
    wg = 0.0
    for i in range(3):
        target += halo[1][i]
        wg += halo[1][i] * grad[i]
    wg /= target
    grad = [g - wg for g in grad]
    halo_rgb = []
    for axis in (1.30, 0.15, -1.45):
        row = [max(halo[1][i] * (1.0 + warmth * axis * grad[i]), 0.0) for i in range(3)]
        t = 0.0
        for v in row:
            t += v
        halo_rgb.append([v * (target / t) for v in row] if t > 0.0 else list(halo[1]))
    scale = max(spatial_scale, 1e-6)
    lam_px, weights = [], [[], [], []]
    for gi, (lam, w) in enumerate((core, halo, bloom)):
        for i, l in enumerate(lam):
            lam_px.append(max(l * scale / pixel_size_um, 1e-6))
            for c in range(3):
                weights[c].append(group_weights[1] * halo_rgb[c][i] if gi == 1 else group_weights[gi] * w[i])
    return lam_px, weights


def highlight_boost(descriptor, carrier_bgr):
    """CPU oracle of the highlight reconstruction (src/Cuda/Film/JuicerCudaHighlightBoost.cu)
    on carrier planes B, G, R; returns (new planes B, G, R, disposition)."""
    import numpy as np

    lib = _o.load()
    fn = lib.oracle_highlight_boost
    fn.restype = C.c_int
    fn.argtypes = [C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long,
                   C.c_int, C.c_int]
    planes = [np.array(p, dtype=np.float32, copy=True, order="C") for p in carrier_bgr]
    h, w = planes[0].shape
    disp = fn(descriptor.recipe_hash, descriptor.protection, descriptor.sharpness, descriptor.peak_gain,
              *[C.c_void_p(p.ctypes.data) for p in planes], w, w, h)
    return planes, disp


def reference_highlight_boost(torch, descriptor, carrier_bgr):
    """The reference's own CUDA highlight reconstruction on device planes (in place);
    returns the disposition."""
    ref = _o.load_reference()
    fn = ref.ref_highlight_boost
    fn.restype = C.c_int
    abi = _o._abi()
    fn.argtypes = [C.POINTER(abi.FjHighlightBoost), C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_int,
                   C.POINTER(C.c_int)]
    b, g, r = carrier_bgr
    h, w = b.shape
    disp = C.c_int()
    rc = fn(C.byref(descriptor), C.c_void_p(b.data_ptr()), C.c_void_p(g.data_ptr()), C.c_void_p(r.data_ptr()),
            b.stride(0), w, h, C.byref(disp))
    if rc != 0:
        raise RuntimeError(f"ref_highlight_boost failed with code {rc}")
    return disp.value


def enlarger_linear(record, density_cmy, dust=None):
    """Print-linear exposure planes (C-, M-, Y-forming) of capture density planes
    (oracle_enlarger_linear)."""
    lib = _o.load()
    abi = _o._abi()
    fn = lib.oracle_enlarger_linear
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.FjPreparedHostData)] + [C.c_void_p] * 4 + [C.c_int, C.c_int] + [C.c_void_p] * 3
    dens = [np.ascontiguousarray(p, dtype=np.float32) for p in density_cmy]
    h, w = dens[0].shape
    out = [np.zeros((h, w), np.float32) for _ in range(3)]
    d = np.ascontiguousarray(dust, dtype=np.float32) if dust is not None else None
    rc = fn(record.pointer(), *[C.c_void_p(p.ctypes.data) for p in dens],
            C.c_void_p(d.ctypes.data) if d is not None else None, w, h, *[C.c_void_p(p.ctypes.data) for p in out])
    if rc != 0:
        raise RuntimeError("oracle_enlarger_linear failed")
    return out


def enlarger_develop(record, linear_cmy):
    """Print density planes C, M, Y from the diffused print-linear exposure."""
    lib = _o.load()
    abi = _o._abi()
    fn = lib.oracle_enlarger_develop
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.FjPreparedHostData)] + [C.c_void_p] * 3 + [C.c_int, C.c_int] + [C.c_void_p] * 3
    lin = [np.ascontiguousarray(p, dtype=np.float32) for p in linear_cmy]
    h, w = lin[0].shape
    out = [np.zeros((h, w), np.float32) for _ in range(3)]
    if fn(record.pointer(), *[C.c_void_p(p.ctypes.data) for p in lin], w, h, *[C.c_void_p(p.ctypes.data) for p in out]):
        raise RuntimeError("oracle_enlarger_develop failed")
    return out


class print_done:
    """Within the block the oracle's render entry points scan the density planes as
    print density (after the enlarger diffusion), without the print step."""

    def __enter__(self):
        _o.load().oracle_set_print_done(1)
        return self

    def __exit__(self, *exc):
        _o.load().oracle_set_print_done(0)


def reference_enlarger(torch, record, stage, planes, dust=None):
    """The reference's own enlarger kernels on device copies of `planes`: stage 0 the
    print-linear exposure of density planes C, M, Y, stage 1 the print density of
    diffused linear planes. None when the harness is not built."""
    lib = _o.load_reference()
    if lib is None or not hasattr(lib, "ref_enlarger"):
        return None
    abi = _o._abi()
    fn = lib.ref_enlarger
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.FjPreparedHostData), C.POINTER(C.c_void_p), C.c_int] + [C.c_void_p] * 4 + \
        [C.c_int, C.c_int] + [C.c_void_p] * 3
    lut = _o.scanner_lut_for(record)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    dev = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.float32)).cuda() for p in planes]
    h, w = dev[0].shape
    out = [torch.zeros((h, w), device="cuda") for _ in range(3)]
    dd = torch.from_numpy(np.ascontiguousarray(dust, dtype=np.float32)).cuda() if dust is not None else None
    rc = fn(record.pointer(), ptrs, stage, *[C.c_void_p(t.data_ptr()) for t in dev],
            C.c_void_p(dd.data_ptr()) if dd is not None else None, w, h, *[C.c_void_p(t.data_ptr()) for t in out])
    if rc != 0:
        raise RuntimeError(f"reference enlarger stage returned {rc}")
    return [t.cpu().numpy() for t in out]
