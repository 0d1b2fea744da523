"""ctypes loader of oracle/liboracle.so -- the CPU restatement used as the checker.

Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's CPU legs load
it; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build() -> str:
    res = subprocess.run(["make", "-C", HERE, "-s"], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    sys.path.insert(0, os.path.dirname(HERE))
    abi = _abi()
    lib = C.CDLL(LIB)
    lib.oracle_scanner_lut.restype = C.c_int
    lib.oracle_scanner_lut.argtypes = [C.POINTER(abi.FjbScannerLutInput)] + [C.c_void_p] * 6
    lib.oracle_render.restype = C.c_int
    lib.oracle_render.argtypes = [C.POINTER(abi.FjPreparedHostData), C.c_int, C.c_void_p, C.c_long, C.c_int,
                                  C.c_int, C.c_int, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_float, C.c_int, C.POINTER(C.c_uint32)]
    lib.oracle_render_post.restype = C.c_int
    lib.oracle_render_post.argtypes = [C.POINTER(abi.FjPreparedHostData), C.POINTER(abi.FjScannerPostEffects),
                                       C.c_uint64, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_long, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_long, C.c_int,
                                       C.POINTER(C.c_uint32)]
    lib.oracle_render_effects.restype = C.c_int
    lib.oracle_render_effects.argtypes = [C.POINTER(abi.FjPreparedHostData), C.POINTER(abi.FjScannerPostEffects),
                                          C.c_uint64, C.c_int, C.c_int, C.POINTER(abi.FjFilmEffects), C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long,
                                          C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_long, C.c_int,
                                          C.POINTER(C.c_uint32)]
    lib.oracle_film_defects.restype = C.c_int
    lib.oracle_film_defects.argtypes = [C.POINTER(abi.FjFilmEffects), C.c_int, C.c_int] + [C.c_void_p] * 4
    lib.oracle_gate_mask.restype = C.c_int
    lib.oracle_gate_mask.argtypes = [C.POINTER(abi.FjFilmEffects), C.c_void_p, C.c_int, C.c_int]
    _lib = lib
    return lib


def film_defects(effects, planes):
    """Film dust / scratches on density planes (C, M, Y): returns (scratched planes, dust
    transmittance plane or None)."""
    import numpy as np

    lib = load()
    p = [np.ascontiguousarray(q, dtype=np.float32).copy() for q in planes]
    h, w = p[0].shape
    dust = np.ones((h, w), np.float32) if effects.film_dust.slot_probability > 0.0 else None
    rc = lib.oracle_film_defects(C.byref(effects), w, h, *[C.c_void_p(q.ctypes.data) for q in p],
                                 C.c_void_p(dust.ctypes.data if dust is not None else 0))
    if rc != 0:
        raise RuntimeError(f"oracle_film_defects failed with code {rc}")
    return p, dust


def gate_mask(effects):
    """Gate dust x gate scratch transmittance on the gate grid (gate_height, gate_width)."""
    import numpy as np

    lib = load()
    mask = np.ones((effects.gate_height, effects.gate_width), np.float32)
    rc = lib.oracle_gate_mask(C.byref(effects), C.c_void_p(mask.ctypes.data), effects.gate_width, effects.gate_height)
    if rc != 0:
        raise RuntimeError(f"oracle_gate_mask failed with code {rc}")
    return mask


def render_effects(record, post, seed: int, origin_x: int, origin_y: int, effects, dust, mask, planes, src=None,
                   threads: int = 1):
    """render_post with the film defects' output effects (dust plane, weave, gate mask)."""
    import numpy as np

    lib = load()
    p = [np.ascontiguousarray(q, dtype=np.float32) for q in planes]
    h, w = p[0].shape
    comps = 3
    if src is not None:
        src = np.ascontiguousarray(src, dtype=np.float32)
        comps = src.shape[2]
    dst = np.zeros((h, w, comps), np.float32)
    flags = C.c_uint32()
    dust = np.ascontiguousarray(dust, dtype=np.float32) if dust is not None else None
    mask = np.ascontiguousarray(mask, dtype=np.float32) if mask is not None else None
    rc = lib.oracle_render_effects(record.pointer(), C.byref(post), seed, origin_x, origin_y,
                                   C.byref(effects) if effects is not None else None,
                                   C.c_void_p(dust.ctypes.data if dust is not None else 0),
                                   C.c_void_p(mask.ctypes.data if mask is not None else 0),
                                   *[C.c_void_p(q.ctypes.data) for q in p],
                                   C.c_void_p(src.ctypes.data if src is not None else 0), w * comps, w, h, comps,
                                   C.c_void_p(dst.ctypes.data), w * comps, threads, C.byref(flags))
    if rc != 0:
        raise RuntimeError(f"oracle_render_effects failed with code {rc}")
    return dst, int(flags.value)


def _abi():
    import importlib
    return importlib.import_module("film_juicer_b200.abi")


def render(record, src, *, stage: int = 0, planes=None, auto_scale: float = 1.0, threads: int = 1):
    """Runs the oracle on a host image.

    stage 0: source -> encoded output (returns (H, W, comps));
    stage 1: source -> capture density planes (returns 3 planes C, M, Y);
    stage 2: density planes -> encoded output; stage 3: source -> camera exposure
    planes B, G, R; stage 4: carrier planes B, G, R -> encoded output; stage 5:
    carrier planes B, G, R -> capture density planes C, M, Y; stage 6: source -> camera
    exposure planes B, G, R with the route correction; stage 7: source -> the scanner's
    linear output RGB planes (before output gamut compression and encoding, NaN where
    the scan fails).
    Returns (result, flags).
    """
    import numpy as np

    lib = load()
    if src is not None:
        src = np.ascontiguousarray(src, dtype=np.float32)
        h, w, comps = src.shape
    else:
        h, w = planes[0].shape
        comps = 3
    flags = C.c_uint32()
    p = [np.zeros((h, w), np.float32) for _ in range(3)] if planes is None else [
        np.ascontiguousarray(q, dtype=np.float32) for q in planes]
    dst = np.zeros((h, w, comps), np.float32)
    rc = lib.oracle_render(record.pointer(), stage, C.c_void_p(src.ctypes.data if src is not None else 0),
                           w * comps, w, h, comps, C.c_void_p(dst.ctypes.data), w * comps,
                           C.c_void_p(p[0].ctypes.data), C.c_void_p(p[1].ctypes.data), C.c_void_p(p[2].ctypes.data),
                           auto_scale, threads, C.byref(flags))
    if rc != 0:
        raise RuntimeError(f"oracle_render failed with code {rc}")
    if stage in (1, 3, 5, 6, 7):
        return p, int(flags.value)
    return dst, int(flags.value)


def scanner_lut(inp):
    import numpy as np

    lib = load()
    r = int(inp.resolution)
    outs = [np.zeros(3 * r ** 3, np.float32) for _ in range(4)] + [np.zeros(3 * (r - 1) ** 3, np.float32)
                                                                    for _ in range(2)]
    rc = lib.oracle_scanner_lut(C.byref(inp), *[C.c_void_p(o.ctypes.data) for o in outs])
    return rc, outs


REF_LIB = os.path.join(HERE, "_ref", "libjuicer_ref.so")
_ref = None


def load_reference():
    """The reference's own CUDA render kernels (oracle/_ref/libjuicer_ref.so) or None."""
    global _ref
    if _ref is not None:
        return _ref
    if not os.path.exists(REF_LIB):
        return None
    abi = _abi()
    lib = C.CDLL(REF_LIB)
    lib.ref_render.restype = C.c_int
    lib.ref_render.argtypes = [C.POINTER(abi.FjPreparedHostData), C.POINTER(C.c_void_p), C.c_void_p, C.c_long,
                               C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint32)]
    lib.ref_capture_density.restype = C.c_int
    lib.ref_capture_density.argtypes = [C.POINTER(abi.FjPreparedHostData), C.POINTER(C.c_void_p), C.c_void_p,
                                        C.c_long, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    if hasattr(lib, "ref_scanner_post"):
        lib.ref_scanner_post.restype = C.c_int
        lib.ref_scanner_post.argtypes = [C.POINTER(abi.FjPreparedHostData), C.POINTER(C.c_void_p),
                                         C.POINTER(abi.FjScannerPostEffects), C.c_ulonglong, C.c_int, C.c_int,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_void_p,
                                         C.c_long, C.c_int, C.c_int, C.c_int]
    if hasattr(lib, "ref_defects_timed"):
        lib.ref_defects_timed.restype = C.c_int
        lib.ref_defects_timed.argtypes = [C.POINTER(abi.FjFilmEffects), C.c_int, C.c_int, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p]
    if hasattr(lib, "ref_effects_render"):
        lib.ref_effects_render.restype = C.c_int
        lib.ref_effects_render.argtypes = [C.POINTER(abi.FjPreparedHostData), C.POINTER(C.c_void_p),
                                           C.POINTER(abi.FjFilmEffects), C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_long, C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_int,
                                           C.c_void_p, C.c_void_p]
    _ref = lib
    return lib


def scanner_lut_for(record):
    """The record's scanner LUT built by the oracle (word-exact to the reference)."""
    import numpy as np

    abi = _abi()
    h = record.h
    sp = h.scanner_spectra
    inp = abi.FjbScannerLutInput()
    inp.eps_c, inp.eps_m, inp.eps_y = sp.dye_c, sp.dye_m, sp.dye_y
    inp.weighted_x, inp.weighted_y, inp.weighted_z = sp.weighted_x, sp.weighted_y, sp.weighted_z
    inp.baseline_min = sp.base_density
    inp.has_baseline = 1 if sp.base_density.count else 0
    inp.sample_count = sp.dye_c.count
    inp.inv_yn = sp.inverse_y_normalization
    prt = h.route in (1, 3)
    for c in range(3):
        inp.range_min_cmy[c] = h.scanner_bounds.min_cmy[c] if prt else -h.scanner_bounds.min_cmy[c]
        inp.inverse_span_cmy[c] = h.scanner_bounds.inv_span_cmy[c]
    inp.medium = 1 if prt else 0
    inp.resolution = h.scanner_lut.resolution
    rc, outs = scanner_lut(inp)
    if rc != 0:
        raise RuntimeError("oracle scanner LUT failed")
    return [np.ascontiguousarray(o) for o in outs]


def auto_exposure(record, meter, src):
    """Exposure scale metered by the oracle (None when the record is rejected)."""
    import numpy as np

    lib = load()
    abi = _abi()
    fn = lib.oracle_auto_exposure
    fn.restype = C.c_float
    fn.argtypes = [C.POINTER(abi.FjPreparedHostData), C.POINTER(abi.FjAutoExposure), C.c_void_p, C.c_long, C.c_int,
                   C.POINTER(C.c_int)]
    src = np.ascontiguousarray(src, dtype=np.float32)
    ok = C.c_int()
    v = fn(record.pointer(), C.byref(meter), C.c_void_p(src.ctypes.data), src.shape[1] * src.shape[2], src.shape[2],
           C.byref(ok))
    return float(v) if ok.value else None


def reference_auto_exposure(torch, record, meter, src):
    """Exposure scale metered by the reference's own CUDA launchers
    (src/Cuda/JuicerCudaAutoExposure.cu:667, :864) on `src` (H, W, comps), or None when
    the harness is not built."""
    import numpy as np

    lib = load_reference()
    if lib is None or not hasattr(lib, "ref_auto_exposure"):
        return None
    abi = _abi()
    fn = lib.ref_auto_exposure
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.FjPreparedHostData), C.POINTER(C.c_void_p), C.POINTER(abi.FjAutoExposure),
                   C.c_void_p, C.c_long, C.c_int, C.POINTER(C.c_float)]
    src = np.ascontiguousarray(src, dtype=np.float32)
    h, w, comps = src.shape
    lut = scanner_lut_for(record)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    s = torch.from_numpy(src).cuda()
    out = C.c_float()
    rc = fn(record.pointer(), ptrs, C.byref(meter), C.c_void_p(s.data_ptr()), w * comps * 4, comps, C.byref(out))
    if rc != 0:
        raise RuntimeError(f"reference auto exposure returned {rc}")
    return float(out.value)


def glare_seed(recipe_hash: int, frame_token: int, x1: int, y1: int) -> int:
    """FNV-1a 64 over the little-endian 8-byte words {recipe hash, frame token, x1, y1}
    (src/Cuda/JuicerCudaExecutor.cpp:2416, src/Hash.h:50)."""
    h = 0xcbf29ce484222325
    for v in (recipe_hash, frame_token, x1, y1):
        for b in (v & 0xFFFFFFFFFFFFFFFF).to_bytes(8, "little"):
            h = ((h ^ b) * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    return h


def render_post(record, post, seed: int, origin_x: int, origin_y: int, planes, src=None, threads: int = 1):
    """Density planes (C, M, Y) -> print -> scan with scanner glare -> lens blur ->
    unsharp -> encoded output (H, W, comps). Returns (result, flags)."""
    import numpy as np

    lib = load()
    p = [np.ascontiguousarray(q, dtype=np.float32) for q in planes]
    h, w = p[0].shape
    comps = 3
    if src is not None:
        src = np.ascontiguousarray(src, dtype=np.float32)
        comps = src.shape[2]
    dst = np.zeros((h, w, comps), np.float32)
    flags = C.c_uint32()
    rc = lib.oracle_render_post(record.pointer(), C.byref(post), seed, origin_x, origin_y,
                                *[C.c_void_p(q.ctypes.data) for q in p],
                                C.c_void_p(src.ctypes.data if src is not None else 0), w * comps, w, h, comps,
                                C.c_void_p(dst.ctypes.data), w * comps, threads, C.byref(flags))
    if rc != 0:
        raise RuntimeError(f"oracle_render_post failed with code {rc}")
    return dst, int(flags.value)
