"""Oracle wrappers for the visual grain stage (test infrastructure only)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import oracle as _o


def _curve_ptrs(base_cmy, layers):
    base = [np.ascontiguousarray(b, dtype=np.float32) for b in base_cmy]
    lay = [np.ascontiguousarray(layers[l][c], dtype=np.float32) for l in range(3) for c in range(3)]
    keep = base + lay
    bp = (C.c_void_p * 3)(*[b.ctypes.data for b in base])
    lp = (C.c_void_p * 9)(*[x.ctypes.data for x in lay])
    return keep, bp, lp


def visual_grain(grain, noise_record, base_cmy, layers, positive, planes_cmy):
    """CPU restatement of the grain schedule; returns new C, M, Y planes.
    base_cmy: the capture density curve values of C, M, Y; layers[layer][channel]."""
    lib = _o.load()
    abi = _o._abi()
    fn = lib.oracle_visual_grain
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.FjVisualGrain), C.POINTER(abi.FjStaticNoise), C.POINTER(C.c_void_p),
                   C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
    keep, bp, lp = _curve_ptrs(base_cmy, layers)
    out = [np.ascontiguousarray(p, dtype=np.float32).copy() for p in planes_cmy]
    h, w = out[0].shape
    rc = fn(C.byref(grain), C.byref(noise_record) if noise_record is not None else None, bp, lp, len(keep[0]),
            1 if positive else 0, *[C.c_void_p(p.ctypes.data) for p in out], w, h)
    if rc != 0:
        raise RuntimeError("oracle_visual_grain failed")
    return out


def reference_visual_grain(torch, grain, noise_record, base_cmy, layers, positive, planes_cmy):
    """The reference's own CUDA grain (None when its harness is not built)."""
    lib = _o.load_reference()
    if lib is None:
        return None
    abi = _o._abi()
    fn = lib.ref_visual_grain
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.FjVisualGrain), C.POINTER(abi.FjStaticNoise), C.POINTER(C.c_void_p),
                   C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
    keep, bp, lp = _curve_ptrs(base_cmy, layers)
    dev = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.float32)).cuda() for p in planes_cmy]
    h, w = dev[0].shape
    rc = fn(C.byref(grain), C.byref(noise_record) if noise_record is not None else None, bp, lp, len(keep[0]),
            1 if positive else 0, *[C.c_void_p(t.data_ptr()) for t in dev], w, h)
    if rc != 0:
        raise RuntimeError(f"reference visual grain returned cudaError {rc}")
    return [t.cpu().numpy() for t in dev]
