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
