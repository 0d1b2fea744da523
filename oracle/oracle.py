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
    _lib = lib
    return lib


def _abi():
    import importlib
    return importlib.import_module("film_juicer_b200.abi")


def render(record, src, *, stage: int = 0, planes=None, auto_scale: float = 1.0, threads: int = 1):
    """Runs the oracle on a host image.

    stage 0: source -> encoded output (returns (H, W, comps));
    stage 1: source -> capture density planes (returns 3 planes C, M, Y);
    stage 2: density planes -> encoded output; stage 3: source -> camera exposure
    planes B, G, R; stage 4: carrier planes B, G, R -> encoded output.
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
    if stage in (1, 3):
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
