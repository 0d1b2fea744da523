"""Oracle wrappers for the spatial-DIR stage (test infrastructure only).

The recursive components' boundary weights come from the oracle's own double-double
restatement of the reference's builder (oracle_dir_boundary in oracle.c, following
rust/film-juicer-core/src/film/dir/boundary.rs:361-489), pinned word for word on the
reference's boundary fixture (tests/test_dir_boundary.py). The oracle then restates
the reference's per-component blur schedule and the source/develop kernels. Nothing
here loads the product library."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import oracle as _o


class OracleDirComp(C.Structure):
    _fields_ = [("op", C.c_int), ("weight", C.c_float), ("radius", C.c_int), ("taps", C.POINTER(C.c_float)),
                ("ff", C.c_double), ("fb", C.c_double * 3), ("h_init", C.POINTER(C.c_double)), ("h_len", C.c_int),
                ("h_ts", C.c_int), ("h_term", C.c_double * 9), ("v_init", C.POINTER(C.c_double)),
                ("v_len", C.c_int), ("v_ts", C.c_int), ("v_term", C.c_double * 9)]


def boundary(g, length):
    """(weights [3 x retained], retained, terminal size, terminal [9]) of one axis."""
    lib = _o.load()
    fn = lib.oracle_dir_boundary
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(C.c_double), C.c_double, C.c_double, C.c_uint, C.c_int, C.POINTER(C.c_double),
                   C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
    coeff = (C.c_double * 9)(g.feedforward, g.feedback[0], g.feedback[1], g.feedback[2], g.normalization_denominator,
                             g.feedforward_numerator, g.feedback_numerators[0], g.feedback_numerators[1],
                             g.feedback_numerators[2])
    w = (C.c_double * (3 * max(length, 1)))()
    t = (C.c_double * 9)()
    n, ts = C.c_int(), C.c_int()
    rc = fn(coeff, g.boundary_truncation_accuracy, g.boundary_certification_tolerance,
            g.boundary_derivation_version, length, w, C.byref(n), C.byref(ts), t)
    if rc != 0:
        raise RuntimeError(f"oracle DIR boundary failed with reason {rc}")
    return np.array(w[: 3 * n.value]), n.value, ts.value, np.array(t[:])


def components(spatial_dir, width, height, active_only=True):
    """OracleDirComp array (and the arrays it points into) for the active components
    (all components, in order, with active_only=False)."""
    from film_juicer_b200 import descriptors

    keep = []
    out = []
    for i in range(spatial_dir.component_count):
        g = spatial_dir.components[i]
        if active_only and not (g.weight > 0.0):
            continue
        c = OracleDirComp()
        c.weight = g.weight
        if g.reference_operator == 1:
            c.op = 1
        elif g.reference_operator == 2:
            c.op = 2
            c.radius = g.radius
            taps = descriptors.gaussian_taps(g.radius, g.sigma_px)
            keep.append(taps)
            c.taps = taps.ctypes.data_as(C.POINTER(C.c_float))
        else:
            c.op = 3
            c.ff = g.feedforward
            for k in range(3):
                c.fb[k] = g.feedback[k]
            for axis, length in (("h", width), ("v", height)):
                w, n, ts, t = boundary(g, length)
                w = np.ascontiguousarray(w)
                keep.append(w)
                setattr(c, f"{axis}_init", w.ctypes.data_as(C.POINTER(C.c_double)))
                setattr(c, f"{axis}_len", n)
                setattr(c, f"{axis}_ts", ts)
                arr = getattr(c, f"{axis}_term")
                for k in range(9):
                    arr[k] = t[k]
        out.append(c)
    arr = (OracleDirComp * max(len(out), 1))(*out)
    return arr, len(out), keep


def spatial_dir(record, spatial_dir_desc, src=None, carrier=None, width=None, height=None):
    """Returns (filtered Y, M, C), (log raw B, G, R), flags -- the oracle's spatial DIR."""
    lib = _o.load()
    abi = _o._abi()
    if src is not None:
        src = np.ascontiguousarray(src, dtype=np.float32)
        height, width, comps = src.shape
    else:
        comps = 3
    planes = [np.zeros((height, width), np.float32) for _ in range(6)]
    fn = lib.oracle_dir_source
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.FjPreparedHostData), C.c_void_p, C.c_long, C.c_int] + [C.c_void_p] * 3 + \
        [C.c_int, C.c_int] + [C.c_void_p] * 6 + [C.POINTER(C.c_uint32)]
    flags = C.c_uint32()
    cptr = [C.c_void_p(np.ascontiguousarray(p, dtype=np.float32).ctypes.data) for p in carrier] if carrier else \
        [None, None, None]
    if carrier:
        carrier = [np.ascontiguousarray(p, dtype=np.float32) for p in carrier]
        cptr = [C.c_void_p(p.ctypes.data) for p in carrier]
    rc = fn(record.pointer(), C.c_void_p(src.ctypes.data if src is not None else 0), width * comps, comps, *cptr,
            width, height, *[C.c_void_p(p.ctypes.data) for p in planes], C.byref(flags))
    if rc != 0:
        raise RuntimeError("oracle_dir_source failed")
    comps_arr, n, keep = components(spatial_dir_desc, width, height)
    blur = lib.oracle_dir_blur
    blur.restype = C.c_int
    blur.argtypes = [C.POINTER(OracleDirComp), C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    filtered = [np.zeros((height, width), np.float32) for _ in range(3)]
    for c in range(3):
        if blur(comps_arr, n, C.c_void_p(planes[c].ctypes.data), width, height, C.c_void_p(filtered[c].ctypes.data)):
            raise RuntimeError("oracle_dir_blur failed")
    del keep
    return filtered, planes[3:], int(flags.value)


def develop_spatial(record, filtered, log_raw):
    lib = _o.load()
    abi = _o._abi()
    fn = lib.oracle_develop_spatial
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.FjPreparedHostData)] + [C.c_void_p] * 6 + [C.c_int, C.c_int] + \
        [C.c_void_p] * 3 + [C.POINTER(C.c_uint32)]
    h, w = filtered[0].shape
    out = [np.zeros((h, w), np.float32) for _ in range(3)]
    flags = C.c_uint32()
    ins = [np.ascontiguousarray(p, dtype=np.float32) for p in (*filtered, *log_raw)]
    rc = fn(record.pointer(), *[C.c_void_p(p.ctypes.data) for p in ins], w, h, *[C.c_void_p(p.ctypes.data) for p in out],
            C.byref(flags))
    if rc != 0:
        raise RuntimeError("oracle_develop_spatial failed")
    return out, int(flags.value)


def reference_spatial_dir(torch, record, spatial_dir_desc, src):
    """The reference's own CUDA spatial DIR on `src` (None if the harness is absent)."""
    lib = _o.load_reference()
    if lib is None:
        return None
    abi = _o._abi()
    src = np.ascontiguousarray(src, dtype=np.float32)
    h, w, comps = src.shape
    comps_arr, n, keep = components(spatial_dir_desc, w, h, active_only=False)
    lut = _o.scanner_lut_for(record)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    fn = lib.ref_spatial_dir
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.FjPreparedHostData), C.POINTER(C.c_void_p), C.c_void_p, C.c_long, C.c_int, C.c_int,
                   C.c_int, C.POINTER(OracleDirComp), C.c_int] + [C.c_void_p] * 6
    s = torch.from_numpy(src).cuda()
    outs = [torch.zeros((h, w), device="cuda") for _ in range(6)]
    rc = fn(record.pointer(), ptrs, C.c_void_p(s.data_ptr()), w * comps * 4, w, h, comps, comps_arr, n,
            *[C.c_void_p(t.data_ptr()) for t in outs])
    del keep
    if rc != 0:
        raise RuntimeError(f"reference spatial DIR returned cudaError {rc}")
    host = [t.cpu().numpy() for t in outs]
    return host[:3], host[3:]
