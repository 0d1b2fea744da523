"""Output gamut boundary (cmax) table, restated in Python FP64 (TEST ORACLE).

Test infrastructure: only tests/ use it, as the checker of the device build.

Follows rust/film-juicer-core/src/gamut.rs: build_output_boundary (:760-829),
boundary_cubics (:727-752), first_channel_exit (:684-726), append_derivative_roots
(:649-683), channel_inside_cube (:641-644), evaluate_cubic (:638-640). Python floats are
IEEE doubles with every operation rounded alone, as the Rust code is. The table's
lightness rows and hue directions (cos, sin of the hue, from the C library) are inputs.
"""
from __future__ import annotations

import math
import struct

import numpy as np

SLACK = float(np.float32(1e-6))
CMAX = 2.0
TOL = 1e-14


def f64(bits: int) -> float:
    return struct.unpack("<d", struct.pack("<Q", bits))[0]


def f32(bits: int) -> float:
    return float(np.uint32(bits).view(np.float32))


def cubic(c, x):
    return ((c[3] * x + c[2]) * x + c[1]) * x + c[0]


def inside(v):
    return math.isfinite(v) and v >= -SLACK and v <= 1.0 + SLACK


def roots(c, parts):
    a, b, cc = 3.0 * c[3], 2.0 * c[2], c[1]

    def add(r):
        if math.isfinite(r) and 0.0 < r < CMAX:
            parts.append(r)

    scale = abs(a)
    for v in (abs(b), abs(cc), 1.0):
        if scale < v:
            scale = v
    if abs(a) <= TOL * scale:
        if abs(b) > TOL * scale:
            add(-cc / b)
        return
    disc = b * b - 4.0 * a * cc
    if not (disc >= 0.0):
        return
    q = -0.5 * (b + math.copysign(math.sqrt(disc), b))
    if abs(q) <= TOL * scale:
        add(-b / (2.0 * a))
        return
    add(q / a)
    add(cc / q)


def first_exit(c):
    if not inside(cubic(c, 0.0)):
        return 0.0
    p = [0.0, CMAX]
    roots(c, p)
    for i in range(1, len(p)):
        v, j = p[i], i
        while j > 0 and v < p[j - 1]:
            p[j] = p[j - 1]
            j -= 1
        p[j] = v
    kept = [p[0]]
    for i in range(1, len(p)):
        if abs(kept[-1] - p[i]) <= 1e-12:
            continue
        kept.append(p[i])
    for k in range(1, len(kept)):
        lo, hi = kept[k - 1], kept[k]
        if inside(cubic(c, hi)):
            continue
        for _ in range(20):
            mid = 0.5 * (lo + hi)
            if inside(cubic(c, mid)):
                lo = mid
            else:
                hi = mid
        return lo
    return math.inf


def build(lms_to_native, directions, lab) -> np.ndarray:
    """64 x 720 float32 cmax; raises ValueError with the reference's requirement."""
    m = list(lms_to_native)
    lab = [float(v) for v in lab]
    lmin, lmax = float(np.float32(0.02)), 1.0
    out = np.empty(64 * 720, np.float32)
    for li in range(64):
        light = lmin + (lmax - lmin) * li / 63.0
        for hi, (dc, ds) in enumerate(directions):
            u = [lab[r * 3] * light for r in range(3)]
            v = [lab[r * 3 + 1] * dc + lab[r * 3 + 2] * ds for r in range(3)]
            cubics = [[0.0] * 4 for _ in range(3)]
            for ch in range(3):
                for k in range(3):
                    w = m[ch * 3 + k]
                    cubics[ch][0] += w * u[k] * u[k] * u[k]
                    cubics[ch][1] += w * 3.0 * u[k] * u[k] * v[k]
                    cubics[ch][2] += w * 3.0 * u[k] * v[k] * v[k]
                    cubics[ch][3] += w * v[k] * v[k] * v[k]
            end_out, neutral_in, fe = False, True, math.inf
            for c in cubics:
                neutral_in = neutral_in and inside(cubic(c, 0.0))
                end_out = end_out or not inside(cubic(c, CMAX))
                e = first_exit(c)
                if e < fe:
                    fe = e
            if not end_out:
                raise ValueError(f"c2_outside lightness_index={li} hue_index={hi}")
            if not neutral_in:
                fe = 0.0
            if not (math.isfinite(fe) and 0.0 <= fe <= CMAX):
                raise ValueError("finite_first_exit")
            out[li * 720 + hi] = np.float32(fe)
    return out
