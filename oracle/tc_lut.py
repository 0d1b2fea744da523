"""TC LUT construction, restated in NumPy float32 (TEST ORACLE).

Test infrastructure: only tests/ use it, as the checker of the device build.

Follows rust/film-juicer-core/src/reconstruction.rs (build_tc_lut :594-677,
blur_spectra :540-569, gaussian_kernel :227-268, gaussian_reflect_index :270-279,
sample_mitchell :501-538, mitchell_weight :139-157, mitchell_coordinate :159-169,
mitchell_reflect_index :171-180, projected_white :124-137, tri2quad :352-356) for the
Hanatos irradiance method (optionally with spectral blur) and the Arctic reflectance
method, and the Hanatos surface correction (eval_hanatos_surface :570-593, exp2 from
the C library as f32::exp2 is), and the input-compression remap (gamut.rs:259-373:
ray_polygon_distance, knee, compress, bilinear, remap_tc_lut; FP64 with the C
library's hypot and pow). Every
float32 product and sum is rounded on its own, as the Rust code is (no fused
multiply-add); reductions run in the reference's order. Raises ValueError with the
reference's requirement name where it fails.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

F = np.float32
# the C library's expf, which the reference's f32::exp calls on this platform
_libm = C.CDLL("libm.so.6")
_libm.expf.restype = C.c_float
_libm.expf.argtypes = [C.c_float]
_libm.exp2f.restype = C.c_float
_libm.exp2f.argtypes = [C.c_float]
for _fn, _n in (("hypot", 2), ("pow", 2)):
    getattr(_libm, _fn).restype = C.c_double
    getattr(_libm, _fn).argtypes = [C.c_double] * _n
CELLS = 192 * 192


def procedural_spectra() -> np.ndarray:
    """The characterization's source: word i = 0x3e000123 + (i % 4093) * 173."""
    i = np.arange(CELLS * 81, dtype=np.uint64)
    return (np.uint64(0x3E000123) + (i % np.uint64(4093)) * np.uint64(173)).astype(np.uint32).view(np.float32)


def gaussian_kernel(sigma: np.float32) -> np.ndarray:
    rounded = F(F(4.0) * sigma + F(0.5))
    if not np.isfinite(rounded) or rounded < 1.0:
        raise ValueError("finite_blur_kernel")
    radius = int(rounded)
    s2 = F(sigma * sigma)
    w = []
    total = F(0.0)
    for k in range(2 * radius + 1):
        off = k - radius
        v = F(_libm.expf(float(F(F(F(-0.5) * F(off * off)) / s2))))
        w.append(v)
        total = F(total + v)
    if not np.isfinite(total) or total <= 0.0:
        raise ValueError("finite_blur_kernel")
    return np.array([F(v / total) for v in w], dtype=np.float32)


def blur(spectra: np.ndarray, sigma: np.float32) -> np.ndarray:
    k = gaussian_kernel(sigma)
    r = len(k) // 2
    src = spectra.reshape(CELLS, 81)
    out = np.empty_like(src)
    for s in range(81):
        v = np.zeros(CELLS, np.float32)
        for j, w in enumerate(k):
            q = (s + j - r) % 162
            q = 161 - q if q >= 81 else q
            v = (v + (w * src[:, q]).astype(np.float32)).astype(np.float32)
        out[:, s] = v
    if not np.all(np.isfinite(out)):
        raise ValueError("finite_blurred_spectra")
    return out.reshape(-1)


def mitchell_weight(t: np.float32) -> np.float32:
    B = F(1.0) / F(3.0)
    C = B
    x = F(abs(t))
    if x < 1.0:
        a = F(F(F(12.0) - F(F(9.0) * B)) - F(F(6.0) * C))
        b = F(F(F(-18.0) + F(F(12.0) * B)) + F(F(6.0) * C))
        c = F(F(6.0) - F(F(2.0) * B))
        return F(F(F(1.0) / F(6.0)) * F(F(F(F(a * x) * x) * x) + F(F(b * x) * x) + c))
    if x < 2.0:
        a = F(-B - F(F(6.0) * C))
        b = F(F(F(6.0) * B) + F(F(30.0) * C))
        c = F(F(F(-12.0) * B) - F(F(48.0) * C))
        d = F(F(F(8.0) * B) + F(F(24.0) * C))
        return F(F(F(1.0) / F(6.0)) * F(F(F(F(F(a * x) * x) * x) + F(F(b * x) * x)) + F(c * x) + d))
    return F(0.0)


def tri2quad(tx: np.float32, ty: np.float32):
    x = F(F(1.0) - tx)
    den = F(1e-10) if x < F(1e-10) else x
    return F(min(max(F(x * x), 0.0), 1.0)), F(min(max(F(ty / den), 0.0), 1.0))


def projected_white(white) -> tuple:
    w = [F(v) for v in white]
    s = F(F(w[0] + w[1]) + w[2])
    if not np.isfinite(s) or s <= 0.0:
        raise ValueError("finite_d65_projection_white")
    c, m = tri2quad(F(w[0] / s), F(w[1] / s))
    if not (np.isfinite(c) and np.isfinite(m)):
        raise ValueError("finite_d65_projection_white")
    return c, m


def sample_mitchell(spectra: np.ndarray, tc, sample: int) -> np.float32:
    def coord(v):
        v = F(F(min(max(v, F(0.0)), F(1.0))) * F(191.0))
        if v >= 191.0:
            return 190, F(1.0)
        b = int(np.floor(v))
        return b, F(v - F(b))

    def refl(i):
        return -i if i < 0 else (382 - i if i >= 192 else i)

    cb, cf = coord(tc[0])
    mb, mf = coord(tc[1])
    cw = [mitchell_weight(F(cf + F(1.0))), mitchell_weight(cf), mitchell_weight(F(cf - F(1.0))),
          mitchell_weight(F(cf - F(2.0)))]
    mw = [mitchell_weight(F(mf + F(1.0))), mitchell_weight(mf), mitchell_weight(F(mf - F(1.0))),
          mitchell_weight(F(mf - F(2.0)))]
    value = F(0.0)
    wsum = F(0.0)
    for dc in range(4):
        c = refl(cb - 1 + dc)
        for dm in range(4):
            m = refl(mb - 1 + dm)
            w = F(cw[dc] * mw[dm])
            wsum = F(wsum + w)
            value = F(value + F(w * spectra[(c * 192 + m) * 81 + sample]))
    return F(value / wsum) if wsum != 0.0 else F(0.0)


def surface_factors(params: np.ndarray, center) -> np.ndarray:
    """exp2 of the Hanatos surface polynomial at every node, (192 * 192, 3) float32."""
    out = np.empty((CELLS, 3), np.float32)
    for c in range(192):
        tcc = F(F(c) / F(191.0))
        for m in range(192):
            tcm = F(F(m) / F(191.0))
            x = F(tcc - center[0])
            y = F(tcm - center[1])
            x2, y2 = F(x * x), F(y * y)
            x3, y3 = F(x2 * x), F(y2 * y)
            for ch in range(3):
                p = params[ch]
                raw = F(p[1] * x)
                raw = F(raw + F(p[2] * y))
                raw = F(raw + F(p[3] * x2))
                raw = F(raw + F(p[4] * y2))
                raw = F(raw + F(F(p[5] * x) * y))
                raw = F(raw + F(p[6] * x3))
                raw = F(raw + F(p[7] * y3))
                raw = F(raw + F(F(p[8] * x2) * y))
                raw = F(raw + F(F(p[9] * x) * y2))
                raw = F(raw + F(F(p[10] * x2) * x2))
                raw = F(raw + F(F(p[11] * y2) * y2))
                raw = F(raw + F(F(p[12] * x3) * y))
                raw = F(raw + F(F(p[13] * x2) * y2))
                raw = F(raw + F(F(p[14] * x) * y3))
                n = F(raw / F(2.0))
                v = F(raw / F(np.sqrt(F(F(1.0) + F(n * n)))))
                out[c * 192 + m, ch] = F(_libm.exp2f(float(v)))
    return out


def build_tc_lut(spectra: np.ndarray, sensitivity: np.ndarray, illuminant: np.ndarray, white, method: int,
                 blur_sigma: np.float32, surface=None, compression: bool = False, hull=None) -> np.ndarray:
    """192 x 192 x 4 (R, G, B, +0) float32 table; method 0 Hanatos, 2 Arctic; `surface`
    (3 x 15 float32, Hanatos only) applies the surface correction; `compression` remaps
    through the input hull (`hull` = (center, 1025 xy points), None when unavailable)."""
    sens = np.asarray(sensitivity, np.float32).reshape(81, 3)
    ill = np.asarray(illuminant, np.float32)
    if not np.all(np.isfinite(ill) & (ill >= 0.0)):
        raise ValueError("finite_nonnegative_reference_illuminant")
    selected = spectra
    if method == 0 and blur_sigma > 0.0:
        if not np.isfinite(blur_sigma):
            raise ValueError("finite_blur")
        selected = blur(spectra, F(blur_sigma))
    den = [F(1.0)] * 3
    if method == 2:
        tc = projected_white(white)
        den = [F(0.0)] * 3
        for s in range(81):
            relit = F(sample_mitchell(selected, tc, s) * ill[s])
            for c in range(3):
                den[c] = F(den[c] + F(relit * sens[s, c]))
        if not all(np.isfinite(d) and d > 0.0 for d in den):
            raise ValueError("finite_positive_neutral_response")
    factors = None
    if method == 0 and surface is not None:
        try:
            center = projected_white(white)
        except ValueError:
            raise ValueError("finite_surface_reference_white") from None
        factors = surface_factors(np.asarray(surface, np.float32).reshape(3, 15), center)
    src = selected.reshape(CELLS, 81)
    raw = np.zeros((CELLS, 3), np.float32)
    for s in range(81):
        e = src[:, s]
        if method == 2:
            e = (e * ill[s]).astype(np.float32)
        raw = (raw + (e[:, None] * sens[s][None, :]).astype(np.float32)).astype(np.float32)
    out = np.zeros((CELLS, 4), np.float32)
    for c in range(3):
        out[:, c] = (raw[:, c] / den[c]).astype(np.float32)
        if factors is not None:
            out[:, c] = (out[:, c] * factors[:, c]).astype(np.float32)
    if not np.all(np.isfinite(out[:, :3])):
        raise ValueError("finite_integrated_samples")
    if compression:
        if hull is None:
            raise ValueError("input_compression_hull")
        return remap(out.reshape(-1), remap_coordinates(*hull))
    return out.reshape(-1)


def digest(table: np.ndarray) -> int:
    """FNV-1a over the little-endian bytes of the table's words."""
    h = 0xCBF29CE484222325
    for b in np.ascontiguousarray(table, np.float32).tobytes():
        h ^= b
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def remap_coordinates(center, hull_xy) -> np.ndarray:
    """TC coordinates every node reads after the input compression, (192 * 192, 2) float32."""
    c0, c1 = float(F(center[0])), float(F(center[1]))
    poly = np.asarray(hull_xy, np.float32).astype(np.float64)
    cc = np.arange(192, dtype=np.float32)
    root = np.sqrt((cc / F(191.0)).astype(np.float32)).astype(np.float32)
    mm = (np.arange(192, dtype=np.float32) / F(191.0)).astype(np.float32)
    x = np.repeat((F(1.0) - root).astype(np.float32), 192)
    y = (mm[None, :] * root[:, None]).astype(np.float32).reshape(-1)
    dx = x.astype(np.float64) - c0
    dy = y.astype(np.float64) - c1
    dist = np.array([_libm.hypot(a, b) for a, b in zip(dx, dy)])
    near = dist < 1e-9
    with np.errstate(divide="ignore", invalid="ignore"):
        ux, uy = dx / dist, dy / dist
        best = np.full(dist.shape, np.inf)
        for k in range(len(poly) - 1):
            ax, ay = poly[k]
            ex, ey = poly[k + 1, 0] - ax, poly[k + 1, 1] - ay
            den = ux * ey - uy * ex
            ox, oy = c0 - ax, c1 - ay
            d = (-ox * ey + oy * ex) / den
            pos = (-ox * uy + oy * ux) / den
            ok = (np.abs(den) > 1e-12) & (d > 1e-9) & (d < best) & (pos >= -1e-9) & (pos <= 1.0 + 1e-9)
            best = np.where(ok, d, best)
    out = np.empty((CELLS, 2), np.float32)
    for n in range(CELLS):
        if near[n]:
            cx, cy = x[n], y[n]
        else:
            b = best[n]
            if not np.isfinite(b) or b <= 1e-12:
                raise ValueError("usable_compressed_coordinates")
            t = dist[n] / b
            if t > 0.815:
                s = 1.0 - 0.815
                u = (t - 0.815) / s
                t = 0.815 + s * (u / _libm.pow(1.0 + _libm.pow(u, 1.2), 1.0 / 1.2))
            cd = t * b
            rx, ry = c0 + ux[n] * cd, c1 + uy[n] * cd
            if not (np.isfinite(rx) and np.isfinite(ry)):
                raise ValueError("usable_compressed_coordinates")
            cx, cy = F(rx), F(ry)
        out[n] = tri2quad(F(cx), F(cy))
    return out


def remap(table: np.ndarray, coords: np.ndarray) -> np.ndarray:
    """Bilinear resampling of the table at the compressed coordinates (float32, unfused)."""
    t = table.reshape(CELLS, 4)
    cp = (np.clip(coords[:, 0], F(0.0), F(1.0)) * F(191.0)).astype(np.float32)
    mp = (np.clip(coords[:, 1], F(0.0), F(1.0)) * F(191.0)).astype(np.float32)
    if not (np.all(np.isfinite(cp)) and np.all(np.isfinite(mp))):
        raise ValueError("usable_sampling_coordinates")
    c0 = np.floor(cp).astype(np.int64)
    m0 = np.floor(mp).astype(np.int64)
    c1, m1 = np.minimum(c0 + 1, 191), np.minimum(m0 + 1, 191)
    cf = (cp - c0.astype(np.float32)).astype(np.float32)
    mf = (mp - m0.astype(np.float32)).astype(np.float32)
    out = np.zeros((CELLS, 4), np.float32)
    for ch in range(3):
        v = lambda c, m: t[c * 192 + m, ch]
        r0 = (v(c0, m0) + (cf * (v(c1, m0) - v(c0, m0)).astype(np.float32)).astype(np.float32)).astype(np.float32)
        r1 = (v(c0, m1) + (cf * (v(c1, m1) - v(c0, m1)).astype(np.float32)).astype(np.float32)).astype(np.float32)
        out[:, ch] = (r0 + (mf * (r1 - r0).astype(np.float32)).astype(np.float32)).astype(np.float32)
    if not np.all(np.isfinite(out[:, :3])):
        raise ValueError("finite_remapped_samples")
    return out.reshape(-1)
