"""Capture-film DIR coupler recipe on the host, as the reference's host builds it
(rust/film-juicer-core/src/film/dir.rs:135-365, film.rs:72-93,
profile/sampled.rs:440-505):

* `processing_defaults`: the stock DIR gammas (same-layer R, G, B and the three
  interlayer pairs) by polarity, usage and reference illuminant, with the three
  per-stock overrides;
* `normalized_curves`: the development's density curves minus their per-channel
  minimum, in f32, the minimum and maximum kept with the reference's ordered
  comparisons, and the curves' NaN-masked content hash;
* `DirRecipe`: the coupler matrix [donor][receiver] (gammas x inhibitions x amount,
  f32), the density maximum and reference (half the maximum), the donor Langmuir knees
  (negative stocks) or receiver references and knees (positive stocks), the three
  compensated log-exposure axes x - sum_d donor_d(D(x)) M[d][r] (binary64, narrowed)
  and the recipe's content hashes;
* `capture_defaults`: the capture DIR controls a fresh recipe starts from.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .print_prep import FNV_OFFSET, MASK64, f32_bits, fnv_update

F32 = np.float32
MODE_INACTIVE, MODE_NEGATIVE_DONOR, MODE_POSITIVE_RECEIVER = 0, 1, 2
F32_MAX = float(np.finfo(np.float32).max)


class DirPrepError(ValueError):
    def __init__(self, kind: str, detail: str = ""):
        super().__init__(f"dir {kind} {detail}".strip())
        self.kind = kind


@dataclass
class DirParams:
    """Capture DIR controls (film/dir.rs Params)."""

    active: bool = True
    amount: float = 1.0
    inhibition_same_layer: float = 1.0
    inhibition_interlayer: float = 1.0
    diffusion_size_um: float = 20.0
    diffusion_tail_um: float = 200.0
    diffusion_tail_weight: float = 0.03
    gamma_use_stock: bool = True
    gamma_same_layer_rgb: tuple = (0.341, 0.324, 0.273)
    gamma_interlayer_r_to_gb: tuple = (0.355, 0.305)
    gamma_interlayer_g_to_rb: tuple = (0.154, 0.358)
    gamma_interlayer_b_to_rg: tuple = (0.171, 0.225)
    langmuir_donor_k_rgb: tuple = (1.0, 1.0, 1.0)
    langmuir_receiver_k_rgb: tuple = (1.0, 1.0, 1.0)


def capture_defaults(active: bool = True, gamma_use_stock: bool = True) -> DirParams:
    """The controls of a fresh capture recipe (film/dir.rs:443-460)."""
    return DirParams(active=active, gamma_use_stock=gamma_use_stock)


# (same R, G, B), (R -> G, B), (G -> R, B), (B -> R, G) per family and per stock
_DEFAULTS_POSITIVE = ((0.2291, 0.1029, 0.2651), (0.1449, 0.1560), (0.0496, 0.0874), (0.0571, 0.2462))
_DEFAULTS_CINE_TUNGSTEN = ((0.4601, 0.4433, 0.4414), (0.4313, 0.3157), (0.3145, 0.3890), (0.2423, 0.2506))
_DEFAULTS_CINE = ((0.5456, 0.5434, 0.3766), (0.4263, 0.2781), (0.2051, 0.5015), (0.2950, 0.2449))
_DEFAULTS_STILL = ((0.5159, 0.5934, 0.2829), (0.4032, 0.2488), (0.2227, 0.4340), (0.1829, 0.1799))
_DEFAULTS_STOCK = {
    "fujifilm_velvia_100": ((0.2398, 0.0662, 0.1440), (0.0707, 0.2367), (0.0119, 0.0380), (0.0111, 0.1413)),
    "kodak_kodachrome_64": ((0.2942, 0.0841, 0.2492), (0.1699, 0.2188), (0.0625, 0.0692), (0.1153, 0.2359)),
    "fujifilm_provia_100f": ((0.2786, 0.1257, 0.3480), (0.1448, 0.2003), (0.0516, 0.1250), (0.0518, 0.3089)),
}


def processing_defaults(info: dict):
    """Stock DIR gammas of a film profile's info block (profile/sampled.rs:440-490)."""
    positive = info.get("type") == "positive"
    cine = info.get("use") == "cine"
    if positive:
        d = _DEFAULTS_POSITIVE
    elif cine and str(info.get("reference_illuminant", "")).startswith("T"):
        d = _DEFAULTS_CINE_TUNGSTEN
    elif cine:
        d = _DEFAULTS_CINE
    else:
        d = _DEFAULTS_STILL
    d = _DEFAULTS_STOCK.get(info.get("stock", ""), d)
    return tuple(tuple(F32(v) for v in part) for part in d)


def nan_mask_hash(samples) -> tuple[int, int]:
    """(values, nan_mask) FNV-1a pair: NaNs hash as +0 with a bit set in a 64-sample mask
    word, either zero sign as +0, other bits unchanged."""
    values, mask = FNV_OFFSET, FNV_OFFSET
    a = np.asarray(samples, dtype=np.float32).reshape(-1)
    for start in range(0, a.size, 64):
        word = 0
        for bit, v in enumerate(a[start:start + 64]):
            if np.isnan(v):
                word |= 1 << bit
                b = 0
            elif v == 0:
                b = 0
            else:
                b = f32_bits(v)
            values = fnv_update(values, int(b).to_bytes(4, "little"))
        mask = fnv_update(mask, int(word).to_bytes(8, "little"))
    return values, mask


def _u64s(values) -> int:
    h = FNV_OFFSET
    for v in values:
        h = fnv_update(h, (int(v) & MASK64).to_bytes(8, "little"))
    return h


def curve_hash(samples) -> int:
    return _u64s(nan_mask_hash(samples))


def normalized_curves(curves):
    """Curves [n, 3] minus their per-channel minimum in f32 (film.rs:72-93): returns
    (normalized, minimum, maximum, hash of the normalized curves)."""
    c = np.array(curves, dtype=np.float32).reshape(-1, 3)
    lo, hi = c[0].copy(), c[0].copy()
    for row in c:
        for ch in range(3):
            if row[ch] < lo[ch]:
                lo[ch] = row[ch]
            if hi[ch] < row[ch]:
                hi[ch] = row[ch]
    with np.errstate(invalid="ignore", over="ignore"):
        out = (c - lo[None, :]).astype(np.float32)
    return out, lo, hi, curve_hash(out)


def _langmuir(value: float, knee: float, reference: float):
    den = knee + value
    res = value * (knee + reference) / den if den != 0.0 else float("nan")
    return res if (den != 0.0 and np.isfinite(res)) else None


def recipe_identity(positive: bool, matrix, density_max, density_ref, donor_k, receiver_c_ref, receiver_kr,
                    axes_hash: int, diffusion) -> int:
    """The recipe's content identity (film/dir.rs:324-359): version 3, polarity and mode,
    the f32 words of the matrix and the five per-channel vectors, the axes hash, then the
    diffusion core size and tail weight when a core is set and the tail width when the
    tail has weight. `diffusion` is (core um, tail um, tail weight)."""
    ident = fnv_update(FNV_OFFSET, (3).to_bytes(8, "little"))
    ident = fnv_update(ident, bytes([1 if positive else 0, 2 if positive else 1]))
    for values in list(np.asarray(matrix, np.float32).reshape(3, 3)) + [density_max, density_ref, donor_k,
                                                                         receiver_c_ref, receiver_kr]:
        for v in np.asarray(values, np.float32):
            ident = fnv_update(ident, f32_bits(v).to_bytes(4, "little"))
    ident = fnv_update(ident, (int(axes_hash) & MASK64).to_bytes(8, "little"))
    size, tail, weight = (F32(v) for v in diffusion)
    if size > 0:
        ident = fnv_update(ident, f32_bits(size).to_bytes(4, "little"))
        ident = fnv_update(ident, f32_bits(weight).to_bytes(4, "little"))
        if weight > 0:
            ident = fnv_update(ident, f32_bits(tail).to_bytes(4, "little"))
    return ident


class DirRecipe:
    """film/dir.rs Recipe::new: the coupler recipe of a development (normalized curves
    [n, 3] on the f32 log-exposure axis) under `params`."""

    def __init__(self, curves_norm, axis, positive: bool, params: DirParams, defaults, curves_hash: int):
        self.mode = MODE_INACTIVE
        self.matrix_rgb = np.zeros((3, 3), np.float32)
        self.diffusion = np.zeros(3, np.float32)  # size um, tail um, tail weight
        self.density_max_rgb = np.zeros(3, np.float32)
        self.density_ref_rgb = np.zeros(3, np.float32)
        self.donor_k_rgb = np.zeros(3, np.float32)
        self.receiver_c_ref_rgb = np.zeros(3, np.float32)
        self.receiver_kr_rgb = np.zeros(3, np.float32)
        self.axes_rgb = None
        self.axes_hash = 0
        self.hash = 0
        self.polarity = 1 if positive else 0
        amount = F32(params.amount)
        if not (params.active and amount > 0):
            return
        size = F32(params.diffusion_size_um)
        if size > 0:
            self.diffusion[0] = size
            weight = F32(params.diffusion_tail_weight)
            if weight > 0:
                self.diffusion[2] = weight
                self.diffusion[1] = F32(params.diffusion_tail_um)
        if params.gamma_use_stock:
            same, red, green, blue = defaults
        else:
            same = tuple(F32(v) for v in params.gamma_same_layer_rgb)
            red = tuple(F32(v) for v in params.gamma_interlayer_r_to_gb)
            green = tuple(F32(v) for v in params.gamma_interlayer_g_to_rb)
            blue = tuple(F32(v) for v in params.gamma_interlayer_b_to_rg)
        s_in, i_in = F32(params.inhibition_same_layer), F32(params.inhibition_interlayer)
        unit = np.zeros((3, 3), np.float32)
        with np.errstate(over="ignore", invalid="ignore"):
            for c in range(3):
                unit[c, c] = F32(same[c]) * s_in
            unit[0, 1], unit[0, 2] = F32(red[0]) * i_in, F32(red[1]) * i_in
            unit[1, 0], unit[1, 2] = F32(green[0]) * i_in, F32(green[1]) * i_in
            unit[2, 0], unit[2, 1] = F32(blue[0]) * i_in, F32(blue[1]) * i_in
            m = (unit * amount).astype(np.float32)
        if not np.all(np.isfinite(m)):
            raise DirPrepError("matrix")
        if not np.any(m != 0):
            self.polarity = None
            self.diffusion[:] = 0
            return
        self.matrix_rgb = m
        ax = np.asarray(axis, dtype=np.float32)
        for i in range(1, ax.size):
            span = float(ax[i]) - float(ax[i - 1])
            if not np.isfinite(span) or span <= 0:
                raise DirPrepError("log_exposure", f"sample {i}")
        cn = np.asarray(curves_norm, dtype=np.float32).reshape(-1, 3)
        dmax = np.full(3, -np.inf, np.float32)
        for row in cn:
            for c in range(3):
                if np.isfinite(row[c]) and dmax[c] < row[c]:
                    dmax[c] = row[c]
        if np.any(~np.isfinite(dmax)) or np.any(dmax <= 0):
            raise DirPrepError("density_maximum")
        self.density_max_rgb = dmax
        self.density_ref_rgb = (F32(0.5) * dmax).astype(np.float32)
        self.mode = MODE_POSITIVE_RECEIVER if positive else MODE_NEGATIVE_DONOR
        with np.errstate(over="ignore", invalid="ignore"):
            if positive:
                for r in range(3):
                    ref = 0.0
                    for d in range(3):
                        ref += float(self.density_ref_rgb[d]) * float(unit[d, r])
                    self.receiver_c_ref_rgb[r] = F32(ref)
                    self.receiver_kr_rgb[r] = F32(params.langmuir_receiver_k_rgb[r]) * (
                        F32(2.0) * self.receiver_c_ref_rgb[r])
                    cr, kr = self.receiver_c_ref_rgb[r], self.receiver_kr_rgb[r]
                    if not np.isfinite(cr) or not np.isfinite(kr) or (cr > 0 and kr <= 0):
                        raise DirPrepError("receiver_k", f"channel {r}")
            else:
                for d in range(3):
                    self.donor_k_rgb[d] = F32(params.langmuir_donor_k_rgb[d]) * dmax[d]
                    if not np.isfinite(self.donor_k_rgb[d]) or self.donor_k_rgb[d] <= 0:
                        raise DirPrepError("donor_k", f"channel {d}")
        axes = np.zeros((3, ax.size), np.float32)
        for i in range(ax.size):
            donors = [0.0, 0.0, 0.0]
            for d in range(3):
                dens = float(cn[i, d])
                if positive:
                    donors[d] = float(dmax[d]) - dens
                else:
                    v = _langmuir(dens, float(self.donor_k_rgb[d]), float(self.density_ref_rgb[d]))
                    if v is None:
                        raise DirPrepError("donor_langmuir", f"channel {d} sample {i}")
                    donors[d] = v
            for r in range(3):
                corr = 0.0
                for d in range(3):
                    corr += donors[d] * float(m[d, r])
                if positive:
                    if self.receiver_c_ref_rgb[r] == 0:
                        corr = 0.0
                    else:
                        v = _langmuir(corr, float(self.receiver_kr_rgb[r]), float(self.receiver_c_ref_rgb[r]))
                        if v is None:
                            raise DirPrepError("receiver_langmuir", f"channel {r} sample {i}")
                        corr = v
                coord = float(ax[i]) - corr
                if not np.isfinite(coord) or coord < -F32_MAX or coord > F32_MAX:
                    raise DirPrepError("compensated_axis", f"channel {r} sample {i}")
                axes[r, i] = F32(coord)
        self.axes_rgb = axes
        h = fnv_update(FNV_OFFSET, (1).to_bytes(8, "little"))
        h = fnv_update(h, (int(curves_hash) & MASK64).to_bytes(8, "little"))
        for r in range(3):
            h = fnv_update(h, curve_hash(axes[r]).to_bytes(8, "little"))
        self.axes_hash = h
        self.hash = recipe_identity(positive, m, self.density_max_rgb, self.density_ref_rgb, self.donor_k_rgb,
                                    self.receiver_c_ref_rgb, self.receiver_kr_rgb, h, self.diffusion)
        if self.hash == 0 or self.axes_hash == 0:
            raise DirPrepError("zero_identity")
