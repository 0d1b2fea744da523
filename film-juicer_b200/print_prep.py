"""Print preparation on the host: the enlarger's filtered illuminants, the preflash raw
integral and the mid-grey print balance, word for word as the reference's host
computes them (rust/film-juicer-core/src/print.rs, recipe.rs, illuminant.rs).

* `filters`: main and preflash CC values from the neutral calibration and the user's
  Y/M/C dials (print.rs:120-158);
* `normalization_mode`: print exposure normalisation mode (print.rs:190-191);
* `filtered_illuminant`: the dichroic Y/M/C filters as erf edges on the 81-sample
  axis, each filter's CC as a transmittance 10^(-cc/100) and the lamp filtered by
  all three, in f32 with the reference's operation order (print.rs:616-658);
* `preflash_raw`: the paper's raw C, M, Y exposure by the film base under the preflash
  illuminant, accumulated in f64 and narrowed (print.rs:558-590);
* `balance`: the raw R, G, B integral of the baseline and the compensated mid-grey
  film densities under the main illuminant, the mid-grey factors exp(-mean ln raw),
  the normaliser of the normalisation mode and the balance's content hash
  (print.rs:435-523);
* `tungsten_kg3`: the enlarger lamp: a 3400 K Planck spectrum times the KG3 heat
  glass transmission resampled onto the axis by the reference's monotone cubic
  Hermite interpolation, normalised to mean 1 (illuminant.rs:97-128, 282-408);
* `sample_density`: the reference densities' curve lookup (film/reference.rs:74-98);
* `neutral_cmy_cc`: the calibrated neutral filtration of a paper / lamp / film
  triple, else the default (recipe.rs:1193-1215, 1709-1714), and `enlarger_illuminant`
  the lamp key of the host's lamp control (recipe.rs:1181-1192).

f32 arithmetic runs on NumPy float32 scalars (one rounding per operation, no fused
multiply-add, as the reference compiles it); erf and the single-precision power are
the C library's `erff` and `powf`, the functions the reference's native build calls.
The reference's Rust build evaluates erff with libm 0.2.15, whose words differ from
the C library's in a few samples by a few ulp; the native words are the ones this
module reproduces exactly.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import json
import math
import os
import struct
from fractions import Fraction

import numpy as np

F32 = np.float32
FNV_OFFSET = 0xCBF29CE484222325
FNV_PRIME = 0x100000001B3
MASK64 = (1 << 64) - 1
N = 81
DICHROIC_EDGES_NM = (516.0, 500.0, 610.0, 607.0)
DICHROIC_TRANSITIONS_NM = (12.0, 8.0, 8.0, 8.0)
DEFAULT_NEUTRAL_CMY_CC = (0.0, 65.0, 55.0)
ENLARGER_ILLUMINANTS = {0: "D65", 1: "D55", 2: "D50", 4: "TH-KG3-L", 5: "T", 6: "K75P", 7: "EQUAL"}
DEFAULT_ENLARGER_CHOICE = 3


def enlarger_illuminant(choice: int = DEFAULT_ENLARGER_CHOICE) -> str:
    """The enlarger lamp's key for the host's lamp control (recipe.rs:1181-1192): the
    listed choices, TH-KG3 (tungsten halogen behind KG3 heat glass) otherwise."""
    return ENLARGER_ILLUMINANTS.get(int(choice), "TH-KG3")


_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.erff.argtypes = [ctypes.c_float]
_libm.erff.restype = ctypes.c_float
_libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]
_libm.powf.restype = ctypes.c_float


class PrintPrepError(ValueError):
    """A preparation step rejected its inputs. `field` names the record the reference's
    diagnostic names (print_balance_raw, print_balance, preflash_raw,
    filtered_print_illuminant, enlarger_illuminant)."""

    def __init__(self, field: str, detail: str):
        super().__init__(f"{field}: {detail}")
        self.field = field


def erff(x) -> F32:
    return F32(_libm.erff(float(x)))


def powf(x, y) -> F32:
    return F32(_libm.powf(float(x), float(y)))


def f32_bits(v) -> int:
    return struct.unpack("<I", struct.pack("<f", float(v)))[0]


def f32_from_bits(w: int) -> F32:
    return np.array([w], dtype=np.uint32).view(np.float32)[0]


def f32_from_decimal(text: str) -> F32:
    """The f32 nearest to a decimal string, ties to even (no rounding through f64)."""
    exact = Fraction(text.strip())
    f = F32(float(exact))
    if not np.isfinite(f):
        return f
    best = None
    for c in (np.nextafter(f, F32(-np.inf)), f, np.nextafter(f, F32(np.inf))):
        if not np.isfinite(c):
            continue
        d = abs(Fraction(float(c)) - exact)
        if best is None or d < best[0] or (d == best[0] and (f32_bits(c) & 1) == 0):
            best = (d, c)
    return best[1]


def fnv_update(h: int, data: bytes) -> int:
    for b in data:
        h ^= b
        h = (h * FNV_PRIME) & MASK64
    return h


def hash_u64s(values) -> int:
    h = FNV_OFFSET
    for v in values:
        h = fnv_update(h, struct.pack("<Q", int(v) & MASK64))
    return h


def hash_finite_f32s(values) -> int | None:
    """FNV-1a of the samples' bits with either zero sign as +0; None when one is not finite."""
    h = FNV_OFFSET
    for v in values:
        v = F32(v)
        if not np.isfinite(v):
            return None
        h = fnv_update(h, struct.pack("<I", 0 if v == 0 else f32_bits(v)))
    return h


def _f32_array(values, n=None) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(values, dtype=np.float32)).reshape(-1)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} samples, got {a.size}")
    return a


def _narrow(x: float) -> F32:
    with np.errstate(over="ignore"):
        return F32(x)


def _pow10(x: float) -> float:
    """10^x in binary64 through the C library's pow (infinite past the range)."""
    try:
        return math.pow(10.0, x)
    except OverflowError:
        return math.inf


# --- filtration ------------------------------------------------------------------

def filters(neutral_cmy_cc, ui_ymc_cc=(0.0, 0.0, 0.0), preflash_m_cc=0.0, preflash_y_cc=0.0):
    """Main and preflash C, M, Y filter values (print.rs:120-131): the user's dials come
    in Y, M, C order and add to the neutral C, M, Y in reverse."""
    n = [F32(v) for v in neutral_cmy_cc]
    ui = [F32(v) for v in ui_ymc_cc]
    main = tuple(F32(n[c] + ui[2 - c]) for c in range(3))
    preflash = (n[0], F32(n[1] + F32(preflash_m_cc)), F32(n[2] + F32(preflash_y_cc)))
    return main, preflash


def normalization_mode(normalize: bool, compensate: bool) -> int:
    return int(bool(normalize)) * 2 + int(bool(compensate))


def filtered_illuminant(cmy_cc, source, edges_nm=DICHROIC_EDGES_NM, transitions_nm=DICHROIC_TRANSITIONS_NM):
    """The lamp `source` (81 samples) through the Y, M, C dichroics set to `cmy_cc`
    (print.rs:616-658). Raises PrintPrepError on a negative or non-finite sample or a
    non-positive total."""
    src = _f32_array(source, N)
    e = [F32(v) for v in edges_nm]
    t = [F32(v) for v in transitions_nm]
    one, half = F32(1.0), F32(0.5)
    out = np.zeros(N, dtype=np.float32)
    with np.errstate(all="ignore"):
        trans = [powf(10.0, F32(-F32(cc)) / F32(100.0)) for cc in cmy_cc]
        energy = F32(0.0)
        for i in range(N):
            wl = F32(380.0) + F32(5.0) * F32(i)
            y = half * erff((wl - e[0]) / t[0]) + half
            if wl <= F32(550.0):
                m_erf = -erff((wl - e[1]) / t[1])
            else:
                m_erf = erff((wl - e[2]) / t[2])
            c = F32(-0.5) * erff((wl - e[3]) / t[3]) + half
            filt = (c, half * m_erf + half, y)
            total = src[i]
            for ch in range(3):
                total = total * (one - (one - filt[ch]) * (one - trans[ch]))
            if not np.isfinite(total) or total < 0:
                raise PrintPrepError("filtered_print_illuminant", f"sample {i}")
            out[i] = total
            energy = energy + total
    if not np.isfinite(energy) or energy <= 0:
        raise PrintPrepError("filtered_print_illuminant", "energy")
    return out


# --- integrals -------------------------------------------------------------------

def preflash_raw(film_base_density, filtered_illuminant_, sensitivity_cmy):
    """Raw C, M, Y of the film base under the preflash illuminant (print.rs:558-590)."""
    base = _f32_array(film_base_density, N)
    ill = _f32_array(filtered_illuminant_, N)
    sens = _f32_array(sensitivity_cmy, 3 * N).reshape(N, 3)
    raw = [0.0, 0.0, 0.0]
    for i in range(N):
        light = _pow10(-float(base[i])) * float(ill[i])
        if math.isnan(light):
            light = 0.0
        for c in range(3):
            s = sens[i, c]
            if np.isfinite(s):
                raw[c] += light * float(s)
    out = np.zeros(3, dtype=np.float32)
    for c in range(3):
        if not math.isfinite(raw[c]) or raw[c] < 0:
            raise PrintPrepError("preflash_raw", f"channel {c}")
        out[c] = _narrow(raw[c])
    return out


class Balance:
    """The mid-grey print balance (print.rs:435-523): raw R, G, B of the baseline and
    compensated densities, the two mid-grey factors, the normaliser and the hashes."""

    def __init__(self, baseline_density_cmy, compensated_density_cmy, reference_hash: int, mode: int,
                 film_base_density, film_channel_density_cmy, sensitivity_rgb, filtered_main_illuminant):
        base = _f32_array(film_base_density, N)
        dens = _f32_array(film_channel_density_cmy, 3 * N).reshape(N, 3)
        sens = _f32_array(sensitivity_rgb, 3 * N).reshape(N, 3)
        ill = _f32_array(filtered_main_illuminant, N)

        def integrate(dcmy):
            dcmy = _f32_array(dcmy, 3)
            acc = [0.0, 0.0, 0.0]
            for i in range(N):
                d = float(base[i])
                for c in range(3):
                    d += float(dcmy[c]) * float(dens[i, c])
                light = _pow10(-d) * float(ill[i])
                if math.isnan(light):
                    continue
                for c in range(3):
                    s = sens[i, c]
                    if np.isfinite(s):
                        acc[c] += light * float(s)
            raw = np.zeros(3, dtype=np.float32)
            for c in range(3):
                raw[c] = _narrow(acc[c])
                if not np.isfinite(raw[c]) or raw[c] < 0:
                    return None, c
            return raw, -1

        self.baseline_raw_rgb, ch = integrate(baseline_density_cmy)
        if self.baseline_raw_rgb is None:
            raise PrintPrepError("print_balance_raw", f"baseline channel {ch}")
        self.compensated_raw_rgb, ch = integrate(compensated_density_cmy)
        if self.compensated_raw_rgb is None:
            raise PrintPrepError("print_balance_raw", f"compensated channel {ch}")

        def factor(raw):
            m = 0.0
            for v in raw:
                m += math.log(max(float(v), 1.0e-10))
            return _narrow(math.exp(-m / 3.0))

        self.factor_midgray = factor(self.baseline_raw_rgb)
        self.factor_midgray_comp = factor(self.compensated_raw_rgb)
        with np.errstate(all="ignore"):
            self.normalizer = {0: F32(1.0), 1: self.factor_midgray_comp / self.factor_midgray,
                               2: self.factor_midgray, 3: self.factor_midgray_comp}.get(int(mode), F32(np.nan))
        self.filtered_main_illuminant_hash = hash_finite_f32s(ill) or 0
        self.hash = hash_u64s([reference_hash, self.filtered_main_illuminant_hash,
                               hash_finite_f32s(self.baseline_raw_rgb) or 0,
                               hash_finite_f32s(self.compensated_raw_rgb) or 0,
                               f32_bits(self.factor_midgray), f32_bits(self.factor_midgray_comp),
                               f32_bits(self.normalizer)])
        ok = all(np.isfinite(v) and v > 0 for v in (self.factor_midgray, self.factor_midgray_comp, self.normalizer))
        if not ok or self.filtered_main_illuminant_hash == 0 or self.hash == 0:
            raise PrintPrepError("print_balance", "invalid balance")

    @property
    def scalars(self):
        return (self.factor_midgray, self.factor_midgray_comp, self.normalizer)


# --- the enlarger lamp -------------------------------------------------------------

def _wavelength(i: int) -> F32:
    return F32(380.0) + F32(5.0) * F32(i)


def planck(wavelength_nm, temperature_k) -> F32:
    """Spectral radiance of a black body in binary64, narrowed (illuminant.rs:100-114)."""
    lam = float(F32(wavelength_nm)) * 1e-9
    c, h, k = 2.99792458e8, 6.62607015e-34, 1.380649e-23
    c1 = 2.0 * h * c * c
    c2 = h * c / k
    den = math.exp(c2 / (lam * float(F32(temperature_k)))) - 1.0
    return _narrow(c1 / (math.pow(lam, 5.0) * den) if den > 0 else 0.0)


def normalize_mean(samples: np.ndarray) -> np.ndarray:
    s = 0.0
    for v in samples:
        s += float(v)
    mean = s / samples.size
    if mean > 0:
        return np.array([_narrow(float(v) / mean) for v in samples], dtype=np.float32)
    return samples


def parse_csv_rows(text: str) -> list:
    """Two-column CSV rows (wavelength nm, value) as f32 pairs, each field rounded once."""
    rows = []
    for line in text.splitlines():
        parts = [p for p in line.replace(";", ",").split(",") if p.strip()]
        if len(parts) < 2:
            continue
        try:
            rows.append((f32_from_decimal(parts[0]), f32_from_decimal(parts[1])))
        except (ValueError, ZeroDivisionError):
            continue
    return rows


def resample(rows) -> np.ndarray:
    """Samples of the rows on the 380-780 nm / 5 nm axis (illuminant.rs:282-392):
    rows already on the axis pass through; otherwise a piecewise cubic Hermite through
    the finite rows sorted by wavelength (first of equal wavelengths kept) whose
    slopes blend the neighbouring secants, weighted by the secant differences on
    either side (two end secants extrapolated linearly); NaN outside the rows' span."""
    if len(rows) == N and all(abs(float(F32(r[0]) - _wavelength(i))) <= 1e-3 for i, r in enumerate(rows)):
        return np.array([r[1] for r in rows], dtype=np.float32)
    pts = [(F32(r[0]), F32(r[1]), i) for i, r in enumerate(rows) if np.isfinite(r[0]) and np.isfinite(r[1])]
    pts.sort(key=lambda p: (float(p[0]), p[2]))
    uniq = []
    for p in pts:
        if not uniq or uniq[-1][0] != p[0]:
            uniq.append(p)
    n = len(uniq)
    if n < 2:
        raise PrintPrepError("enlarger_illuminant", "resample needs two finite unique points")
    x = [float(p[0]) for p in uniq]
    y = [float(p[1]) for p in uniq]
    slopes = [0.0] * n
    if n == 2:
        s = (y[1] - y[0]) / (x[1] - x[0])
        slopes = [s, s]
    else:
        ext = [0.0] * (n + 3)
        for i in range(n - 1):
            ext[i + 2] = (y[i + 1] - y[i]) / (x[i + 1] - x[i])
        ext[1] = 2.0 * ext[2] - ext[3]
        ext[0] = 2.0 * ext[1] - ext[2]
        ext[n + 1] = 2.0 * ext[n] - ext[n - 1]
        ext[n + 2] = 2.0 * ext[n + 1] - ext[n]
        defaults = [0.5 * (ext[i] + ext[i + 3]) for i in range(n)]
        diff = [abs(ext[i + 1] - ext[i]) for i in range(n + 2)]
        fwd = [diff[i + 2] for i in range(n)]
        bwd = [diff[i] for i in range(n)]
        sums = [fwd[i] + bwd[i] for i in range(n)]
        top = 0.0
        for v in sums:
            if top < v:
                top = v
        cutoff = 1e-9 * top
        for i in range(n):
            s = defaults[i]
            if sums[i] > cutoff:
                s = ext[i + 1] + bwd[i] * (ext[i + 2] - ext[i + 1]) / sums[i]
            slopes[i] = s
    coef = []
    for i in range(n - 1):
        inv = 1.0 / (x[i + 1] - x[i])
        inv2 = inv * inv
        delta = (y[i + 1] - y[i]) * inv
        coef.append((y[i], slopes[i], (3.0 * delta - 2.0 * slopes[i] - slopes[i + 1]) * inv,
                     (slopes[i] + slopes[i + 1] - 2.0 * delta) * inv2))
    out = np.zeros(N, dtype=np.float32)
    for j in range(N):
        w = float(_wavelength(j))
        if w < x[0] or w > x[-1]:
            out[j] = np.nan
            continue
        upper = 0
        while upper < n and x[upper] <= w:
            upper += 1
        seg = min(max(upper, 1), n - 1) - 1
        off = w - x[seg]
        c0, c1, c2, c3 = coef[seg]
        v = c3
        v = v * off + c2
        v = v * off + c1
        v = v * off + c0
        out[j] = _narrow(v)
    return out


def tungsten_kg3(kg3_rows) -> np.ndarray:
    """The TH-KG3 enlarger lamp: Planck 3400 K times the KG3 transmission, mean 1
    (illuminant.rs:394-408). The rows must cover 370-790 nm."""
    finite = [float(r[0]) for r in kg3_rows if np.isfinite(r[0])]
    if not finite or min(finite) > 370.0 or max(finite) < 790.0:
        raise PrintPrepError("enlarger_illuminant", "KG3 filter coverage incomplete")
    kg3 = resample(kg3_rows)
    with np.errstate(invalid="ignore"):
        samples = np.array([planck(_wavelength(i), 3400.0) * kg3[i] for i in range(N)], dtype=np.float32)
    return normalize_mean(samples)


def sample_density(query, axis, curves, channel: int):
    """Density of `channel` at log exposure `query` by linear interpolation on the
    nondecreasing f32 axis, clamped to the end rows, in f32 (film/reference.rs:74-98);
    None for a NaN query."""
    q = F32(query)
    if np.isnan(q):
        return None
    axis = np.asarray(axis, dtype=np.float32)
    curves = np.asarray(curves, dtype=np.float32)
    if q <= axis[0]:
        return curves[0, channel]
    if q >= axis[-1]:
        return curves[-1, channel]
    hi = int(np.searchsorted(axis, q, side="right"))
    if hi == 0 or hi == axis.size:
        return None
    lo = hi - 1
    span = axis[hi] - axis[lo]
    t = (q - axis[lo]) / span if span > 0 else F32(0.0)
    return curves[lo, channel] + t * (curves[hi, channel] - curves[lo, channel])


def linear_sensitivity(log_sensitivity) -> np.ndarray:
    """10^log in f32 through powf, non-finite -> 0 (profile/sampled.rs:419-424)."""
    a = np.asarray(log_sensitivity, dtype=np.float32)
    out = np.array([powf(10.0, v) for v in a.reshape(-1)], dtype=np.float32).reshape(a.shape)
    return np.where(np.isfinite(out), out, np.float32(0.0)).astype(np.float32)


def neutral_cmy_cc(resources: str, paper: str, illuminant: str, film: str):
    """The calibrated neutral C, M, Y filtration for (paper, lamp, film) from
    filters/neutral_print_filters.json, else the default filtration."""
    path = os.path.join(resources, "filters", "neutral_print_filters.json")
    try:
        with open(path) as fh:
            table = json.load(fh)
        cc = table[paper][illuminant][film]
        return tuple(F32(v) for v in cc), True
    except (OSError, KeyError, ValueError, TypeError):
        return tuple(F32(v) for v in DEFAULT_NEUTRAL_CMY_CC), False
