"""Colour-difference metrics for the precision reports (test infrastructure only).

CIEDE2000 follows Sharma, Wu and Dalal, "The CIEDE2000 color-difference formula:
implementation notes, supplementary test data, and mathematical observations", Color
Research & Application 30(1), 2005 (equations 1-22, kL = kC = kH = 1). Encoded sRGB
outputs are decoded with the IEC 61966-2-1 curve, converted to XYZ with the sRGB / D65
primaries matrix and to CIELAB against the D65 white.
"""
from __future__ import annotations

import numpy as np

_M_SRGB_TO_XYZ = np.array([[0.4124564, 0.3575761, 0.1804375],
                           [0.2126729, 0.7151522, 0.0721750],
                           [0.0193339, 0.1191920, 0.9503041]])
_WHITE_D65 = np.array([0.95047, 1.0, 1.08883])


def srgb_encoded_to_lab(rgb: np.ndarray) -> np.ndarray:
    """(..., 3) encoded sRGB in [0, 1] -> (..., 3) CIELAB (D65)."""
    c = np.clip(np.asarray(rgb, dtype=np.float64), 0.0, 1.0)
    lin = np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4)
    xyz = lin @ _M_SRGB_TO_XYZ.T / _WHITE_D65
    eps, kappa = 216.0 / 24389.0, 24389.0 / 27.0
    f = np.where(xyz > eps, np.cbrt(xyz), (kappa * xyz + 16.0) / 116.0)
    return np.stack([116.0 * f[..., 1] - 16.0, 500.0 * (f[..., 0] - f[..., 1]), 200.0 * (f[..., 1] - f[..., 2])], -1)


def delta_e2000(lab1: np.ndarray, lab2: np.ndarray) -> np.ndarray:
    """CIEDE2000 between two (..., 3) CIELAB arrays."""
    L1, a1, b1 = (np.asarray(lab1, dtype=np.float64)[..., i] for i in range(3))
    L2, a2, b2 = (np.asarray(lab2, dtype=np.float64)[..., i] for i in range(3))
    C1, C2 = np.hypot(a1, b1), np.hypot(a2, b2)
    Cm = 0.5 * (C1 + C2)
    G = 0.5 * (1.0 - np.sqrt(Cm ** 7 / (Cm ** 7 + 25.0 ** 7)))
    a1p, a2p = (1.0 + G) * a1, (1.0 + G) * a2
    C1p, C2p = np.hypot(a1p, b1), np.hypot(a2p, b2)
    h1p = np.where((a1p == 0) & (b1 == 0), 0.0, np.degrees(np.arctan2(b1, a1p)) % 360.0)
    h2p = np.where((a2p == 0) & (b2 == 0), 0.0, np.degrees(np.arctan2(b2, a2p)) % 360.0)
    dLp = L2 - L1
    dCp = C2p - C1p
    dh = h2p - h1p
    dh = np.where(dh > 180.0, dh - 360.0, np.where(dh < -180.0, dh + 360.0, dh))
    dh = np.where(C1p * C2p == 0, 0.0, dh)
    dHp = 2.0 * np.sqrt(C1p * C2p) * np.sin(np.radians(dh) / 2.0)
    Lpm = 0.5 * (L1 + L2)
    Cpm = 0.5 * (C1p + C2p)
    hsum = h1p + h2p
    hpm = np.where(C1p * C2p == 0, hsum,
                   np.where(np.abs(h1p - h2p) <= 180.0, 0.5 * hsum,
                            np.where(hsum < 360.0, 0.5 * (hsum + 360.0), 0.5 * (hsum - 360.0))))
    T = (1.0 - 0.17 * np.cos(np.radians(hpm - 30.0)) + 0.24 * np.cos(np.radians(2.0 * hpm))
         + 0.32 * np.cos(np.radians(3.0 * hpm + 6.0)) - 0.20 * np.cos(np.radians(4.0 * hpm - 63.0)))
    dtheta = 30.0 * np.exp(-(((hpm - 275.0) / 25.0) ** 2))
    Rc = 2.0 * np.sqrt(Cpm ** 7 / (Cpm ** 7 + 25.0 ** 7))
    Sl = 1.0 + 0.015 * (Lpm - 50.0) ** 2 / np.sqrt(20.0 + (Lpm - 50.0) ** 2)
    Sc = 1.0 + 0.045 * Cpm
    Sh = 1.0 + 0.015 * Cpm * T
    Rt = -np.sin(np.radians(2.0 * dtheta)) * Rc
    return np.sqrt((dLp / Sl) ** 2 + (dCp / Sc) ** 2 + (dHp / Sh) ** 2 + Rt * (dCp / Sc) * (dHp / Sh))


def delta_e_stats(out_a: np.ndarray, out_b: np.ndarray) -> dict:
    """p50 / p99 / max CIEDE2000 between two encoded sRGB frames (first three channels)."""
    de = delta_e2000(srgb_encoded_to_lab(out_a[..., :3]), srgb_encoded_to_lab(out_b[..., :3])).ravel()
    return {"p50": float(np.percentile(de, 50)), "p99": float(np.percentile(de, 99)), "max": float(de.max())}
