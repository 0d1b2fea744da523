"""Frame descriptors of the spatial stages (host side), filled the way the reference's
Rust host builds them.

* spatial_dir_record: rust/film-juicer-core/src/film/dir/frame.rs:185-280 -- a core
  Gaussian (diffusion size / pixel size, weight 1 - tail weight) and, when the tail
  weight is positive, three tail Gaussians (tail size x {0.5360, 1.5236, 2.7684},
  amplitudes {0.1633, 0.6496, 0.1870} normalised, times the tail weight); operator
  identity for radius 0, FIR below sigma 3, the reflected recursive Gaussian from
  sigma 3 with Young-van Vliet coefficients (frame.rs:70-99), boundary accuracy 1e-11,
  tolerance 5e-7, derivation version 1 (frame.rs:60-68).
* gaussian_taps: rust/film-juicer-core/src/optics/gaussian.rs:16-52.
"""
from __future__ import annotations

import numpy as np

from . import abi

DIR_TAIL_AMPLITUDES = (0.1633, 0.6496, 0.1870)
DIR_TAIL_RATIOS = (0.5360, 1.5236, 2.7684)


def gaussian_taps(radius: int, sigma_px: float) -> np.ndarray:
    sigma = float(np.float32(sigma_px))
    s2 = sigma * sigma * 2.0
    x = np.arange(-radius, radius + 1, dtype=np.float64)
    w64 = np.exp(-(x * x) / s2)
    w32 = w64.astype(np.float32)
    total = float(np.sum(w64))
    rec = 1.0 / total if total != 0.0 else 0.0
    return (w32.astype(np.float64) * rec).astype(np.float32)


def _dir_component(g: "abi.FjDirGaussian", sigma_px: np.float32, weight: np.float32) -> None:
    g.sigma_px = float(sigma_px)
    g.weight = float(weight)
    radius = 3.0 * float(sigma_px) + 0.5
    g.radius = int(radius)
    g.boundary_truncation_accuracy = 1.0e-11
    g.boundary_certification_tolerance = 5.0e-7
    g.boundary_derivation_version = 1
    if sigma_px <= 0.0 or g.radius == 0:
        g.reference_operator = abi.FJ_DIR_OPERATOR_IDENTITY
        g.radius = 0
        return
    if sigma_px >= 3.0:
        g.reference_operator = abi.FJ_DIR_OPERATOR_YVV_REFLECT
        g.radius = int(radius)
        q = 0.98711 * float(sigma_px) - 0.96330
        q2, q3 = q * q, q * q * q
        den = 1.57825 + 2.44413 * q + 1.4281 * q2 + 0.422205 * q3
        g.normalization_denominator = den
        g.feedforward_numerator = 1.57825
        g.feedback_numerators[0] = 2.44413 * q + 2.0 * 1.4281 * q2 + 3.0 * 0.422205 * q3
        g.feedback_numerators[1] = -(1.4281 * q2 + 3.0 * 0.422205 * q3)
        g.feedback_numerators[2] = 0.422205 * q3
        g.feedforward = g.feedforward_numerator / den
        for i in range(3):
            g.feedback[i] = g.feedback_numerators[i] / den
        return
    g.reference_operator = abi.FJ_DIR_OPERATOR_FIR_REFLECT


def spatial_dir_record(pixel_size_um: float, width: int, height: int, *, diffusion_size_um: float = 20.0,
                       tail_um: float = 200.0, tail_weight: float = 0.03) -> "abi.FjSpatialDir":
    sd = abi.FjSpatialDir()
    for ext in (sd.render_extent, sd.full_frame_extent, sd.filter_domain_extent):
        ext.x, ext.y, ext.width, ext.height = 0, 0, width, height
    px = np.float32(pixel_size_um)
    tw = np.float32(tail_weight)
    comps = [(np.float32(np.float32(diffusion_size_um) / px), np.float32(np.float32(1.0) - tw))]
    if tw > 0:
        total = np.float32(np.float32(DIR_TAIL_AMPLITUDES[0]) + np.float32(DIR_TAIL_AMPLITUDES[1])
                           + np.float32(DIR_TAIL_AMPLITUDES[2]))
        tail_sigma = np.float32(np.float32(tail_um) / px)
        for a, r in zip(DIR_TAIL_AMPLITUDES, DIR_TAIL_RATIOS):
            comps.append((np.float32(tail_sigma * np.float32(r)), np.float32(tw * np.float32(np.float32(a) / total))))
    sd.component_count = len(comps)
    for i, (s, w) in enumerate(comps):
        _dir_component(sd.components[i], s, w)
    sd.recipe_hash = sd.hash = 1
    return sd


def diffusion_record(pixel_size_um: float, width: int, *, family: int = 2, scatter_fraction: float = 0.12,
                     group_weights=(0.55, 0.30, 0.15), group_lambda_um=(8.0, 40.0, 150.0), warmth: float = 0.3,
                     spatial_scale: float = 1.0, radius_fraction_of_width: float = 0.005) -> "abi.FjDiffusion":
    """A camera diffusion filter record; the radius is the given fraction of the frame
    width (0.5 % -> 10 px at 1920, 20 px at 3840, the configuration of the 1080p/4K
    benchmarks)."""
    d = abi.FjDiffusion()
    d.family = family
    d.scatter_fraction = scatter_fraction
    for i in range(3):
        d.group_weights[i] = group_weights[i]
        d.group_lambda_um[i] = group_lambda_um[i]
    d.warmth = warmth
    d.spatial_scale = spatial_scale
    d.pixel_size_um = pixel_size_um
    d.radius_px = max(1, int(round(radius_fraction_of_width * width)))
    d.sample_hash = d.hash = 1
    return d


def scanner_post_record(*, glare_percent: float = 0.0, glare_roughness: float = 0.4, glare_blur_sigma_px: float = 0.0,
                        glare_blur_radius: int = 0, lens_blur_sigma_px: float = 0.0, lens_blur_radius: int = 0,
                        unsharp_sigma_px: float = 0.0, unsharp_radius: int = 0, unsharp_amount: float = 0.0,
                        hash: int = 0x5C9E7):
    """FjScannerPostEffects as the host projects it (rust/film-juicer-plugin/src/cuda/
    projection.rs:336-352): glare on when its percent is positive; each blur on when its
    sigma is positive; the record is active when its hash is non-zero. Radii default to
    the 4 sigma + 0.5 rule when not given."""
    from . import abi

    def radius(sigma, r):
        return r if r > 0 else (int(4.0 * sigma + 0.5) if sigma > 0 else 0)

    p = abi.FjScannerPostEffects()
    p.flags = abi.FJ_POST_GLARE if glare_percent > 0 else 0
    p.glare_percent = glare_percent
    p.glare_roughness = glare_roughness
    p.glare_blur_sigma_px = glare_blur_sigma_px
    p.glare_blur_radius = radius(glare_blur_sigma_px, glare_blur_radius)
    p.lens_blur_sigma_px = lens_blur_sigma_px
    p.lens_blur_radius = radius(lens_blur_sigma_px, lens_blur_radius)
    p.unsharp_sigma_px = unsharp_sigma_px
    p.unsharp_radius = radius(unsharp_sigma_px, unsharp_radius)
    p.unsharp_amount = unsharp_amount
    p.hash = hash
    return p


def highlight_boost_record(protection: float = 1.0, sharpness: float = 4.0, peak_gain: float = 2.0,
                           recipe_hash: int = 0xB0057):
    """FjHighlightBoost: samples above `protection` are lifted so that the frame maximum
    reaches maximum * peak_gain; `sharpness` shapes the curve."""
    from . import abi

    d = abi.FjHighlightBoost()
    d.recipe_hash = recipe_hash
    d.protection = protection
    d.sharpness = sharpness
    d.peak_gain = peak_gain
    return d
