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


def film_effects_record(*, film_dust: dict | None = None, film_scratch: dict | None = None,
                        gate_dust: dict | None = None, gate_scratch: dict | None = None, origins=(), flags: int = 0,
                        sample_step_mm=(0.0, 0.0), roi_offset=(0, 0), gate_size=(0, 0), session_seed: int = 0,
                        clip_token: int = 0, weave=(0.0, 0.0, 1.0, 0.0), extent=(0, 0, 0, 0),
                        recipe_hash: int = 1, hash: int = 1) -> "abi.FjFilmEffects":
    """An FjFilmEffects record (film / gate dust and scratches, weave) from field values:
    the family dicts map FjDust / FjScratch field names to floats; origins are up to four
    (cell_x, cell_y, local_x_mm, local_y_mm); weave is (dx_px, dy_px, cos, sin)."""
    e = abi.FjFilmEffects()
    for name, values in (("film_dust", film_dust), ("film_scratch", film_scratch), ("gate_dust", gate_dust),
                         ("gate_scratch", gate_scratch)):
        rec = getattr(e, name)
        for k, v in (values or {}).items():
            setattr(rec, k, float(v))
    for i, o in enumerate(origins):
        e.origins[i].cell_x, e.origins[i].cell_y, e.origins[i].local_x_mm, e.origins[i].local_y_mm = o
    for ext in (e.render_extent, e.full_frame_extent):
        ext.x, ext.y, ext.width, ext.height = extent
    e.sample_step_x_mm, e.sample_step_y_mm = sample_step_mm
    e.roi_offset_x, e.roi_offset_y = roi_offset
    e.gate_width, e.gate_height = gate_size
    e.session_seed, e.clip_token = session_seed, clip_token
    e.weave_dx_px, e.weave_dy_px, e.weave_cos_rot, e.weave_sin_rot = weave
    e.flags = flags
    e.recipe_hash, e.hash = (recipe_hash, hash) if flags & (abi.FJ_EFFECTS_FILM | abi.FJ_EFFECTS_GATE_OUTPUT) else (0, 0)
    return e


# Film dust and scratch families of the reference's effects-frame characterization
# (tests/film/effects-frame-fixtures/inputs.json, case 0), slot probabilities aside.
DUST_FAMILY = dict(
    cell_width_mm=0.5, cell_height_mm=0.5, softness_min_mm=0.00025, softness_max_mm=0.003,
    softness_size_cap_fraction=0.25, support_x_mm=0.415, support_y_mm=0.415, fiber_fraction=0.25,
    fiber_drift_fraction=0.1, fiber_first_knot_min=0.08, fiber_first_knot_max=0.35, fiber_second_knot_min=0.65,
    fiber_second_knot_max=0.92, fiber_interior_width_min_fraction=0.45, fiber_interior_width_max_fraction=1.0,
    diameter_min_mm=0.008, diameter_bulk_max_mm=0.08, diameter_max_mm=0.25, diameter_tail_fraction=0.2,
    fiber_length_min_mm=0.04, fiber_length_max_mm=0.65, fiber_width_min_mm=0.003, fiber_width_max_mm=0.025,
    opacity_faint_cumulative=0.5, opacity_intermediate_cumulative=0.85, compact_opacity_min=0.1,
    compact_opacity_faint_end=0.45, compact_opacity_intermediate_end=0.85, compact_opacity_max=0.99,
    fiber_opacity_min=0.08, fiber_opacity_faint_end=0.35, fiber_opacity_intermediate_end=0.75,
    fiber_opacity_max=0.97, compact_dominant_aspect_min=0.52, compact_dominant_aspect_max=0.95,
    compact_subsidiary_scale_min=0.3, compact_subsidiary_scale_max=0.75, compact_subsidiary_aspect_min=0.45,
    compact_subsidiary_aspect_max=1.0, compact_subsidiary_offset_max=0.68,
    compact_subsidiary_angle_max_radians=3.1415927)
SCRATCH_FAMILY = dict(
    cell_width_mm=1.0, cell_height_mm=8.0, softness_min_mm=0.00015, softness_max_mm=0.0015,
    softness_size_cap_fraction=0.25, support_x_mm=0.68, support_y_mm=12.08, length_min_mm=0.25,
    length_bulk_max_mm=6.0, length_max_mm=24.0, length_tail_fraction=0.16, width_min_mm=0.002,
    width_bulk_max_mm=0.025, width_max_mm=0.08, width_tail_fraction=0.18, drift_fraction=0.025,
    first_knot_min=0.06, first_knot_max=0.28, second_knot_min=0.72, second_knot_max=0.94,
    interior_width_min_fraction=0.35, interior_width_max_fraction=1.0, interior_depth_min_fraction=0.35,
    interior_depth_max_fraction=1.0, endpoint_abrupt_probability=0.3, interruption_probability=0.15,
    gap_center_min=0.25, gap_center_max=0.75, gap_span_min=0.02, gap_span_max=0.12, scuff_probability=0.1,
    scuff_length_max_mm=0.75, scuff_angle_max_radians=0.61086524, strength_min=0.1425, strength_max=0.95)


def default_film_effects(width: int, height: int, *, frame_width_mm: float = 36.0,
                         slots=(0.02, 0.05, 0.01, 0.02), weave=(-0.35, 0.22, 0.99995, 0.01),
                         session_seed: int = 0x0123456789ABCDEF, clip_token: int = 0x0FEDCBA987654321):
    """Film dust and scratches, gate dust and scratches (gate grid at half resolution) and
    gate weave for a full frame of width x height pixels; `slots` are the slot
    probabilities of film dust, film scratch, gate dust, gate scratch."""
    step = frame_width_mm / width
    fams = [dict(DUST_FAMILY, slot_probability=slots[0]), dict(SCRATCH_FAMILY, slot_probability=slots[1]),
            dict(DUST_FAMILY, slot_probability=slots[2]), dict(SCRATCH_FAMILY, slot_probability=slots[3])]
    flags = (abi.FJ_EFFECTS_FILM | abi.FJ_EFFECTS_GATE_TRANSMITTANCE | abi.FJ_EFFECTS_GATE_OUTPUT
             | abi.FJ_EFFECTS_WEAVE | abi.FJ_EFFECTS_FULL_FRAME)
    return film_effects_record(film_dust=fams[0], film_scratch=fams[1], gate_dust=fams[2], gate_scratch=fams[3],
                               origins=[(0, 67, 0.0, 0.25), (0, 4, 0.0, 1.75), (0, 0, 0.0, 0.0), (0, 0, 0.0, 0.0)],
                               flags=flags, sample_step_mm=(step, step), gate_size=((width + 1) // 2, (height + 1) // 2),
                               session_seed=session_seed, clip_token=clip_token, weave=weave,
                               extent=(0, 0, width, height), recipe_hash=0x5EED, hash=0xEFFEC7)
