"""Whole-frame FjPreparedHostData for the full optical print schedule.

Builds the record a host hands to fj_cuda_render for a frame with every spatial stage
of the path switched on: camera diffusion (radius 0.5 % of the width), emulsion
scatter and halation, the spatial DIR tail (200 um, weight 0.03), density-space grain
(35 mm format, fixed seeds) and optionally camera auto exposure. Pixel size follows
a 35 mm wide film gate (35000 um / width). The stage descriptors come from
descriptors.py, prepare.py and grain_plan.py; the noise is seeded synthetic bytes in
the production shapes unless a Noise is given.
"""
from __future__ import annotations

from . import abi, descriptors, grain_plan, prepare


class FrameRecord:
    """A HostRecord plus the objects its spans point into."""

    def __init__(self, recipe: "prepare.PreparedRecipe", width: int, height: int, *, recipe_hash: int = 0x5EED,
                 diffusion: bool = True, halation: bool = True, spatial_dir: bool = True, grain: bool = True,
                 auto_exposure: bool = False, noise: "grain_plan.Noise | None" = None,
                 pixel_size_um: float | None = None, frame_time: float = 0.0, descriptor_width: int | None = None,
                 post=None, highlight_boost=None, effects=None, enlarger: bool = False):
        """descriptor_width: the frame width the pixel size and diffusion radius are
        derived for (defaults to `width`; a crop of a larger frame passes the full width);
        post: an FjScannerPostEffects record (descriptors.scanner_post_record);
        highlight_boost: an FjHighlightBoost record (descriptors.highlight_boost_record);
        effects: an FjFilmEffects record (film / gate defects, weave);
        enlarger: enlarger diffusion (print routes; a warm family-0 filter of radius
        0.3 % of the width on the print-linear exposure)."""
        self.width, self.height = width, height
        dw = descriptor_width or width
        self.pixel_size_um = pixel_size_um or 35000.0 / dw
        self.host = prepare.HostRecord(recipe, recipe_hash=recipe_hash, auto_exposure=auto_exposure)
        h = self.host.h
        px = self.pixel_size_um
        if auto_exposure:
            from .runtime import meter_record

            h.auto_exposure = meter_record(width, height)
        flags = 0
        h.optics.full_frame.x, h.optics.full_frame.y = 0, 0
        h.optics.full_frame.width, h.optics.full_frame.height = width, height
        if diffusion:
            h.optics.camera = descriptors.diffusion_record(px, dw)
            flags |= abi.FJ_OPTICS_CAMERA_DIFFUSION
        if halation:
            h.optics.scatter_halation = prepare.scatter_halation_record(px)
            flags |= abi.FJ_OPTICS_SCATTER_HALATION
        if enlarger:
            h.optics.enlarger = descriptors.diffusion_record(px, dw, family=0, scatter_fraction=0.2, warmth=0.5,
                                                             radius_fraction_of_width=0.003)
            flags |= abi.FJ_OPTICS_ENLARGER_DIFFUSION
        if highlight_boost is not None:
            h.optics.highlight_boost = highlight_boost
            flags |= abi.FJ_OPTICS_HIGHLIGHT_BOOST
        h.optics.flags = flags
        if spatial_dir:
            h.spatial_dir = descriptors.spatial_dir_record(px, width, height)
        if post is not None:
            h.scanner_post = post
        if effects is not None:
            h.effects = effects
        self.noise = None
        if grain:
            a = recipe.arrays
            layers = [[a["density_layers"][:, l, c] for c in range(3)] for l in range(3)]
            inp = grain_plan.GrainInput(render_extent=(0, 0, width, height), full_frame_extent=(0, 0, width, height),
                                        pixel_size_um=px, frame_time=frame_time, layer_curves=layers)
            plan = grain_plan.plan(inp)
            h.grain = grain_plan.visual_grain_record(inp, plan, grain_plan.GrainCoefficients(),
                                                     curves_cmy=a["density_rgb"])
            self.noise = noise if noise is not None else grain_plan.synthetic_noise()
            h.noise = self.noise.record

    def pointer(self):
        return self.host.pointer()
