"""The oracle's whole-frame chain for the staged schedule (test infrastructure only):
camera exposure -> highlight reconstruction -> camera diffusion -> scatter/halation -> spatial DIR -> capture
density -> grain -> film defects -> (enlarger: print-linear exposure, enlarger diffusion, print development)
-> print/scan/output, each stage the CPU restatement in oracle/."""
from __future__ import annotations

import contextlib

import numpy as np

from . import dir as odir
from . import grain as ograin
from . import optics as ooptics
from . import oracle as orc


class _Components:
    def __init__(self, lam, w):
        self.lambda_px, self.red_weights, self.green_weights, self.blue_weights = lam, w[0], w[1], w[2]


def render_frame(frame_record, recipe, src, threads: int = 1, frame_token: int = 0, diffusion_form: str = "direct",
                 stages: dict | None = None):
    """frame_record: film_juicer_b200.frame_records.FrameRecord; recipe: the
    PreparedRecipe it was built from; src: (H, W, comps) float32. Returns the encoded
    output (H, W, comps) and the error flags. `threads` parallelises the per-pixel
    stages and the FFT (the line stages use the oracle's OpenMP default).
    diffusion_form: "direct" (FP64 direct sum, the parity form) or "fft" (the
    reference's FFT convolution in FP64, same results after float rounding; the CPU
    baseline's form). stages: when a dict, it receives a copy of each stage's planes
    (camera_exposure, camera_diffusion, scatter_halation: B, G, R carrier;
    spatial_dir_filtered: Y, M, C; capture_density, grain: C, M, Y density)."""

    def keep(name, planes):
        if stages is not None:
            stages[name] = [np.array(q, dtype=np.float32, copy=True) for q in planes]

    abi = orc._abi()
    host = frame_record.host
    h = host.h
    scale = 1.0
    if h.film_exposure.flags & abi.FJ_FILM_AUTO_EXPOSURE:
        scale = orc.auto_exposure(host, h.auto_exposure, src)
    carrier, _ = orc.render(host, src, stage=3, auto_scale=scale, threads=threads)  # B, G, R
    keep("camera_exposure", carrier)
    flags = h.optics.flags
    if flags & abi.FJ_OPTICS_HIGHLIGHT_BOOST:
        carrier, disp = ooptics.highlight_boost(h.optics.highlight_boost, carrier)
        if disp not in (0, 1):
            raise RuntimeError(f"highlight boost disposition {disp}")
    if flags & abi.FJ_OPTICS_CAMERA_DIFFUSION:
        d = h.optics.camera
        lam, w = ooptics.diffusion_components(d.family, list(d.group_weights), list(d.group_lambda_um), d.warmth,
                                              d.spatial_scale, d.pixel_size_um)
        planes = [carrier[2], carrier[1], carrier[0]]
        if diffusion_form == "fft":
            r, g, b = ooptics.diffusion_fft(_Components(lam, w), d.radius_px, d.scatter_fraction, planes,
                                            workers=threads)
        else:
            r, g, b = ooptics.diffusion(_Components(lam, w), d.radius_px, d.scatter_fraction, planes)
        carrier = [b, g, r]
        keep("camera_diffusion", carrier)
    if flags & abi.FJ_OPTICS_SCATTER_HALATION:
        r, g, b = ooptics.scatter_halation(h.optics.scatter_halation, [carrier[2], carrier[1], carrier[0]])
        carrier = [b, g, r]
        keep("scatter_halation", carrier)
    if h.spatial_dir.component_count > 0:
        filtered, log_raw, _ = odir.spatial_dir(host, h.spatial_dir, carrier=carrier, width=src.shape[1],
                                               height=src.shape[0])
        keep("spatial_dir_filtered", filtered)
        density, _ = odir.develop_spatial(host, filtered, log_raw)
    else:
        density, _ = orc.render(host, None, stage=5, planes=carrier, threads=threads)
    keep("capture_density", density)
    if h.grain.flags & abi.FJ_GRAIN_ACTIVE:
        a = recipe.arrays
        layers = [[a["density_layers"][:, l, c] for c in range(3)] for l in range(3)]
        base = [a["density_rgb"][:, c] for c in range(3)]
        noise = frame_record.noise.record if frame_record.noise is not None else None
        density = ograin.visual_grain(h.grain, noise, base, layers, h.capture_polarity == 1, density)
        keep("grain", density)
    fx = h.effects
    film = bool(fx.flags & abi.FJ_EFFECTS_FILM)
    gate_output = bool(fx.flags & abi.FJ_EFFECTS_GATE_OUTPUT)
    dust = mask = None
    if film:
        # film dust / scratches on the developed capture density, after grain
        density, dust = orc.film_defects(fx, density)
    if gate_output and (fx.flags & abi.FJ_EFFECTS_GATE_TRANSMITTANCE):
        mask = orc.gate_mask(fx)
    enlarger = bool(flags & abi.FJ_OPTICS_ENLARGER_DIFFUSION)
    if enlarger:
        # print-linear exposure (film dust applied here), the enlarger's diffusion, print
        # development; the scan then reads print density
        lin = ooptics.enlarger_linear(host, density, dust)
        d = h.optics.enlarger
        lam, w = ooptics.diffusion_components(d.family, list(d.group_weights), list(d.group_lambda_um), d.warmth,
                                              d.spatial_scale, d.pixel_size_um)
        if diffusion_form == "fft":
            lin = ooptics.diffusion_fft(_Components(lam, w), d.radius_px, d.scatter_fraction, lin, workers=threads)
        else:
            lin = ooptics.diffusion(_Components(lam, w), d.radius_px, d.scatter_fraction, lin)
        density = ooptics.enlarger_develop(host, lin)
        dust = None
    with (ooptics.print_done() if enlarger else contextlib.nullcontext()):
        return _scan(host, h, fx, film, gate_output, dust, mask, density, src, threads, frame_token, abi)


def _scan(host, h, fx, film, gate_output, dust, mask, density, src, threads, frame_token, abi):
    """Print (unless the enlarger already developed it) / scan / output of the density planes."""
    if h.scanner_post.hash != 0 or film or gate_output:
        # linear planes before the encoding; the source origin of these frames is (0, 0)
        seed = orc.glare_seed(h.recipe_hash, frame_token, 0, 0)
        return orc.render_effects(host, h.scanner_post, seed, 0, 0, fx if (film or gate_output) else None, dust,
                                  mask, density, src=src, threads=threads)
    return orc.render(host, src, stage=2, planes=density, threads=threads)
