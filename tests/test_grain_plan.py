"""Grain frame plan (host, no GPU) against the reference's visual-grain frame
characterization (tests/grain/frame-fixtures of the reference): every successful
case's published fields as exact float32/int/u64 words, and the Gaussian, energy and
period primitives. Also the Wang tile table against the resource's tiles.json."""
import json
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN
from film_juicer_b200 import grain_plan as gp


def f32(bits):
    return struct.unpack("<f", struct.pack("<I", bits))[0]


def f64(bits):
    return struct.unpack("<d", struct.pack("<Q", bits))[0]


def bits32(v):
    return gp.f32_bits(v)


def load():
    with open(os.path.join(GOLDEN, "grain_plan_cases.json")) as fh:
        return json.load(fh)


def grain_input(i):
    curves = [[np.array([f32(b) for b in ch], np.float32) for ch in layer] for layer in i["layer_curves"]]
    return gp.GrainInput(
        render_extent=tuple(i["render_extent"]), full_frame_extent=tuple(i["full_frame_extent"]),
        pixel_size_um=f32(i["pixel_size_um"]), frame_time=f64(i["frame_time"]), frame_rate=f64(i["frame_rate"]),
        session_seed=i["session_seed"], clip_token=i["clip_token"], recipe_hash=i["recipe_hash"],
        positive=i["capture_polarity"] == 1,
        authored_max_cmy=tuple(f32(b) for b in i["authored_max_cmy"]),
        particle_area_um2=f32(i["particle_area_um2"]),
        particle_scale_cmy=tuple(f32(b) for b in i["particle_scale_cmy"]),
        particle_scale_layers=tuple(f32(b) for b in i["particle_scale_layers"]),
        particle_density_min_cmy=tuple(f32(b) for b in i["particle_density_min_cmy"]),
        correlation_sigma_px=f32(i["correlation_sigma_px"]), dye_cloud_blur_um=f32(i["dye_cloud_blur_um"]),
        sublayers_active=i["sublayers_active"], sublayer_count=i["sublayer_count"],
        size_mix_scale=f32(i["size_mix_scale"]), fine_weight=f32(i["fine_weight"]), mid_weight=f32(i["mid_weight"]),
        coarse_weight=f32(i["coarse_weight"]), clump_morph_period_sec=f32(i["clump_morph_period_sec"]),
        layer_curves=curves, layers_hash=i["film_layers_hash"])


def gauss_words(g):
    return [bits32(g.sigma_px), g.radius, g.hash]


def test_plan_matches_reference_cases():
    data = load()
    assert len(data["cases"]) == 89
    for case in data["cases"]:
        i, e = case["input"], case["expected"]
        p = gp.plan(grain_input(i))
        name = i["name"]
        got = {
            "frame0": p.frame0, "frame_alpha": bits32(p.frame_alpha), "seed_base": p.seed_base,
            "seed_base_next": p.seed_base_next, "pitch_px": p.pitch_px,
            "breathing_period_frames": p.breathing_period_frames,
            "clump_morph_period_frames": p.clump_morph_period_frames, "wang_cell_mm": bits32(p.wang_cell_mm),
            "breathing_amplitude": bits32(p.breathing_amplitude),
            "breathing_cell_um_small": bits32(p.breathing_cell_um_small),
            "breathing_cell_um_large": bits32(p.breathing_cell_um_large), "breathing_mix": bits32(p.breathing_mix),
            "breathing_drift_um_per_frame": bits32(p.breathing_drift_um_per_frame),
            "debug_scale": bits32(p.debug_scale),
            "density_max_cmy": [bits32(v) for v in p.density_max_cmy],
            "n_particles_cmy": [bits32(v) for v in p.n_particles_cmy],
            "od_particle_cmy": [bits32(v) for v in p.od_particle_cmy],
            "density_min_layers": [[bits32(v) for v in row] for row in p.density_min_layers],
            "density_max_layers": [[bits32(v) for v in row] for row in p.density_max_layers],
            "n_particles_layers": [[bits32(v) for v in row] for row in p.n_particles_layers],
            "od_particle_layers": [[bits32(v) for v in row] for row in p.od_particle_layers],
            "correlation": [gauss_words(g) for g in p.correlation],
            "dye_cloud": [[gauss_words(g) for g in row] for row in p.dye_cloud],
            "size_mix_weights": [bits32(v) for v in p.size_mix_weights],
            "size_mix_gain": bits32(p.size_mix_gain), "requires_full_frame": p.requires_full_frame,
            "density_layers_hash": p.density_layers_hash,
        }
        for k, v in e.items():
            assert got[k] == v, (name, k, got[k], v)


def test_primitives():
    for prim in load()["primitives"]:
        op, arg, want = prim["input"]["op"], prim["input"]["input"], prim["result"]
        if op == "gaussian":
            assert gauss_words(gp.Gaussian.new(f32(arg))) == want, prim
        elif op == "energy":
            assert bits32(gp._energy(f32(arg))) == want, prim
        elif op == "period":
            try:
                got = gp._period_rounded(f64(arg))
            except gp.PlanError:
                got = None
            assert got == want or (got is None and want is None), prim


def test_wang_lut_matches_tile_set():
    with open(os.path.join(GOLDEN, "wang_lut.json")) as fh:
        want = json.load(fh)
    assert list(int(v) for v in gp.wang_lut_two_colors()) == want
