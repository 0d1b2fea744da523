"""Visual grain (a15) on the GPU through fjb_visual_grain.

Against the reference's own CUDA grain (compiled from its sources into the test
harness): identical float32 values, case by case -- the random streams, Poisson
counts, blurs and mixes are the same arithmetic in the same order.

Against the CPU oracle: libm's expf/logf/cosf differ from CUDA's in the last bits,
which can move a Poisson count by one at a threshold and shifts modulated values by
an ulp; the bound is on the share of pixels that differ by more than 1e-4 (at most
0.5 %) and on the median difference (at most 1e-6).
"""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def density_planes(w, h, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    planes = []
    for c in range(3):
        base = 0.15 + 1.6 * (0.5 + 0.5 * np.sin(xx / (7.0 + c) + yy / 11.0 + c))
        planes.append(np.ascontiguousarray((base + rng.normal(0, 0.05, size=(h, w))).astype(np.float32)))
    planes[0][0, 0] = -0.02  # below zero: clamped by the particle model
    return planes


def small_noise(seed, pow2=True):
    from film_juicer_b200 import grain_plan as gp

    rng = np.random.default_rng(seed)
    shape = (16, 64, 64) if pow2 else (7, 48, 40)
    return gp.Noise(rng.integers(0, 256, size=shape, dtype=np.uint8),
                    rng.integers(0, 256, size=(16, 32, 32), dtype=np.uint8), gp.wang_lut_two_colors())


def make_case(recipe, name, w, h):
    from film_juicer_b200 import grain_plan as gp

    a = recipe.arrays
    layers = [[a["density_layers"][:, l, c] for c in range(3)] for l in range(3)]
    inp = gp.GrainInput(render_extent=(0, 0, w, h), full_frame_extent=(0, 0, w, h), pixel_size_um=2.0,
                        layer_curves=layers, frame_time=3.0)
    coeff = gp.GrainCoefficients()
    positive = False
    noise_pow2 = True
    use_noise = True
    tweak = None
    if name == "simple":
        inp.sublayers_active = False
        inp.sublayer_count = 3
        inp.correlation_sigma_px = 0.9
    elif name == "simple_retime":
        inp.sublayers_active = False
        inp.sublayer_count = 2
        inp.frame_time = 10.375
    elif name == "mixed_scales":
        inp.size_mix_scale = 4.0
        inp.fine_weight, inp.mid_weight, inp.coarse_weight = 0.5, 0.3, 0.2
        coeff.chroma_mix, coeff.chroma_shared_weight, coeff.chroma_independent_weight = 0.5, 0.6, 0.8
    elif name == "independent":
        coeff.chroma_mix = 1.0
        coeff.amplitude = 0.8
    elif name == "dye_zero":
        inp.dye_cloud_blur_um = 0.0
    elif name == "dye_shared":
        tweak = "dye_shared"
    elif name == "dye_partial":
        tweak = "dye_partial"
    elif name == "clump_temporal":
        coeff.clump_temporal_mix = 0.6
        inp.frame_time = 37.6
    elif name == "philox":
        use_noise = False
    elif name == "stbn_odd":
        noise_pow2 = False
    elif name == "positive":
        positive = True
    elif name.startswith("debug"):
        coeff.debug_view = int(name[5:])
        inp.size_mix_scale = 3.0
        inp.fine_weight, inp.mid_weight, inp.coarse_weight = 0.6, 0.2, 0.2
    elif name == "offset_origin":
        inp.render_extent = (37, 21, w, h)
        inp.full_frame_extent = (0, 0, w + 100, h + 80)
        inp.correlation_sigma_px = 0.0
        inp.dye_cloud_blur_um = 0.0
    p = gp.plan(inp)
    rec = gp.visual_grain_record(inp, p, coeff, curves_cmy=a["density_rgb"])
    if tweak == "dye_shared":
        for l in range(3):
            for c in range(3):
                rec.dye_cloud[l][c] = copy.copy(rec.dye_cloud[0][c])
    elif tweak == "dye_partial":
        for c in range(3):
            rec.dye_cloud[2][c].radius = 0
            rec.dye_cloud[2][c].sigma_px = 0.0
            rec.dye_cloud[2][c].hash = 0
    base = [a["density_rgb"][:, c] for c in range(3)]
    noise = small_noise(5, noise_pow2) if use_noise else None
    return rec, noise, base, layers, positive


CASES = ["default", "simple", "simple_retime", "mixed_scales", "independent", "dye_zero", "dye_shared",
         "dye_partial", "clump_temporal", "philox", "stbn_odd", "positive", "offset_origin", "debug1", "debug2",
         "debug3", "debug4", "debug5", "debug6"]


def run_library(torch, recipes, name, w, h, seed):
    from film_juicer_b200 import prepare, runtime

    recipe = recipes["print"]
    rec, noise, base, layers, positive = make_case(recipe, name, w, h)
    host = prepare.HostRecord(recipe)
    if positive:
        host.h.capture_polarity = 1
    dev_recipe = runtime.DeviceRecipe(host)
    planes = density_planes(w, h, seed)
    dev = [torch.from_numpy(p).cuda() for p in planes]
    dnoise = runtime.DeviceNoise(noise.record) if noise is not None else None
    runtime.visual_grain(dev_recipe, rec, dev, dnoise)
    torch.cuda.synchronize()
    got = [t.cpu().numpy() for t in dev]
    return got, (rec, noise, base, layers, positive, planes)


@pytest.mark.parametrize("name", CASES)
def test_grain_matches_reference_cuda(torch_cuda, recipes, oracle, name):
    from oracle import grain as og

    w, h = 61, 45
    got, (rec, noise, base, layers, positive, planes) = run_library(torch_cuda, recipes, name, w, h, 3)
    ref = og.reference_visual_grain(torch_cuda, rec, noise.record if noise is not None else None, base, layers,
                                    positive, planes)
    if ref is None:
        pytest.skip("reference CUDA harness not built")
    for c in range(3):
        assert np.all(np.isfinite(got[c]))
        diff = got[c] != ref[c]
        assert not diff.any(), (name, c, int(diff.sum()), float(np.abs(got[c] - ref[c]).max()))


@pytest.mark.parametrize("name", CASES)
def test_grain_matches_oracle(torch_cuda, recipes, oracle, name):
    from oracle import grain as og

    w, h = 61, 45
    got, (rec, noise, base, layers, positive, planes) = run_library(torch_cuda, recipes, name, w, h, 4)
    want = og.visual_grain(rec, noise.record if noise is not None else None, base, layers, positive, planes)
    for c in range(3):
        d = np.abs(got[c] - want[c])
        assert float(np.mean(d > 1e-4)) <= 0.005, (name, c, float(np.mean(d > 1e-4)), float(d.max()))
        assert float(np.median(d)) <= 1e-6, (name, c, float(np.median(d)))


def test_grain_changes_density_and_is_deterministic(torch_cuda, recipes):
    got1, ctx = run_library(torch_cuda, recipes, "default", 80, 50, 9)
    got2, _ = run_library(torch_cuda, recipes, "default", 80, 50, 9)
    planes = ctx[5]
    for c in range(3):
        np.testing.assert_array_equal(got1[c], got2[c])
        assert float(np.std(got1[c] - planes[c])) > 1e-3


def test_grain_rejects_bad_records(torch_cuda, recipes):
    from film_juicer_b200 import prepare, runtime

    rec, noise, *_ = make_case(recipes["print"], "default", 16, 16)
    dev_recipe = runtime.DeviceRecipe(prepare.HostRecord(recipes["print"]))
    planes = [torch_cuda.zeros((16, 16), device="cuda") for _ in range(3)]
    bad = copy.copy(rec)
    bad.size_mix_weights[0] = 0.5  # weights no longer sum to one
    with pytest.raises(runtime.FjError, match="size mix"):
        runtime.visual_grain(dev_recipe, bad, planes)
    bad = copy.copy(rec)
    bad.correlation[0].radius = 76
    with pytest.raises(runtime.FjError, match="radius"):
        runtime.visual_grain(dev_recipe, bad, planes)
