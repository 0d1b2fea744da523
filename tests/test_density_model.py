"""The test recipes' density curves come from each profile's Gaussian-CDF model, as the
reference's host evaluates them (rust/film-juicer-core/src/profile.rs:482-520):
prepare.density_model_samples against the reference's frozen characterization
(tests/profile/fixtures/density.json + density-samples.bin of the reference, in
tests/golden/density_model_cases.npz): every valid sample (totals and layers) of all
122 cases with samples, the shipped models over their authored axes included.

The reference takes erfcf from the Rust libm crate (=0.2.15); the restatement rounds an
FP64 erfc to f32, so words may differ in the last bits: the bound is 4 ulp per value,
and at least 85 % of the values are bit-identical. Runs on the CPU."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
Z = np.load(os.path.join(GOLDEN, "density_model_cases.npz"))
NAMES = [str(n) for n in Z["names"]]


def _case(name):
    m = Z[f"{name}__model"].view(np.float64)
    return m[0], m[1], m[2], bool(Z[f"{name}__positive"][0]), Z[f"{name}__axis"].view(np.float64), \
        Z[f"{name}__records"]


def test_density_model_matches_reference_samples(prepare):
    total = exact = 0
    worst = 0
    for name in NAMES:
        centers, amplitudes, sigmas, positive, axis, records = _case(name)
        tot, lay = prepare.density_model_samples(centers, amplitudes, sigmas, axis, positive)
        for i in range(axis.size):
            if records[i, 0] != 1:
                continue
            want = records[i, 1:].view("<u4")
            got = np.concatenate([tot[i], lay[i].ravel()]).view(np.uint32)
            d = np.abs(got.astype(np.int64) - want.astype(np.int64))
            total += 12
            exact += int((d == 0).sum())
            worst = max(worst, int(d.max()))
    assert total >= 12 * 19000
    assert worst <= 4, worst
    assert exact >= 0.85 * total, exact / total


def test_recipe_curves_are_the_model(recipes, prepare):
    """The committed print recipe's film curves equal the model on the recipe's axis."""
    a = recipes["print"].arrays
    assert a["density_rgb"].shape[1] == 3 and a["density_layers"].shape[1:] == (3, 3)
    np.testing.assert_allclose(a["density_layers"].sum(axis=1), a["density_rgb"], rtol=1e-5, atol=1e-6)
    assert float(a["density_rgb"].min()) >= 0.0
