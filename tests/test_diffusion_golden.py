"""Diffusion (a17) oracle pinned on the reference's external diffusion cohort
(tests/diffusion/fixtures/diffusion_reference_v1 of the reference: 72 RGB images of
17x19 .. 23x11, radius 6, four filter families, camera and enlarger stages, HDR
inputs). No GPU. The oracle convolves directly in FP64 with the float PSF; the
cohort came from an FFT convolution, whose round-off scales with the largest value
of the frame, so the bound is one float32 rounding step of that magnitude:
|d| <= 1.5e-7 max(1, max |input|)."""
import os

import numpy as np

from conftest import GOLDEN
from oracle import optics


class Components:
    def __init__(self, lam, w):
        self.lambda_px, self.red_weights, self.green_weights, self.blue_weights = lam, w[0], w[1], w[2]


def cases():
    z = np.load(os.path.join(GOLDEN, "diffusion_images.npz"))
    for i, name in enumerate(z["names"]):
        p = z["params"][i]
        lam, w = optics.diffusion_components(int(z["family"][i]), p[0:3], p[3:6], p[6], p[7], p[8])
        yield (str(name), Components(lam, w), int(z["radius"][i]), float(p[9]),
               z[f"input_{int(z['input_index'][i])}"], z[f"output_{i}"])


def test_oracle_matches_external_cohort():
    n = 0
    for name, comps, radius, fraction, x, want in cases():
        got = np.stack(optics.diffusion(comps, radius, fraction, [x[..., c] for c in range(3)]), -1)
        err = np.abs(got - want)
        assert np.all(err <= 1.5e-7 * max(1.0, float(np.abs(x).max()))), (name, float(err.max()))
        n += 1
    assert n == 72


def test_fft_form_matches_external_cohort_and_direct_form():
    """The oracle's FFT form (the CPU baseline's diffusion) on the same cohort: same
    bound against the reference's outputs, and within one float32 rounding of the
    direct FP64 sum (both convolve the same float PSF in FP64)."""
    n = 0
    for name, comps, radius, fraction, x, want in cases():
        planes = [x[..., c] for c in range(3)]
        got = np.stack(optics.diffusion_fft(comps, radius, fraction, planes), -1)
        direct = np.stack(optics.diffusion(comps, radius, fraction, planes), -1)
        scale = max(1.0, float(np.abs(x).max()))
        assert np.all(np.abs(got - want) <= 1.5e-7 * scale), (name, float(np.abs(got - want).max()))
        assert np.all(np.abs(got - direct) <= 1.2e-7 * np.maximum(1.0, np.abs(direct))), name
        n += 1
    assert n == 72
