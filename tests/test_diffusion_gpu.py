"""Diffusion (a17) on the GPU through fjb_diffusion, against the reference's external
diffusion cohort and the CPU oracle.

Radii below 8 convolve directly with FP32 accumulation (the PSF rows folded by
vertical symmetry); larger radii go through the FP32 FFT convolution; the oracle
accumulates the direct sum in FP64. Bound: |d| <= 2e-6 max(1,
max |input|) -- a few float32 roundings of a sum whose weights add to one."""
import numpy as np
import pytest

from test_diffusion_golden import cases

pytestmark = pytest.mark.gpu
TOL = 2e-6


def run(torch, comps_abi, radius, fraction, planes, stride=None):
    from film_juicer_b200 import runtime

    h, w = planes[0].shape
    stride = stride or w
    src = []
    for p in planes:
        t = torch.zeros((h, stride), dtype=torch.float32, device="cuda")
        t[:, :w] = torch.from_numpy(np.ascontiguousarray(p))
        src.append(t)
    dst = [torch.full_like(t, -7.0) for t in src]
    runtime.diffusion(comps_abi, radius, fraction, [t[:, :w] for t in src], [t[:, :w] for t in dst])
    torch.cuda.synchronize()
    out = [t.cpu().numpy() for t in dst]
    for o in out:  # the padding columns stay untouched
        assert np.all(o[:, w:] == -7.0)
    return [o[:, :w] for o in out]


def to_abi(comps):
    from film_juicer_b200 import abi

    c = abi.FjDiffusionComponents()
    for i in range(9):
        c.lambda_px[i] = comps.lambda_px[i]
        c.red_weights[i] = comps.red_weights[i]
        c.green_weights[i] = comps.green_weights[i]
        c.blue_weights[i] = comps.blue_weights[i]
    return c


def test_matches_external_cohort(torch_cuda):
    for name, comps, radius, fraction, x, want in cases():
        got = np.stack(run(torch_cuda, to_abi(comps), radius, fraction, [x[..., c] for c in range(3)]), -1)
        err = np.abs(got - want)
        assert np.all(err <= TOL * max(1.0, float(np.abs(x).max()))), (name, float(err.max()))


SHAPES = {
    # name: (width, height, radius, stride)
    "r10": (150, 70, 10, None),
    "r20_strided": (131, 45, 20, 160),
    "r40": (97, 83, 40, None),
    "r80_max": (170, 90, 80, None),
    "tiny": (7, 5, 3, None),
    "one_row": (64, 1, 4, None),
    "one_col": (1, 40, 4, None),
    "radius_beyond_frame": (9, 6, 12, None),
    # FFT form (radius >= 8): odd log2 transform lengths (128 x 128), and a larger frame
    "fft_odd_lengths": (200, 100, 9, 224),
    "fft_frame": (640, 360, 16, None),
}


@pytest.mark.parametrize("name", list(SHAPES))
def test_matches_oracle(torch_cuda, name):
    from film_juicer_b200 import descriptors, runtime
    from oracle import optics

    w, h, radius, stride = SHAPES[name]
    d = descriptors.diffusion_record(4.0, 4 * w, family=1, warmth=0.8)
    comps = runtime.diffusion_components(d)
    rng = np.random.default_rng(radius * 1000 + w)
    planes = [rng.uniform(0.0, 1.5, size=(h, w)).astype(np.float32) for _ in range(3)]
    planes[0][h // 2, w // 2] += 40.0
    got = run(torch_cuda, comps, radius, 0.3, planes, stride)
    want = optics.diffusion(comps, radius, 0.3, planes)
    for g, r, p in zip(got, want, planes):
        err = np.abs(g - r)
        assert np.all(err <= TOL * max(1.0, float(np.abs(p).max()))), float(err.max())


def test_constant_plane_and_zero_fraction(torch_cuda):
    from film_juicer_b200 import descriptors, runtime

    d = descriptors.diffusion_record(3.0, 3840)
    comps = runtime.diffusion_components(d)
    flat = [np.full((33, 70), v, dtype=np.float32) for v in (0.25, 1.0, 3.0)]
    for g, p in zip(run(torch_cuda, comps, 20, 0.5, flat), flat):
        np.testing.assert_allclose(g, p, rtol=2e-6)
    rng = np.random.default_rng(5)
    planes = [rng.uniform(0, 1, size=(20, 30)).astype(np.float32) for _ in range(3)]
    for g, p in zip(run(torch_cuda, comps, 5, 0.0, planes), planes):
        np.testing.assert_array_equal(g, p)


def test_rejects_bad_arguments(torch_cuda):
    from film_juicer_b200 import descriptors, runtime

    torch = torch_cuda
    comps = runtime.diffusion_components(descriptors.diffusion_record(3.0, 3840))
    a = [torch.zeros((8, 8), device="cuda") for _ in range(3)]
    b = [torch.zeros((8, 8), device="cuda") for _ in range(3)]
    with pytest.raises(runtime.FjError, match="alias"):
        runtime.diffusion(comps, 2, 0.5, a, a)
    with pytest.raises(runtime.FjError, match="radius"):
        runtime.diffusion(comps, 81, 0.5, a, b)
    with pytest.raises(runtime.FjError, match="fraction"):
        runtime.diffusion(comps, 2, 1.5, a, b)
