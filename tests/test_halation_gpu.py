"""Scatter / halation (a16) on the GPU against the CPU oracle and the reference's own
CUDA kernels.

The B200 pass evaluates every Gaussian of a channel in one row sweep and one column
sweep and filters rows before columns for every operator kind (the reference filters
FIR columns first); in exact arithmetic the result is identical, in FP32 it differs
by rounding only. Bound: the reference's own FIR parity bound, max |d| <= 2e-5 +
2e-5 |ref| (tests/scatter_halation/README.md:30-32 of the reference), on planes of
O(1) values.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL_ABS, TOL_REL = 2e-5, 2e-5

CASES = {
    # (pixel size um, width, height, legacy YVV)
    "1080p_35mm": (18.23, 240, 135, True),
    "4k_35mm": (9.11, 160, 97, True),
    "factored": (12.0, 131, 77, False),
    "tiny": (18.0, 7, 5, True),
    "one_row": (18.0, 64, 1, True),
    "one_col": (18.0, 1, 40, True),
    # lines too long for shared memory: the global-memory block-parallel form
    "long_rows": (9.11, 12800, 2, True),
    "long_cols": (9.11, 2, 6600, False),
}


def planes(w, h, seed):
    rng = np.random.default_rng(seed)
    base = rng.uniform(0.0, 2.0, size=(3, h, w)).astype(np.float32)
    base[:, h // 2, w // 2] += 50.0  # an impulse, as the reference's impulse rows
    return [np.ascontiguousarray(p) for p in base]


@pytest.mark.parametrize("name", list(CASES))
def test_scatter_halation_matches_oracle(torch_cuda, prepare, name):
    torch = torch_cuda
    from film_juicer_b200 import runtime
    from oracle import optics

    px, w, h, legacy = CASES[name]
    d = prepare.scatter_halation_record(px, legacy=legacy)
    src = planes(w, h, 11)
    dev = [torch.from_numpy(p).cuda() for p in src]
    runtime.scatter_halation(d, dev)
    got = [t.cpu().numpy() for t in dev]
    ref = optics.scatter_halation(d, src)
    for g, r in zip(got, ref):
        assert np.all(np.isfinite(g))
        err = np.abs(g - r)
        assert np.all(err <= TOL_ABS + TOL_REL * np.abs(r)), float(err.max())


@pytest.mark.parametrize("name", ["1080p_35mm", "factored", "tiny"])
def test_scatter_halation_matches_reference_cuda(torch_cuda, prepare, oracle, name):
    torch = torch_cuda
    from film_juicer_b200 import runtime
    from oracle import optics

    px, w, h, legacy = CASES[name]
    d = prepare.scatter_halation_record(px, legacy=legacy)
    src = planes(w, h, 12)
    ref = optics.reference_scatter_halation(torch, d, src)
    if ref is None:
        pytest.skip("reference CUDA harness not built")
    dev = [torch.from_numpy(p).cuda() for p in src]
    runtime.scatter_halation(d, dev)
    orc = optics.scatter_halation(d, src)
    for g, o, r in zip([t.cpu().numpy() for t in dev], orc, ref):
        assert np.all(np.abs(g - r) <= TOL_ABS + TOL_REL * np.abs(r)), float(np.abs(g - r).max())
        assert np.all(np.abs(o - r) <= TOL_ABS + TOL_REL * np.abs(r)), float(np.abs(o - r).max())


def test_scatter_off_and_strength_zero_are_identity(torch_cuda, prepare):
    torch = torch_cuda
    from film_juicer_b200 import runtime

    d = prepare.scatter_halation_record(18.0, scatter_amount=0.0, strength=(0.0, 0.0, 0.0))
    src = planes(33, 21, 3)
    dev = [torch.from_numpy(p).cuda() for p in src]
    runtime.scatter_halation(d, dev)
    for t, p in zip(dev, src):
        assert np.array_equal(t.cpu().numpy(), p)


def test_energy_is_preserved_by_renormalized_halation(torch_cuda, prepare):
    """Interior mass: scatter mixes normalized kernels, renormalized bounces divide by
    1 + s after adding s * (normalized blur), so a flat field stays flat."""
    torch = torch_cuda
    from film_juicer_b200 import runtime

    d = prepare.scatter_halation_record(9.11)
    flat = [np.full((120, 200), v, np.float32) for v in (0.5, 1.0, 2.0)]
    dev = [torch.from_numpy(p).cuda() for p in flat]
    runtime.scatter_halation(d, dev)
    for t, v in zip(dev, (0.5, 1.0, 2.0)):
        got = t.cpu().numpy()
        assert np.allclose(got, v, rtol=2e-5, atol=0), float(np.abs(got - v).max())
