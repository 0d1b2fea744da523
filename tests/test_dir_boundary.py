"""The library's host construction of the reflected recursive-Gaussian boundary
(start weights and end matrix of each axis) against the reference's characterization
fixture (tests/dir/boundary-fixtures: 87 successful cases with the exact binary64
words the reference's double-double builder produced).

The library computes in binary64 throughout, the reference carries double-double
intermediates, so words may differ in the last bits: the bound is
1e-13 max(1, |ref|) per word (the reference certifies row sums to ~1e-12), with the
retained lengths and terminal sizes exactly equal. Runs on the CPU (host code of the
library; no GPU call)."""
import ctypes as C
import os

import numpy as np
import pytest

from film_juicer_b200 import abi, load_library

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_cases():
    z = np.load(os.path.join(GOLDEN, "dir_boundary_cases.npz"))
    cases = []
    for name in z["names"]:
        name = str(name)
        g = abi.FjDirGaussian()
        u32 = z[f"{name}__u32"].view(np.float32)
        g.sigma_px, g.weight = float(u32[0]), float(u32[1])
        radius, op, version, width, height = (int(v) for v in z[f"{name}__i32"])
        g.radius, g.reference_operator, g.boundary_derivation_version = radius, op, version
        f = z[f"{name}__f64"].view(np.float64)
        g.feedforward = f[0]
        for i in range(3):
            g.feedback[i] = f[1 + i]
        g.normalization_denominator = f[4]
        g.feedforward_numerator = f[5]
        for i in range(3):
            g.feedback_numerators[i] = f[6 + i]
        g.boundary_truncation_accuracy = f[9]
        g.boundary_certification_tolerance = f[10]
        axes = {}
        for axis, length in (("horizontal", width), ("vertical", height)):
            meta = z[f"{name}__{axis}_meta"]
            axes[axis] = (length, int(meta[0]), int(meta[1]), z[f"{name}__{axis}_weights"].view(np.float64),
                          z[f"{name}__{axis}_terminal"].view(np.float64))
        cases.append((name, g, axes))
    return cases


CASES = load_cases()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_boundary_matches_reference_words(case):
    lib = load_library()
    name, g, axes = case
    for axis, (length, exp_len, exp_ts, exp_w, exp_t) in axes.items():
        cap = 3 * max(length, 1)
        w = (C.c_double * cap)()
        t = (C.c_double * 9)()
        n, ts = C.c_int32(), C.c_int32()
        err = abi.ErrorText()
        st = lib.fjb_dir_boundary_host(C.byref(g), length, w, cap, C.byref(n), C.byref(ts), t, C.byref(err.buf))
        assert st.category == 0, err.text
        assert n.value == exp_len, (axis, n.value, exp_len)
        assert ts.value == exp_ts
        got_w = np.array(w[: 3 * n.value])
        assert got_w.shape == exp_w.shape
        tol_w = 1e-13 * np.maximum(1.0, np.abs(exp_w))
        assert np.all(np.abs(got_w - exp_w) <= tol_w), (axis, np.max(np.abs(got_w - exp_w)))
        got_t = np.array(t[:])
        assert np.all(np.abs(got_t - exp_t) <= 1e-13 * np.maximum(1.0, np.abs(exp_t))), (axis, got_t, exp_t)


def test_fixture_covers_frame_geometries():
    sizes = {(c[2]["horizontal"][0], c[2]["vertical"][0]) for c in CASES}
    assert (64, 48) in sizes and (1, 1) in sizes
