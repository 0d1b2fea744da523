"""Construction of the reflected recursive-Gaussian boundary (start weights and end
matrix of each axis) against the reference's characterization fixture
(tests/dir/boundary-fixtures: 87 successful cases with the exact binary64 words the
reference's double-double builder produced), for both builders:

* the library's host builder (fjb_dir_boundary_host), which the render path uses;
* the oracle's own restatement (oracle_dir_boundary in oracle/oracle.c), which the
  oracle's spatial-DIR chain uses, so that the oracle does not depend on the product.

Both carry the reference's double-double intermediates in the same operation order,
so every word must be bit-identical, with the retained lengths and terminal sizes
equal. Runs on the CPU (host code; no GPU call)."""
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
        assert np.array_equal(got_w.view(np.uint64), exp_w.view(np.uint64)), (axis, np.max(np.abs(got_w - exp_w)))
        got_t = np.array(t[:])
        assert np.array_equal(got_t.view(np.uint64), exp_t.view(np.uint64)), (axis, got_t, exp_t)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_oracle_boundary_matches_reference_words(case, oracle):
    from oracle import dir as odir

    name, g, axes = case
    for axis, (length, exp_len, exp_ts, exp_w, exp_t) in axes.items():
        w, n, ts, t = odir.boundary(g, length)
        assert (n, ts) == (exp_len, exp_ts), axis
        assert np.array_equal(w.view(np.uint64), exp_w.view(np.uint64)), (axis, np.max(np.abs(w - exp_w)))
        assert np.array_equal(t.view(np.uint64), exp_t.view(np.uint64)), axis


@pytest.mark.parametrize("length", [1, 2, 3, 4, 61, 1080, 1920, 2160, 3840])
@pytest.mark.parametrize("frame_width", [1920, 3840])
def test_oracle_and_library_boundaries_agree_at_frame_lengths(length, frame_width, oracle):
    """The frame lengths the parity tests and the bench use, which the fixture does not
    hold: both builders give the same words for the 200 um tail components of a 35 mm
    gate scanned at 1920 or 3840 pixels."""
    from film_juicer_b200 import descriptors
    from oracle import dir as odir

    lib = load_library()
    rec = descriptors.spatial_dir_record(35000.0 / frame_width, frame_width, frame_width)
    checked = 0
    for i in range(rec.component_count):
        g = rec.components[i]
        if g.reference_operator != 3 or not g.weight > 0.0:
            continue
        w, n, ts, t = odir.boundary(g, length)
        cap = 3 * length
        lw = (C.c_double * cap)()
        lt = (C.c_double * 9)()
        ln, lts = C.c_int32(), C.c_int32()
        err = abi.ErrorText()
        st = lib.fjb_dir_boundary_host(C.byref(g), length, lw, cap, C.byref(ln), C.byref(lts), lt, C.byref(err.buf))
        assert st.category == 0, err.text
        assert (ln.value, lts.value) == (n, ts)
        assert np.array_equal(np.array(lw[: 3 * n]).view(np.uint64), w.view(np.uint64))
        assert np.array_equal(np.array(lt[:]).view(np.uint64), t.view(np.uint64))
        checked += 1
    assert checked >= 1


def test_fixture_covers_frame_geometries():
    sizes = {(c[2]["horizontal"][0], c[2]["vertical"][0]) for c in CASES}
    assert (64, 48) in sizes and (1, 1) in sizes
