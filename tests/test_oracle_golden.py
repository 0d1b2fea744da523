"""The CPU oracle is pinned against the reference's characterization fixtures.

scanner_lut_cases.npz holds every successful case of the reference's scanner LUT
fixture (tests/scanner/lut-fixtures/native.json): tiny cases covering NaN/inf/zero/
negative weights, baseline on/off, media 0/1/2/255, plus four real 81-sample,
resolution-17 products. The oracle must reproduce all six arrays word for word.
"""
import ctypes as C
import os

import numpy as np
import pytest

from film_juicer_b200 import abi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ARRAYS = ("log2_xyz", "slope_c", "slope_m", "slope_y", "cell_min", "cell_max")


def scanner_inputs():
    z = np.load(os.path.join(GOLDEN, "scanner_lut_cases.npz"))
    cases = []
    for name in z["names"]:
        name = str(name)
        keep = []

        def span(words):
            a = np.ascontiguousarray(np.asarray(words, dtype=np.uint32).view(np.float32))
            keep.append(a)
            return abi.FjFloatSpan(a.ctypes.data_as(C.POINTER(C.c_float)), a.size)

        inp = abi.FjbScannerLutInput()
        for key, field in (("eps_c", "eps_c"), ("eps_m", "eps_m"), ("eps_y", "eps_y"),
                           ("weighted_x", "weighted_x"), ("weighted_y", "weighted_y"),
                           ("weighted_z", "weighted_z"), ("baseline", "baseline_min")):
            setattr(inp, field, span(z[f"{name}__in_{key}"]))
        for i, v in enumerate(z[f"{name}__in_range_min_cmy"].view(np.float32)):
            inp.range_min_cmy[i] = v
        for i, v in enumerate(z[f"{name}__in_inverse_span_cmy"].view(np.float32)):
            inp.inverse_span_cmy[i] = v
        sc = z[f"{name}__in_scalars"]
        inp.inv_yn = np.array([sc[0]], dtype=np.uint32).view(np.float32)[0]
        inp.has_baseline, inp.medium, inp.resolution, inp.sample_count = int(sc[1]), int(sc[2]), int(sc[3]), int(sc[4])
        expected = {k: z[f"{name}__out_{k}"] for k in ARRAYS}
        cases.append((name, inp, expected, keep))
    return cases


CASES = scanner_inputs()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_oracle_scanner_lut_matches_reference_words(oracle, case):
    name, inp, expected, _keep = case
    rc, outs = oracle.scanner_lut(inp)
    assert rc == 0
    for key, got in zip(ARRAYS, outs):
        assert np.array_equal(got.view(np.uint32), expected[key]), f"{name}.{key}"


def test_fixture_covers_products_and_edge_cases():
    names = [c[0] for c in CASES]
    assert sum(n.startswith("LUT_PRODUCT") for n in names) == 4
    assert any("NAN" in n for n in names) and any("INFINITE" in n for n in names)
