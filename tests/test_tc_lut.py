"""The film TC LUT oracle (oracle/tc_lut.py) pinned on the reference's characterization
(tests/golden/tc_lut_cases.json, from tests/ffi/fixtures/tc_lut/records-0.json): the
FNV-1a digest of every complete table it builds (Hanatos with and without spectral
blur, surface correction or input compression, Arctic, negative and NaN blur
bypasses) and the requirement of every case the
reference rejects."""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "tc_lut_cases.json")
with open(GOLDEN) as fh:
    CASES = json.load(fh)
with open(os.path.join(os.path.dirname(__file__), "golden", "tc_lut_hull.json")) as fh:
    _HULL = json.load(fh)
# cases whose first source word the characterization replaces (tests/ffi/tc_lut_test.cpp:101-105)
PATCH = {21: np.inf, 22: np.nan}


def f32(bits):
    return np.uint32(bits).view(np.float32)


def inputs(case):
    from oracle import tc_lut

    spectra = tc_lut.procedural_spectra()
    if case["id"] in PATCH:
        spectra = spectra.copy()
        spectra[0] = PATCH[case["id"]]
    sens = np.array([[f32(v) for v in row] for row in case["sensitivity"]], np.float32)
    ill = np.array([f32(v) for v in case["spd"]], np.float32)
    white = [f32(v) for v in case["white"]]
    surface = None
    if case.get("surface"):
        surface = np.array([[f32(v) for v in row] for row in case["surface_params"]], np.float32)
    hull = None
    if case.get("compression") and case.get("hull_available"):
        hull = ([f32(v) for v in _HULL["center"]], np.array([[f32(a), f32(b)] for a, b in _HULL["xy"]], np.float32))
    return spectra, sens, ill, white, case["method"], f32(case["blur"]), surface, bool(case.get("compression")), hull


@pytest.mark.parametrize("case", CASES, ids=[str(c["id"]) for c in CASES])
def test_oracle_tc_lut_matches_reference_words(case):
    from oracle import tc_lut

    args = inputs(case)
    if not case["built"]:
        with np.errstate(invalid="ignore", over="ignore"):
            with pytest.raises(ValueError) as e:
                tc_lut.build_tc_lut(*args)
        assert str(e.value) == case["requirement"]
        return
    table = tc_lut.build_tc_lut(*args)
    assert tc_lut.digest(table) == int(case["digest"])
    words = table.view(np.uint32).reshape(-1, 4)
    for sel in case["selected"]:
        assert list(words[sel["cell"], :3]) == sel["rgb"]
