"""The output gamut boundary oracle (oracle/gamut.py) pinned on the reference's
characterization (tests/golden/gamut_cases.json, from tests/ffi/fixtures/output_gamut):
the FNV-1a digest of the 64 x 720 cmax table of every output space it builds, and the
rejection of the space whose chroma endpoint stays inside the cube."""
import json
import os

import numpy as np
import pytest

with open(os.path.join(os.path.dirname(__file__), "golden", "gamut_cases.json")) as fh:
    GAMUT = json.load(fh)
# a few spaces on the CPU (each table is 46 080 bisections in Python); all of them on the GPU
CPU_ROWS = [r for r in GAMUT["rows"] if (r["tag"], r["variant"]) in ((0, 0), (0, 6), (3, 0))]


def gamut_inputs(row):
    from oracle import gamut

    m = [gamut.f64(b) for b in row["lms_to_native"]]
    d = [(gamut.f64(a), gamut.f64(b)) for a, b in GAMUT["directions"]]
    lab = [gamut.f32(b) for b in GAMUT["lab_to_lms_root"]]
    return m, d, lab


def fnv(table):
    h = 0xCBF29CE484222325
    for b in np.ascontiguousarray(table, np.float32).tobytes():
        h = ((h ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


@pytest.mark.parametrize("row", CPU_ROWS, ids=[f"{r['tag']}-{r['variant']}" for r in CPU_ROWS])
def test_oracle_gamut_boundary_matches_reference_words(row):
    from oracle import gamut

    args = gamut_inputs(row)
    if not row["ok"]:
        with pytest.raises(ValueError, match=row["requirement"]):
            gamut.build(*args)
        return
    assert fnv(gamut.build(*args)) == int(row["digest"])


@pytest.mark.gpu
@pytest.mark.parametrize("row", GAMUT["rows"], ids=[f"{r['tag']}-{r['variant']}" for r in GAMUT["rows"]])
def test_device_gamut_boundary_matches_reference_words(torch_cuda, row):
    import ctypes as C

    import film_juicer_b200 as pkg
    from film_juicer_b200 import abi

    torch = torch_cuda
    m, _, _ = gamut_inputs(row)
    mm = (C.c_double * 9)(*m)
    cmax = torch.full((64 * 720,), -1.0, device="cuda")
    err = abi.ErrorText()
    st = pkg.load_library().fjb_gamut_boundary_build(mm, C.c_void_p(cmax.data_ptr()), None, C.byref(err.buf))
    if not row["ok"]:
        assert st.category == abi.FJ_STATUS_PREPARATION_FAILURE and ("requirement=" + row["requirement"]) in err.text
        return
    assert st.category == abi.FJ_STATUS_SUCCESS, err.text
    assert fnv(cmax.cpu().numpy()) == int(row["digest"])


def _failing_matrices():
    """Matrices the reference rejects at an entry other than the first: the first output
    space scaled and one native channel zeroed (that channel stays inside the cube at
    the chroma endpoint for some hues)."""
    m, _, _ = gamut_inputs(GAMUT["rows"][0])
    out = []
    for scale, row in ((0.05, 1), (0.1, 2)):
        mm = [v * scale for v in m]
        for k in range(3):
            mm[row * 3 + k] = 0.0
        out.append(mm)
    return out


FAILING = _failing_matrices()


@pytest.mark.parametrize("case", range(len(FAILING)))
def test_oracle_reports_first_failing_entry(case):
    from oracle import gamut

    _, d, lab = gamut_inputs(GAMUT["rows"][0])
    with pytest.raises(ValueError) as info:
        gamut.build(FAILING[case], d, lab)
    assert str(info.value).startswith("c2_outside lightness_index=0 hue_index=")
    assert not str(info.value).endswith("hue_index=0")


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(FAILING)))
def test_device_reports_the_oracles_first_failing_entry(torch_cuda, case):
    """The device build reports the same requirement, and for c2_outside the same
    (lightness, hue) entry, as the reference's sequential scan (oracle)."""
    import ctypes as C

    import film_juicer_b200 as pkg
    from film_juicer_b200 import abi
    from oracle import gamut

    torch = torch_cuda
    _, d, lab = gamut_inputs(GAMUT["rows"][0])
    with pytest.raises(ValueError) as info:
        gamut.build(FAILING[case], d, lab)
    cmax = torch.full((64 * 720,), -1.0, device="cuda")
    err = abi.ErrorText()
    mm = (C.c_double * 9)(*FAILING[case])
    st = pkg.load_library().fjb_gamut_boundary_build(mm, C.c_void_p(cmax.data_ptr()), None, C.byref(err.buf))
    assert st.category == abi.FJ_STATUS_PREPARATION_FAILURE
    assert err.text.endswith("requirement=" + str(info.value)), (err.text, str(info.value))
