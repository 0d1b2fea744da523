"""The film TC LUT built on the device (fjb_tc_lut_build) against the reference's
characterization: the complete table's FNV-1a digest for every case it builds, the
rejected cases with the reference's requirement, and the table word for word equal to
the oracle's."""
import numpy as np
import pytest

from test_tc_lut import CASES, PATCH, inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", CASES, ids=[str(c["id"]) for c in CASES])
def test_device_tc_lut_matches_reference_words(torch_cuda, case):
    from film_juicer_b200 import runtime
    from oracle import tc_lut

    torch = torch_cuda
    spectra, sens, ill, white, method, blur, surface, compression, hull = inputs(case)
    dev = torch.from_numpy(spectra).cuda()
    if not case["built"]:
        with pytest.raises(runtime.FjError) as e:
            runtime.tc_lut_build(dev, sens, ill, white, method, float(blur), surface, compression, hull)
        assert str(e.value).rstrip().endswith("requirement=" + case["requirement"])
        return
    table = runtime.tc_lut_build(dev, sens, ill, white, method, float(blur), surface, compression, hull).cpu().numpy()
    assert tc_lut.digest(table) == int(case["digest"])
    want = tc_lut.build_tc_lut(spectra, sens, ill, white, method, blur, surface, compression, hull)
    assert np.array_equal(table.view(np.uint32), want.view(np.uint32))


def test_device_tc_lut_rejects_unknown_methods(torch_cuda):
    import ctypes as C

    import film_juicer_b200 as pkg
    from film_juicer_b200 import abi

    lib = pkg.load_library()
    sens = np.ones(243, np.float32)
    ill = np.ones(81, np.float32)
    inp = abi.FjbTcLutInput()
    inp.spectra = 16
    inp.sensitivity_rgb = sens.ctypes.data_as(C.POINTER(C.c_float))
    inp.reference_illuminant = ill.ctypes.data_as(C.POINTER(C.c_float))
    inp.method = 1
    err = abi.ErrorText()
    st = lib.fjb_tc_lut_build(C.byref(inp), C.c_void_p(16), None, C.byref(err.buf))
    assert st.category == abi.FJ_STATUS_PREPARATION_FAILURE and "method" in err.text
