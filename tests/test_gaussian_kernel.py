"""Gaussian taps of the library (fjb_gaussian_kernel_host, which replaces the host's
FjHostPreparation.gaussian callback) against the reference's native characterization:
188 arrays (scanner lens/unsharp/glare, grain correlation and dye-cloud, small FIR DIR
kernels, literal edge cases), exact f32 words. Cases the reference records as empty are
inputs its active API rejects. No GPU."""
import ctypes as C
import json
import os
import struct

from conftest import GOLDEN


def test_gaussian_taps_match_reference_words():
    import __graft_entry__

    pkg = __graft_entry__.package()
    lib = pkg.load_library()
    from film_juicer_b200 import abi

    with open(os.path.join(GOLDEN, "gaussian_cases.json")) as fh:
        cases = json.load(fh)
    assert len(cases) == 188
    checked = rejected = 0
    for c in cases:
        sigma = struct.unpack("<f", struct.pack("<I", c["sigma_bits"]))[0]
        n = 2 * max(c["radius"], 0) + 1
        buf = (C.c_float * n)()
        err = abi.ErrorText()
        st = lib.fjb_gaussian_kernel_host(c["radius"], sigma, buf, n, C.byref(err.buf))
        if not c["weights"]:
            assert st.category != 0, c["name"]
            rejected += 1
            continue
        assert st.category == 0, (c["name"], err.text)
        got = [struct.unpack("<I", struct.pack("<f", v))[0] for v in buf]
        assert got == c["weights"], c["name"]
        checked += 1
    assert (checked, rejected) == (101, 87)
