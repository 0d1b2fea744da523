"""The oracle renders the records of tests/test_color_paths_gpu.py on the CPU (Mallett
reconstruction, input spaces and decodings, the reference's nine output encodings):
finite output inside [0, 1] and distinct results where the branch changes the math.
The values themselves are pinned against the reference's CUDA in the GPU test."""
import json
import os

import numpy as np
import pytest

from film_juicer_b200 import abi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(GOLDEN, "output_encoding_cases.json")) as fh:
    ENCODINGS = json.load(fh)["entries"]


def test_encoding_fixture_covers_every_cctf_kind():
    assert sorted({e["cctf_kind"] for e in ENCODINGS}) == [0, 1, 2, 3, 4, 5]
    assert [e["color_space"] for e in ENCODINGS] == list(range(9))


@pytest.mark.parametrize("route", ["direct", "print"])
def test_oracle_renders_mallett_and_encodings(oracle, recipes, prepare, route):
    src = np.ascontiguousarray(prepare.synthetic_frame(24, 16, seed=3))
    base, _ = oracle.render(prepare.HostRecord(recipes[route]), src)
    mal, _ = oracle.render(prepare.HostRecord(recipes[route], method=abi.FJ_RAW_MALLETT_2019), src)
    assert np.all(np.isfinite(mal)) and float(np.abs(mal - base).max()) > 1e-3
    outs = []
    for e in ENCODINGS:
        out, _ = oracle.render(prepare.HostRecord(recipes[route], encoding=e), src)
        assert np.all(np.isfinite(out)) and out.min() >= 0.0 and out.max() <= 1.0
        outs.append(out)
    assert len({o.tobytes() for o in outs}) >= 6
