import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402

__graft_entry__.package()
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")


@pytest.fixture(scope="session")
def prepare():
    from film_juicer_b200 import prepare as p

    return p


@pytest.fixture(scope="session")
def recipes(prepare):
    return {name: prepare.PreparedRecipe.load(os.path.join(GOLDEN, f"recipe_{name}.npz"))
            for name in ("direct", "print", "positive")}


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as orc

    orc.load()
    return orc


@pytest.fixture(scope="session")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="session")
def effects_case():
    """FjFilmEffects records of the reference's effects-frame characterization
    (tests/golden/effects_cases.json), with the defect slot probabilities raised so
    that a small frame shows dust and scratches."""
    import json
    import struct

    from film_juicer_b200 import abi, descriptors

    with open(os.path.join(GOLDEN, "effects_cases.json")) as fh:
        cases = {c["case"]: c["native"] for c in json.load(fh)}

    def f32(bits):
        return struct.unpack("<f", struct.pack("<I", bits & 0xFFFFFFFF))[0]

    def i64(v):
        return v - (1 << 64) if v >= (1 << 63) else v

    def make(case: int, slots=(0.12, 0.3, 0.1, 0.25)):
        n = cases[case]
        fams = {}
        for k, (name, rec) in enumerate((("film_dust", abi.FjDust), ("film_scratch", abi.FjScratch),
                                         ("gate_dust", abi.FjDust), ("gate_scratch", abi.FjScratch))):
            values = {field: f32(bits) for (field, _), bits in zip(rec._fields_, n[name])}
            if values["slot_probability"] > 0.0 and slots is not None:
                values["slot_probability"] = slots[k]
            fams[name] = values
        flags = ((abi.FJ_EFFECTS_WEAVE if n["weave_active"] else 0) | (abi.FJ_EFFECTS_FILM if n["film_active"] else 0)
                 | (abi.FJ_EFFECTS_GATE_TRANSMITTANCE if n["gate_transmittance_active"] else 0)
                 | (abi.FJ_EFFECTS_GATE_OUTPUT if n["gate_output_active"] else 0)
                 | (abi.FJ_EFFECTS_FULL_FRAME if n["requires_full_frame"] else 0))
        e = descriptors.film_effects_record(
            **fams, origins=[(i64(o[0]), i64(o[1]), f32(o[2]), f32(o[3])) for o in n["origins"]], flags=flags,
            sample_step_mm=(f32(n["sample_step_x_mm"]), f32(n["sample_step_y_mm"])),
            roi_offset=(n["roi_offset_x"], n["roi_offset_y"]), gate_size=(n["gate_width"], n["gate_height"]),
            session_seed=n["session_seed"], clip_token=n["clip_token"],
            weave=(f32(n["weave_dx_px"]), f32(n["weave_dy_px"]), f32(n["weave_cos_rot"]), f32(n["weave_sin_rot"])),
            recipe_hash=n["recipe_hash"], hash=n["hash"])
        x, y, w, h = n["render_extent"]
        e.render_extent.x, e.render_extent.y, e.render_extent.width, e.render_extent.height = x, y, w, h
        x, y, w, h = n["full_frame_extent"]
        e.full_frame_extent.x, e.full_frame_extent.y = x, y
        e.full_frame_extent.width, e.full_frame_extent.height = w, h
        return e

    make.cases = sorted(cases)
    return make
