"""Generates the committed golden fixtures from the reference tree (run in the build
container, where the reference is mounted read-only).

* scanner_lut_cases.npz: the reference's scanner LUT characterization
  (tests/scanner/lut-fixtures/native.json): every case's input words and the exact
  f32 words of the six arrays the native builder produced.
* recipe_direct.npz / recipe_print.npz: prepared recipes (film_juicer_b200.prepare)
  for kodak_portra_400 direct and kodak_portra_400 -> kodak_portra_endura print,
  built from the reference's Resources/ profiles and spectral tables.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("FJ_REFERENCE_ROOT", "/root/reference")


def scanner_cases():
    with open(os.path.join(REF, "tests", "scanner", "lut-fixtures", "native.json")) as fh:
        d = json.load(fh)
    out = {}
    names = []
    for group in ("cases", "products"):
        for case in d[group]:
            inp, nat = case["input"], case["native"]
            if not nat.get("success", False):
                continue
            cid = case["id"].replace("-", "_")
            names.append(cid)
            for key in ("eps_c", "eps_m", "eps_y", "weighted_x", "weighted_y", "weighted_z", "baseline"):
                out[f"{cid}__in_{key}"] = np.array(inp.get(key, []), dtype=np.uint32)
            for key in ("range_min_cmy", "inverse_span_cmy"):
                out[f"{cid}__in_{key}"] = np.array(inp[key], dtype=np.uint32)
            out[f"{cid}__in_scalars"] = np.array([inp["inv_yn"], int(inp["has_baseline"]), inp["medium"],
                                                  inp["resolution"], inp["sample_count"]], dtype=np.uint64)
            for key in ("log2_xyz", "slope_c", "slope_m", "slope_y", "cell_min", "cell_max"):
                out[f"{cid}__out_{key}"] = np.array(nat[key], dtype=np.uint32)
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "scanner_lut_cases.npz"), **out)
    print("scanner cases:", len(names))


def dir_boundary_cases():
    """Reflected-YVV boundary characterization (tests/dir/boundary-fixtures): inputs and
    the exact binary64 words of both axes' weights and terminal matrices."""
    base = os.path.join(REF, "tests", "dir", "boundary-fixtures")
    with open(os.path.join(base, "inputs.json")) as fh:
        inputs = json.load(fh)["cases"]
    with open(os.path.join(base, "linux-release.json")) as fh:
        outputs = {c["input"]["name"] if "name" in c.get("input", {}) else i: c
                   for i, c in enumerate(json.load(fh)["cases"])}
    out = {}
    names = []
    for i, case in enumerate(inputs):
        res = outputs.get(case["name"], outputs.get(i))
        if res is None or not res.get("success"):
            continue
        cid = f"c{i:03d}"
        names.append(cid)
        comp = case["component"]
        out[f"{cid}__u32"] = np.array([comp["sigma"], comp["weight"]], dtype=np.uint32)
        out[f"{cid}__i32"] = np.array([comp["radius"], comp["operator"], comp["version"], case["width"],
                                       case["height"]], dtype=np.int64)
        out[f"{cid}__f64"] = np.array([comp["feedforward"], *comp["feedback"], comp["denominator"],
                                       comp["numerator"], *comp["numerators"], comp["accuracy"],
                                       comp["tolerance"]], dtype=np.uint64)
        for axis in ("horizontal", "vertical"):
            ax = res[axis]
            out[f"{cid}__{axis}_meta"] = np.array([ax["length"], ax["terminal_size"]], dtype=np.int64)
            out[f"{cid}__{axis}_weights"] = np.array(ax["weights"], dtype=np.uint64)
            out[f"{cid}__{axis}_terminal"] = np.array(ax["terminal"], dtype=np.uint64)
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "dir_boundary_cases.npz"), **out)
    print("dir boundary cases:", len(names))


def recipes():
    sys.path.insert(0, ROOT)
    import __graft_entry__

    __graft_entry__.package()
    from film_juicer_b200 import prepare

    res = os.path.join(REF, "Resources")
    prepare.prepare_recipe(res, "kodak_portra_400").save(os.path.join(HERE, "recipe_direct.npz"))
    prepare.prepare_recipe(res, "kodak_portra_400", "kodak_portra_endura").save(os.path.join(HERE, "recipe_print.npz"))
    print("recipes written")


if __name__ == "__main__":
    scanner_cases()
    dir_boundary_cases()
    recipes()
