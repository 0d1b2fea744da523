"""Generates the committed golden fixtures from the reference tree (run in the build
container, where the reference is mounted read-only).

* scanner_lut_cases.npz: the reference's scanner LUT characterization
  (tests/scanner/lut-fixtures/native.json): every case's input words and the exact
  f32 words of the six arrays the native builder produced.
* diffusion_component_cases.npz: the reference's diffusion component
  characterization (tests/diffusion/frame-fixtures/manifest.json, production cases
  "diffusion/components/*"): input words (family, 3 group weights, 3 group centers,
  warmth, spatial scale, pixel size, radius, hash) and the 36 binary64 output words
  (lambda_px, red, green, blue weights), or the failure flag.
* diffusion_images.npz: the reference's external diffusion cohort
  (tests/diffusion/fixtures/diffusion_reference_v1.{json,npz}, produced by the
  upstream model the reference ports): 17x19, 16x18, 23x11, 11x23 RGB inputs, the
  filter parameters of each case mapped onto the diffusion record (group weights =
  family weights x intensities, group centres = family centres x sizes, warmth =
  family base + halo warmth clamped to [-1.5, 1.5], scatter fraction from the
  strength table) and the float32 outputs.
* grain_plan_cases.json: the reference's visual-grain frame characterization
  (tests/grain/frame-fixtures/linux-release.json): inputs and exact native output
  fields of every successful case, and the gaussian / energy / period primitives.
* wang_lut.json: the Wang tile index table of Resources/Noise/Wang/tiles.json.
* density_model_cases.npz: the reference's density-model characterization
  (tests/profile/fixtures/density.json + density-samples.bin): per case with frozen
  samples, the model's centre / amplitude / sigma f64 bits ([channel][layer]), the
  polarity, the log-exposure axis (f64 bits) and the 49-byte sample records (validity
  byte, then totals C, M, Y and layers [layer][channel] as f32 bits).
* output_encoding_cases.json: the reference's frozen output-encoding table
  (tests/scanner/output_encoding_native.inc): per output colour space index, the CCTF
  kind, its six f32 parameters (gamma, a, b, c, d, linear cutoff) and the DWG-to-output
  matrix, as f32 words.
* abi_layout_reference.json: sizeof of every record of the reference's C-ABI header
  (native/juicer_cuda_api.h) and offsetof of every field, as the system C compiler
  lays them out; the drop-in boundary test compares the repository's header with it.
* print_cases.npz: the reference's print characterizations (tests/print/
  {balance,preflash,illuminant}-fixtures, linux-release native profile): the inputs
  and exact f32 output words and hashes of the 42 balance cases and 60 balance product
  records, the 19 preflash cases, the 127 filtered-illuminant literal cases (with the
  Rust build's words beside the native ones), the distinct product main / preflash
  illuminants on the TH-KG3 lamp, and the KG3 transmission rows (Resources/filters/
  heat_absorbing/schott/KG3.csv) that lamp is built from.
* dir_recipe_cases.json: the reference's capture DIR characterization
  (tests/film/dir-fixtures/linux.json, 64 products of four stocks): controls and the
  exact words and hashes of each recipe, and per stock the profile's info block,
  Gaussian density model and log-exposure axis.
* recipe_direct.npz / recipe_print.npz: prepared recipes (film_juicer_b200.prepare)
  for kodak_portra_400 direct and kodak_portra_400 -> kodak_portra_endura print, and
  recipe_vision3_500t_2383.npz / recipe_ektar100_endura.npz for the mixed-stock
  batches (kodak_vision3_500t -> kodak_2383, kodak_ektar_100 -> kodak_portra_endura),
  and recipe_positive.npz (fujifilm_provia_100f scanned directly, the positive route),
  built from the reference's Resources/ profiles, spectral tables and filters.
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


def diffusion_component_cases():
    with open(os.path.join(REF, "tests", "diffusion", "frame-fixtures", "manifest.json")) as fh:
        m = json.load(fh)
    inputs = m["production_inputs"]
    names, words, outputs, failed = [], [], [], []
    for case in m["production_cases"]:
        if not case["case"].startswith("diffusion/components/"):
            continue
        names.append(case["case"])
        words.append(np.array(inputs[case["case"]]["words"], dtype=np.uint64))
        outputs.append(np.array(case["output"], dtype=np.uint64))
        failed.append(case["envelope"][0] != 0)
    np.savez_compressed(os.path.join(HERE, "diffusion_component_cases.npz"), names=np.array(names),
                        words=np.stack(words), outputs=np.stack(outputs), failed=np.array(failed))
    print("diffusion component cases:", len(names))


def diffusion_images():
    base = os.path.join(REF, "tests", "diffusion", "fixtures")
    with open(os.path.join(base, "diffusion_reference_v1.json")) as fh:
        j = json.load(fh)
    z = np.load(os.path.join(base, "diffusion_reference_v1.npz"))
    families = {c["family"]: c for c in j["family_cases"]}
    order = j["family_order"]
    fractions = {(c["family"], c["strength"]): c["scatter_fraction"] for c in j["strength_cases"]}
    inputs, input_names = [], []
    out = {"names": [], "input_index": [], "family": [], "params": [], "radius": [], "outputs": []}
    for case in j["image_cases"] + j["radius_cases"] + j["hdr_cases"]:
        p, f = case["params"], families[case["family"]]
        weights = (f["w_c"] * p["core_intensity"], f["w_h"] * p["halo_intensity"], f["w_b"] * p["bloom_intensity"])
        centers = (f["core"]["lambda_um"] * p["core_size"], f["halo"]["lambda_um"] * p["halo_size"],
                   f["bloom"]["lambda_um"] * p["bloom_size"])
        warmth = max(-1.5, min(1.5, f["halo_warmth_base"] + p["halo_warmth"]))
        if case["input_array"] not in input_names:
            input_names.append(case["input_array"])
            inputs.append(z[case["input_array"]])
        out["names"].append(case["output_array"])
        out["input_index"].append(input_names.index(case["input_array"]))
        out["family"].append(order.index(case["family"]))
        out["params"].append([*weights, *centers, warmth, p["spatial_scale"], case["pixel_size_um"],
                              fractions[(case["family"], p["strength"])]])
        out["radius"].append(case["psf_radius"])
        out["outputs"].append(z[case["output_array"]])
    arrays = {k: np.array(v) for k, v in out.items() if k != "outputs"}
    for i, a in enumerate(inputs):
        arrays[f"input_{i}"] = a
    for i, a in enumerate(out["outputs"]):
        arrays[f"output_{i}"] = a
    np.savez_compressed(os.path.join(HERE, "diffusion_images.npz"), **arrays)
    print("diffusion image cases:", len(out["names"]))


def grain_plan_cases():
    with open(os.path.join(REF, "tests", "grain", "frame-fixtures", "linux-release.json")) as fh:
        j = json.load(fh)
    keep = ["frame0", "frame_alpha", "seed_base", "seed_base_next", "pitch_px", "breathing_period_frames",
            "clump_morph_period_frames", "wang_cell_mm", "breathing_amplitude", "breathing_cell_um_small",
            "breathing_cell_um_large", "breathing_mix", "breathing_drift_um_per_frame", "debug_scale",
            "density_max_cmy", "n_particles_cmy", "od_particle_cmy", "density_min_layers", "density_max_layers",
            "n_particles_layers", "od_particle_layers", "correlation", "dye_cloud", "size_mix_weights",
            "size_mix_gain", "requires_full_frame", "density_layers_hash"]
    cases = [{"input": c["input"], "expected": {k: c["native"][k] for k in keep}}
             for c in j["cases"] if c["success"] and c["native"]["active"]]
    prims = [p for p in j["primitives"] if p["input"]["op"] in ("gaussian", "energy", "period")]
    with open(os.path.join(HERE, "grain_plan_cases.json"), "w") as fh:
        json.dump({"cases": cases, "primitives": prims}, fh, separators=(",", ":"))
    with open(os.path.join(REF, "Resources", "Noise", "Wang", "tiles.json")) as fh:
        tiles = json.load(fh)
    lut = [0] * 16
    for e in tiles["mapping"]:
        lab = e["labels"]
        lut[((lab["L"] * 2 + lab["R"]) * 2 + lab["T"]) * 2 + lab["B"]] = e["index"]
    with open(os.path.join(HERE, "wang_lut.json"), "w") as fh:
        json.dump(lut, fh)
    print("grain plan cases:", len(cases), "primitives:", len(prims))


def gaussian_cases():
    """Normalised Gaussian taps: the reference's native characterization
    (tests/optics/gaussian-fixtures/linux-payload.json, 188 arrays of exact f32 words;
    empty arrays are inputs the active API rejects)."""
    with open(os.path.join(REF, "tests", "optics", "gaussian-fixtures", "linux-payload.json")) as fh:
        j = json.load(fh)
    cases = [{"name": c["name"], "radius": c["radius"], "sigma_bits": c["sigma_bits"], "weights": c["weights"]}
             for c in j["cases"]]
    with open(os.path.join(HERE, "gaussian_cases.json"), "w") as fh:
        json.dump(cases, fh, separators=(",", ":"))
    print("gaussian cases:", len(cases))


def effects_cases():
    """Composed film-effects records of the reference's effects-frame characterization
    (tests/film/effects-frame-fixtures/linux-debug-payload.json): the native fields of
    the active cases (float fields as IEEE bit patterns), for the defects tests."""
    with open(os.path.join(REF, "tests", "film", "effects-frame-fixtures", "linux-debug-payload.json")) as fh:
        doc = json.load(fh)
    keep, per = [], {}
    for i, case in enumerate(doc["cases"]):
        n = case.get("native") or {}
        contract = case["input"].get("contract")
        if not case.get("success") or not n.get("hash") or per.get(contract, 0) >= 3:
            continue
        per[contract] = per.get(contract, 0) + 1
        keep.append(dict(case=i, contract=contract, native=n))
    with open(os.path.join(HERE, "effects_cases.json"), "w") as fh:
        json.dump(keep, fh, separators=(",", ":"), sort_keys=True)
    print("effects cases:", len(keep))


def tc_lut_cases():
    """TC LUT characterization (tests/ffi/fixtures/tc_lut/records-0.json, built by
    tests/ffi/tc_lut_test.cpp): the cases whose source is the procedural spectra
    (word i = 0x3e000123 + (i % 4093) * 173), with the input hull of the compression
    cases in tc_lut_hull.json: inputs as IEEE bit patterns, the expected
    status and requirement, and the FNV-1a digest of the complete table."""
    with open(os.path.join(REF, "tests", "ffi", "fixtures", "tc_lut", "records-0.json")) as fh:
        doc = json.load(fh)
    keep = []
    for c in doc["leaves"]["cases"]:
        i = c["input"]
        if i["source"] != "procedural_4093_173" or i["id"] in (16, 17):
            continue
        row = dict(id=i["id"], built=c["built"], method=i["method"], blur=i["blur"], sensitivity=i["sensitivity"],
                   spd=i["spd"], white=i["white"], surface=i["surface"], surface_params=i["surface_params"],
                   compression=i["compression"], hull_available=i["hull_available"],
                   requirement=c["diagnostic"].split("requirement=")[-1] if not c["built"] else "")
        if c["built"]:
            row["digest"] = str(c["table"]["native_byte_digest_fnv1a64"])
            row["selected"] = c["table"]["selected"]
        keep.append(row)
    with open(os.path.join(HERE, "tc_lut_cases.json"), "w") as fh:
        json.dump(keep, fh, separators=(",", ":"))
    hull = doc["leaves"]["hull"]
    with open(os.path.join(HERE, "tc_lut_hull.json"), "w") as fh:
        json.dump(dict(center=hull["center"], xy=hull["xy"]), fh, separators=(",", ":"))
    print("tc lut cases:", [r["id"] for r in keep])


def gamut_cases():
    """Output gamut boundary tables (tests/ffi/fixtures/output_gamut/records-0.json and
    tables-0.bin): per output space the LMS-to-native matrix (FP64 bits), the FNV-1a
    digest of its 64 x 720 cmax table, or the builder's rejection; the 720 hue
    directions (cos, sin as FP64 bits) and the Lab-to-LMS-root matrix (f32 bits)."""
    base = os.path.join(REF, "tests", "ffi", "fixtures", "output_gamut")
    with open(os.path.join(base, "records-0.json")) as fh:
        doc = json.load(fh)
    tables = np.fromfile(os.path.join(base, "tables-0.bin"), dtype=np.uint8)
    rows = []
    for r in doc["rows"]:
        if not r["transform_ok"]:
            continue
        row = dict(tag=r["tag"], variant=r["variant"], lms_to_native=r["lms_to_native"], ok=r["boundary_ok"],
                   requirement=r["boundary_diagnostic"].split("requirement=")[-1].split(" ")[0])
        if r["boundary_ok"]:
            words = tables[r["table_offset"]:r["table_offset"] + 4 * r["table_count"]]
            h = 0xCBF29CE484222325
            for b in words.tobytes():
                h = ((h ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
            row["digest"] = str(h)
        rows.append(row)
    out = dict(rows=rows, directions=[[d[1], d[2]] for d in doc["directions"]], lab_to_lms_root=doc["oklab"][3])
    with open(os.path.join(HERE, "gamut_cases.json"), "w") as fh:
        json.dump(out, fh, separators=(",", ":"))
    print("gamut cases:", [(r["tag"], r["variant"], r["ok"]) for r in rows])


def density_model_cases():
    fx = os.path.join(REF, "tests", "profile", "fixtures")
    with open(os.path.join(fx, "density.json")) as fh:
        d = json.load(fh)
    with open(os.path.join(fx, "density-samples.bin"), "rb") as fh:
        raw = fh.read()
    out, names = {}, []
    for k, case in enumerate(d["cases"]):
        if case.get("sample_start") is None or case.get("model") is None:
            continue
        axis = d["axes"][case["axis"]]
        n = len(axis)
        name = f"c{k:03d}"
        names.append(name)
        m = case["model"]
        out[f"{name}__model"] = np.array([m["centers"], m["amplitudes"], m["sigmas"]], dtype=np.uint64)
        out[f"{name}__positive"] = np.array([1 if case["positive"] else 0], dtype=np.uint8)
        out[f"{name}__axis"] = np.array(axis, dtype=np.uint64)
        s0 = case["sample_start"] * 49
        out[f"{name}__records"] = np.frombuffer(raw[s0:s0 + n * 49], dtype=np.uint8).reshape(n, 49).copy()
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "density_model_cases.npz"), **out)
    print("density model cases:", len(names))


def output_encoding_cases():
    import re

    with open(os.path.join(REF, "tests", "scanner", "output_encoding_native.inc")) as fh:
        text = fh.read()
    body = text[text.index("kEntries"):]
    rows = []
    for chunk in body.split("{{static_cast<CctfKind>(")[1:]:
        kind = int(chunk[: chunk.index(")")])
        words = [int(w, 16) for w in re.findall(r"0x([0-9a-fA-F]+)u", chunk)]
        assert len(words) == 15, len(words)
        rows.append({"color_space": len(rows), "cctf_kind": kind, "params": words[:6], "dwg_to_output": words[6:]})
    assert len(rows) == 9
    with open(os.path.join(HERE, "output_encoding_cases.json"), "w") as fh:
        json.dump({"source": "tests/scanner/output_encoding_native.inc", "entries": rows}, fh, indent=0)
    print("output encodings:", len(rows))


def abi_layout():
    import shutil
    import subprocess
    import tempfile

    sys.path.insert(0, ROOT)
    import __graft_entry__

    __graft_entry__.package()
    from film_juicer_b200 import abi

    header = os.path.join(REF, "native", "juicer_cuda_api.h")
    with open(header) as fh:
        text = fh.read()
    records = [r for r in abi.ALL_RECORDS if f"}} {r.__name__};" in text]
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{header}"', "int main(void) {"]
    for rec in records:
        name = rec.__name__
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in rec._fields_:
            lines.append(f'printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines.append("return 0; }")
    cc = shutil.which("gcc") or shutil.which("cc")
    with tempfile.TemporaryDirectory() as tmp:
        src, exe = os.path.join(tmp, "layout.c"), os.path.join(tmp, "layout")
        with open(src, "w") as fh:
            fh.write("\n".join(lines))
        subprocess.run([cc, "-std=c11", src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    layout = {k: int(v) for k, v in (line.rsplit(" ", 1) for line in out if line)}
    with open(os.path.join(HERE, "abi_layout_reference.json"), "w") as fh:
        json.dump({"header": "native/juicer_cuda_api.h", "records": [r.__name__ for r in records],
                   "layout": layout}, fh, indent=0, sort_keys=True)
    print("abi layout:", len(records), "records")


def print_cases():
    """Print balance, preflash and filtered-illuminant characterizations as f32 words."""
    pdir = os.path.join(REF, "tests", "print")

    def load(*parts):
        with open(os.path.join(pdir, *parts)) as fh:
            return json.load(fh)

    u32 = lambda v: np.asarray(v, dtype=np.uint32)
    out = {}
    # Balance: the 42 characterization cases and the 60 product records that carry inputs.
    bal = load("balance-fixtures", "linux-release.json")
    rows = list(bal["cases"]) + [p for p in bal["products"] if "film_base_density" in p]
    for key, n in (("film_base_density", 81), ("film_channel_density_cmy", 243), ("print_sensitivity_rgb", 243),
                   ("filtered_main_illuminant", 81), ("baseline_density_cmy", 3), ("compensated_density_cmy", 3)):
        out[f"balance_{key}"] = np.stack([u32(r[key]) for r in rows])
        assert out[f"balance_{key}"].shape[1] == n
    out["balance_reference_hash"] = np.asarray([r["reference_hash"] for r in rows], dtype=np.uint64)
    out["balance_mode"] = np.asarray([r["normalization_mode"] for r in rows], dtype=np.int32)
    out["balance_success"] = np.asarray([bool(r.get("success", True)) for r in rows])
    out["balance_field"] = np.asarray([r.get("diagnostic", "").rsplit("field=", 1)[-1] if not r.get("success", True)
                                       else "" for r in rows])
    res = [r.get("balance") if r.get("success", True) else None for r in rows]
    zero = {"baseline_raw_rgb": [0] * 3, "compensated_raw_rgb": [0] * 3, "scalars": [0] * 3,
            "filtered_main_illuminant_hash": 0, "hash": 0}
    res = [b if b is not None else zero for b in res]
    out["balance_baseline_raw"] = np.stack([u32(b["baseline_raw_rgb"]) for b in res])
    out["balance_compensated_raw"] = np.stack([u32(b["compensated_raw_rgb"]) for b in res])
    out["balance_scalars"] = np.stack([u32(b["scalars"]) for b in res])
    out["balance_illuminant_hash"] = np.asarray([b["filtered_main_illuminant_hash"] for b in res], dtype=np.uint64)
    out["balance_hash"] = np.asarray([b["hash"] for b in res], dtype=np.uint64)
    out["balance_id"] = np.asarray([r.get("id", f"product-{i}") for i, r in enumerate(rows)])
    # Preflash raw integral
    pre = load("preflash-fixtures", "linux-release.json")["cases"]
    out["preflash_film_base_density"] = np.stack([u32(c["film_base_density"]) for c in pre])
    out["preflash_filtered_illuminant"] = np.stack([u32(c["filtered_illuminant"]) for c in pre])
    out["preflash_sensitivity_cmy"] = np.stack([u32(c["print_sensitivity_cmy"]) for c in pre])
    out["preflash_raw"] = np.stack([u32(c["raw"]) if c["success"] else u32([0, 0, 0]) for c in pre])
    out["preflash_success"] = np.asarray([c["success"] for c in pre])
    out["preflash_id"] = np.asarray([c["id"] for c in pre])
    # Filtered print illuminant: native (glibc erff) and Rust (libm 0.2.15 erff) expectations
    lit = load("illuminant-fixtures", "linux-release-literal.json")["cases"]
    rlit = {c["id"]: c for c in load("illuminant-fixtures", "linux-release-rust-literal.json")["cases"]}
    for key in ("edges_nm", "transitions_nm", "cmy_cc", "source", "samples"):
        out[f"illum_{key}"] = np.stack([u32(c[key]) for c in lit])
    out["illum_rust_samples"] = np.stack([u32(rlit[c["id"]]["samples"]) for c in lit])
    out["illum_success"] = np.asarray([c["success"] for c in lit])
    assert all(rlit[c["id"]]["success"] == c["success"] for c in lit)
    out["illum_id"] = np.asarray([c["id"] for c in lit])
    # Product main / preflash illuminants on the TH-KG3 enlarger source (distinct records)
    prods, seen = [], set()
    for p in load("illuminant-fixtures", "linux-release-products.json")["products"]:
        key = json.dumps([p.get("main_cmy"), p.get("main"), p.get("preflash_cmy"), p.get("preflash")])
        if p.get("main_present") and key not in seen:
            assert p["source_key"] == "TH-KG3"
            seen.add(key)
            prods.append(p)
    for key in ("main_cmy", "main", "preflash_cmy", "preflash"):
        out[f"product_{key}"] = np.stack([u32(p[key]) for p in prods])
    # the enlarger source's inputs: the KG3 heat-absorbing glass transmission rows, as text
    with open(os.path.join(REF, "Resources", "filters", "heat_absorbing", "schott", "KG3.csv")) as fh:
        out["kg3_csv"] = np.asarray(fh.read())
    np.savez_compressed(os.path.join(HERE, "print_cases.npz"), **out)
    print("print cases: balance", len(rows), "preflash", len(pre), "illuminant", len(lit), "products", len(prods))


def dir_recipe_cases():
    """Capture DIR recipe characterization (tests/film/dir-fixtures/linux.json): per case
    the stock, its controls and the exact f32 words and hashes of the recipe; per stock
    the profile's info block, Gaussian density model and log-exposure axis
    (Resources/profiles) the development curves are sampled from."""
    with open(os.path.join(REF, "tests", "film", "dir-fixtures", "linux.json")) as fh:
        cases = json.load(fh)["cases"]
    stocks = {}
    for c in cases:
        if c["key"] not in stocks:
            with open(os.path.join(REF, "Resources", "profiles", f"{c['key']}.json")) as fh:
                prof = json.load(fh)
            stocks[c["key"]] = {"info": prof["info"], "model": prof["data"]["density_curves_model"],
                                "log_exposure": prof["data"]["log_exposure"]}
    keep = ("key", "kind", "route", "controls", "dir", "success", "diagnostic")
    out = {"source": "tests/film/dir-fixtures/linux.json", "stocks": stocks,
           "cases": [{k: c[k] for k in keep if k in c} | {"authored_minimum": c["bounds"]["authored_minimum"],
                                                           "authored_maximum": c["bounds"]["authored_maximum"]}
                     for c in cases]}
    with open(os.path.join(HERE, "dir_recipe_cases.json"), "w") as fh:
        json.dump(out, fh, separators=(",", ":"))
    print("dir recipe cases:", len(cases), "stocks", len(stocks))


def recipes():
    sys.path.insert(0, ROOT)
    import __graft_entry__

    __graft_entry__.package()
    from film_juicer_b200 import prepare

    res = os.path.join(REF, "Resources")
    prepare.prepare_recipe(res, "kodak_portra_400").save(os.path.join(HERE, "recipe_direct.npz"))
    prepare.prepare_recipe(res, "kodak_portra_400", "kodak_portra_endura").save(os.path.join(HERE, "recipe_print.npz"))
    # the mixed-stock batch: three capture stocks on two print papers
    # a reversal stock scanned directly (positive route, receiver-Langmuir DIR)
    prepare.prepare_recipe(res, "fujifilm_provia_100f").save(os.path.join(HERE, "recipe_positive.npz"))
    prepare.prepare_recipe(res, "kodak_vision3_500t", "kodak_2383").save(
        os.path.join(HERE, "recipe_vision3_500t_2383.npz"))
    prepare.prepare_recipe(res, "kodak_ektar_100", "kodak_portra_endura").save(
        os.path.join(HERE, "recipe_ektar100_endura.npz"))
    print("recipes written")


if __name__ == "__main__":
    scanner_cases()
    dir_boundary_cases()
    diffusion_component_cases()
    diffusion_images()
    grain_plan_cases()
    gaussian_cases()
    effects_cases()
    tc_lut_cases()
    gamut_cases()
    density_model_cases()
    output_encoding_cases()
    abi_layout()
    print_cases()
    dir_recipe_cases()
    recipes()
