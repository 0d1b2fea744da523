"""Capture DIR recipe (film_juicer_b200.dir_prep) against the reference's DIR
characterization (tests/film/dir-fixtures/linux.json: four stocks, direct and print
routes, gamma 1 / 0.85, DIR disabled / zero amount / stock / custom controls; compact
copy in tests/golden/dir_recipe_cases.json):

* mode, coupler matrix, density maximum and reference, donor knees, receiver
  references and knees and the spatial diffusion controls: exact f32 words in all 64
  cases, and the inactive cases' zero identities;
* the three compensated log-exposure axes: within 2.4e-7 (one f32 ulp at |x| in
  [2, 4)). The development curves are sampled here from the profiles' Gaussian density
  model with erfc in binary64, which differs from the reference's libm erfcf by at
  most 4 ulp; the axes inherit that, so their words and the hashes that cover them
  are not compared;
* the recipe identity, built as `DirRecipe` builds it from the fixture's own scalar
  words and axes hash, equals the fixture's identity."""
import json
import os

import numpy as np
import pytest


@pytest.fixture(scope="module")
def cases():
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dir_recipe_cases.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="module")
def dp():
    from film_juicer_b200 import dir_prep

    return dir_prep


def _f(a):
    return np.asarray(a, dtype=np.uint32).view(np.float32)


def _development(stock, prepare, dp):
    m = stock["model"]
    axis = np.asarray(stock["log_exposure"], dtype=np.float64).astype(np.float32)
    tot, _ = prepare.density_model_samples(m["centers"], m["amplitudes"], m["sigmas"], axis,
                                           stock["info"].get("type") == "positive")
    return (*dp.normalized_curves(tot), axis)


def _params(ct, dp):
    return dp.DirParams(
        active=ct["active"], amount=_f(ct["amount"])[0], inhibition_same_layer=_f(ct["inhibition"])[0],
        inhibition_interlayer=_f(ct["inhibition"])[1], diffusion_size_um=_f(ct["diffusion"])[0],
        diffusion_tail_um=_f(ct["diffusion"])[1], diffusion_tail_weight=_f(ct["diffusion"])[2],
        gamma_use_stock=ct["stock"], gamma_same_layer_rgb=tuple(_f(ct["same"])),
        gamma_interlayer_r_to_gb=tuple(_f(ct["red"])), gamma_interlayer_g_to_rb=tuple(_f(ct["green"])),
        gamma_interlayer_b_to_rg=tuple(_f(ct["blue"])), langmuir_donor_k_rgb=tuple(_f(ct["donor_k"])),
        langmuir_receiver_k_rgb=tuple(_f(ct["receiver_k"])))


def test_dir_recipes_against_reference(cases, dp, prepare):
    devs = {k: _development(s, prepare, dp) for k, s in cases["stocks"].items()}
    active = 0
    for c in cases["cases"]:
        stock = cases["stocks"][c["key"]]
        cn, lo, hi, ch, axis = devs[c["key"]]
        assert np.array_equal(hi.view(np.uint32), np.asarray(c["authored_maximum"], np.uint32))
        assert np.allclose(lo, _f(c["authored_minimum"]), rtol=1e-6, atol=0)
        r = dp.DirRecipe(cn, axis, stock["info"]["type"] == "positive", _params(c["controls"], dp),
                         dp.processing_defaults(stock["info"]), ch)
        o = c["dir"]
        assert r.mode == o["mode"] and bool(r.mode) == o["active"]
        for ours, theirs in (("matrix_rgb", "matrix"), ("density_max_rgb", "maximum"), ("density_ref_rgb", "reference"),
                             ("donor_k_rgb", "donor_k"), ("receiver_c_ref_rgb", "receiver_c_ref"),
                             ("receiver_kr_rgb", "receiver_kr"), ("diffusion", "diffusion")):
            got = np.ascontiguousarray(getattr(r, ours), np.float32).view(np.uint32).ravel()
            assert np.array_equal(got, np.asarray(o[theirs], np.uint32).ravel()), (c["key"], ours)
        if not r.mode:
            assert r.hash == o["hash"] == 0 and r.axes_hash == o["axes_hash"] == 0
            continue
        active += 1
        want = _f(o["axes"]).reshape(3, -1).astype(np.float64)
        assert float(np.abs(r.axes_rgb.astype(np.float64) - want).max()) <= 2.4e-7, c["key"]
    assert active == 32


def test_dir_identity_on_reference_words(cases, dp):
    """dir_prep.recipe_identity (film/dir.rs:324-359) on the fixture's own scalar words
    and axes hash equals the fixture's identity in every active case."""
    active = 0
    for c in cases["cases"]:
        o = c["dir"]
        if not o["active"]:
            continue
        active += 1
        positive = cases["stocks"][c["key"]]["info"]["type"] == "positive"
        ident = dp.recipe_identity(positive, _f(o["matrix"]), _f(o["maximum"]), _f(o["reference"]),
                                   _f(o["donor_k"]), _f(o["receiver_c_ref"]), _f(o["receiver_kr"]),
                                   o["axes_hash"], _f(o["diffusion"]))
        assert ident == o["hash"], c["key"]
    assert active == 32


def test_recipe_dir_is_the_reference_stock_recipe(cases, recipes):
    """The prepared recipes (kodak_portra_400) carry the reference's stock DIR recipe:
    matrix, density maximum and reference and donor knees equal the fixture's
    stock-controls case word for word, the axes within 2.4e-7."""
    want = [c for c in cases["cases"] if c["key"] == "kodak_portra_400" and c["controls"]["stock"]
            and c["controls"]["active"] and _f(c["controls"]["amount"])[0] == 1.0
            and tuple(_f(c["controls"]["inhibition"])) == (1.0, 1.0) and c["dir"]["active"]]
    assert want
    o = want[0]["dir"]
    for name in ("direct", "print"):
        s, a = recipes[name].scalars, recipes[name].arrays
        assert s["dir_mode"] == o["mode"] == 1
        for ours, theirs in (("dir_matrix_rgb", "matrix"), ("dir_dmax", "maximum"), ("dir_dref", "reference"),
                             ("dir_donor_k", "donor_k")):
            got = np.asarray(s[ours], np.float32).view(np.uint32).ravel()
            assert np.array_equal(got, np.asarray(o[theirs], np.uint32).ravel()), (name, ours)
        err = np.abs(a["dir_axes_rgb"].astype(np.float64) - _f(o["axes"]).reshape(3, -1))
        assert float(err.max()) <= 2.4e-7
