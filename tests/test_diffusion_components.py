"""Diffusion component expansion (host code, no GPU): the library's
fjb_diffusion_components_host against the oracle's restatement of
rust/film-juicer-core/src/optics/diffusion_frame.rs:238-421, and its admission checks."""
import ctypes as C

import numpy as np
import pytest

from film_juicer_b200 import abi, load_library, descriptors
from oracle import optics


def _expand(d):
    lib = load_library()
    out = abi.FjDiffusionComponents()
    err = abi.ErrorText()
    st = lib.fjb_diffusion_components_host(C.byref(d), C.byref(out), C.byref(err.buf))
    return st, out, err.text


@pytest.mark.parametrize("family", [0, 1, 2, 3])
@pytest.mark.parametrize("warmth", [-1.5, -0.4, 0.0, 0.7, 1.5])
def test_components_match_restatement(family, warmth):
    d = descriptors.diffusion_record(2.5, 1920, family=family, warmth=warmth, group_weights=(0.5, 0.3, 0.2),
                                     group_lambda_um=(6.0, 30.0, 120.0), spatial_scale=1.3)
    st, out, text = _expand(d)
    assert st.category == abi.FJ_STATUS_SUCCESS, text
    lam, w = optics.diffusion_components(family, (0.5, 0.3, 0.2), (6.0, 30.0, 120.0), warmth, 1.3, d.pixel_size_um)
    np.testing.assert_array_equal(np.array(out.lambda_px), np.array(lam))
    for c, arr in enumerate((out.red_weights, out.green_weights, out.blue_weights)):
        np.testing.assert_allclose(np.array(arr), np.array(w[c]), rtol=1e-15, atol=0)


def test_extreme_warmth_clamps_and_renormalises():
    d = descriptors.diffusion_record(3.0, 3840, warmth=1.5)
    st, out, text = _expand(d)
    assert st.category == abi.FJ_STATUS_SUCCESS, text
    halo = slice(2, 5)
    for arr in (out.red_weights, out.green_weights, out.blue_weights):
        v = np.array(arr)[halo]
        assert np.all(v >= 0.0)
        assert abs(v.sum() - d.group_weights[1]) < 1e-12


@pytest.mark.parametrize("field,value", [("family", 4), ("warmth", 1.6), ("warmth", float("nan")),
                                         ("spatial_scale", 0.0), ("pixel_size_um", -1.0), ("radius_px", 0)])
def test_rejects_invalid_fields(field, value):
    d = descriptors.diffusion_record(2.5, 1920)
    setattr(d, field, value)
    st, _, text = _expand(d)
    assert st.category == abi.FJ_STATUS_PREPARATION_FAILURE
    assert text


def test_rejects_invalid_group_weights():
    d = descriptors.diffusion_record(2.5, 1920, group_weights=(0.0, 0.0, 0.0))
    assert _expand(d)[0].category == abi.FJ_STATUS_PREPARATION_FAILURE
    d = descriptors.diffusion_record(2.5, 1920, group_weights=(0.5, -0.1, 0.2))
    assert _expand(d)[0].category == abi.FJ_STATUS_PREPARATION_FAILURE
    d = descriptors.diffusion_record(2.5, 1920, group_lambda_um=(0.0, 30.0, 100.0))
    assert _expand(d)[0].category == abi.FJ_STATUS_PREPARATION_FAILURE


def _golden():
    import os

    from conftest import GOLDEN

    return np.load(os.path.join(GOLDEN, "diffusion_component_cases.npz"))


def _record(words):
    f = words.view(np.float64)
    d = abi.FjDiffusion()
    d.family = int(words[0])
    for i in range(3):
        d.group_weights[i] = float(f[1 + i])
        d.group_lambda_um[i] = float(f[4 + i])
    d.warmth, d.spatial_scale, d.pixel_size_um = float(f[7]), float(f[8]), float(f[9])
    d.radius_px = int(np.int64(words[10]))
    d.sample_hash = d.hash = int(words[11])
    return d


def test_components_golden_words():
    """All 159 component cases of the reference's characterization: the 36 binary64
    output words exactly, failures as preparation failures."""
    g = _golden()
    assert len(g["names"]) == 159
    for name, words, want, failed in zip(g["names"], g["words"], g["outputs"], g["failed"]):
        st, out, text = _expand(_record(words))
        if failed:
            assert st.category == abi.FJ_STATUS_PREPARATION_FAILURE, name
            continue
        assert st.category == abi.FJ_STATUS_SUCCESS, (name, text)
        got = np.concatenate([np.array(a, dtype=np.float64) for a in
                              (out.lambda_px, out.red_weights, out.green_weights, out.blue_weights)])
        np.testing.assert_array_equal(got.view(np.uint64), want, err_msg=str(name))


def test_oracle_components_golden_words():
    """The oracle's pure-Python restatement against the same words (successful cases)."""
    g = _golden()
    for name, words, want, failed in zip(g["names"], g["words"], g["outputs"], g["failed"]):
        if failed:
            continue
        d = _record(words)
        lam, w = optics.diffusion_components(d.family, list(d.group_weights), list(d.group_lambda_um), d.warmth,
                                             d.spatial_scale, d.pixel_size_um)
        got = np.array(lam + w[0] + w[1] + w[2], dtype=np.float64)
        np.testing.assert_array_equal(got.view(np.uint64), want, err_msg=str(name))
