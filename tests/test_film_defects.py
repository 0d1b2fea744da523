"""Film and gate defects on the CPU: the oracle's restatement on the reference's
composed effects records (tests/golden/effects_cases.json), properties of the defect
identity hashing, and the product's record validation (which rejects a malformed
record before any device work, so it runs without a GPU)."""
import ctypes as C

import numpy as np
import pytest


def planes(h, w, seed=1):
    rng = np.random.default_rng(seed)
    return [rng.uniform(0.2, 2.0, (h, w)).astype(np.float32) for _ in range(3)]


@pytest.mark.parametrize("case", [0, 18, 20, 25])
def test_oracle_defects_are_bounded_and_visible(oracle, effects_case, case):
    e = effects_case(case)
    w, h = e.render_extent.width, e.render_extent.height
    base = planes(h, w)
    out, dust = oracle.film_defects(e, base)
    assert dust is not None and np.all((dust >= 0.0) & (dust <= 1.0))
    assert float(dust.min()) < 0.999
    ratio = out[0] / base[0]
    assert np.all((ratio >= 0.0) & (ratio <= 1.0 + 1e-7))
    assert np.allclose(out[1] / base[1], ratio, rtol=1e-6) and np.allclose(out[2] / base[2], ratio, rtol=1e-6)
    mask = oracle.gate_mask(e)
    assert mask.shape == (e.gate_height, e.gate_width)
    assert np.all((mask >= 0.0) & (mask <= 1.0)) and float(mask.min()) < 0.999
    again, dust2 = oracle.film_defects(e, base)
    assert np.array_equal(dust, dust2) and all(np.array_equal(a, b) for a, b in zip(out, again))


def test_oracle_clip_token_moves_film_defects_only(oracle, effects_case):
    # the film families hash the clip token, the gate families do not
    # (src/Cuda/Scan/JuicerCudaScanPipeline.cu:875-883)
    e = effects_case(0)
    f = effects_case(0)
    f.clip_token = e.clip_token ^ 0x5A5A
    w, h = e.render_extent.width, e.render_extent.height
    base = planes(h, w)
    _, dust_e = oracle.film_defects(e, base)
    _, dust_f = oracle.film_defects(f, base)
    assert not np.array_equal(dust_e, dust_f)
    assert np.array_equal(oracle.gate_mask(e), oracle.gate_mask(f))


def test_oracle_zero_probability_is_identity(oracle, effects_case):
    e = effects_case(0, slots=(0.0, 0.0, 0.0, 0.0))
    w, h = e.render_extent.width, e.render_extent.height
    base = planes(h, w)
    out, dust = oracle.film_defects(e, base)
    assert dust is None
    assert all(np.array_equal(a, b) for a, b in zip(out, base))
    assert np.all(oracle.gate_mask(e) == 1.0)


def _reject(effects):
    import film_juicer_b200 as pkg
    from film_juicer_b200 import abi

    lib = pkg.load_library()
    err = abi.ErrorText()
    dummy = C.c_void_p(16)  # never dereferenced: validation fails first
    st = lib.fjb_film_defects(C.byref(effects), 8, 8, dummy, dummy, dummy, dummy, None, 0, None, C.byref(err.buf))
    return st.category, err.text


def test_product_rejects_malformed_records(effects_case):
    from film_juicer_b200 import abi

    e = effects_case(0)
    e.flags |= 64
    cat, why = _reject(e)
    assert cat == abi.FJ_STATUS_PREPARATION_FAILURE and "flags" in why
    e = abi.FjFilmEffects()
    e.hash = 7  # inactive but carries an identity
    cat, why = _reject(e)
    assert cat == abi.FJ_STATUS_PREPARATION_FAILURE and "inactive" in why
    e = effects_case(0)
    e.hash = 0
    cat, why = _reject(e)
    assert cat == abi.FJ_STATUS_PREPARATION_FAILURE and "identity" in why
    e = effects_case(0)
    e.film_dust.cell_width_mm = 1e-7  # an enormous cell range per tile
    cat, why = _reject(e)
    assert cat == abi.FJ_STATUS_PREPARATION_FAILURE and "too many" in why
    e = effects_case(0)
    e.sample_step_x_mm = float("nan")
    cat, why = _reject(e)
    assert cat == abi.FJ_STATUS_PREPARATION_FAILURE and "finite" in why
    e = effects_case(0)
    e.gate_width = 0
    lib_err = abi.ErrorText()
    import film_juicer_b200 as pkg

    st = pkg.load_library().fjb_gate_mask(C.byref(e), C.c_void_p(16), 0, 0, None, 0, None, C.byref(lib_err.buf))
    assert st.category == abi.FJ_STATUS_PREPARATION_FAILURE and "grid" in lib_err.text


def test_particle_tables_cover_the_frame(effects_case):
    # the table sizes follow the frame's cell range: non-zero for active families, zero
    # for a record with every family off
    import film_juicer_b200 as pkg

    lib = pkg.load_library()
    e = effects_case(0)
    film = lib.fjb_film_defects_scratch_bytes(C.byref(e), 64, 48)
    gate = lib.fjb_gate_mask_scratch_bytes(C.byref(e), e.gate_width, e.gate_height)
    assert film > 0 and gate > 0 and film % 256 == 0
    off = effects_case(0, slots=(0.0, 0.0, 0.0, 0.0))
    assert lib.fjb_film_defects_scratch_bytes(C.byref(off), 64, 48) == 0
    # this record's 0.56 mm sample step over 3840 x 2160 pixels spans more cells than a
    # table holds: no table, the tiles build their own candidates
    assert lib.fjb_film_defects_scratch_bytes(C.byref(e), 3840, 2160) == 0
