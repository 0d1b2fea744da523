"""Print preparation (film_juicer_b200.print_prep) against the reference's print
characterizations (tests/print/{balance,preflash,illuminant}-fixtures, linux-release
native profile; compact copy in tests/golden/print_cases.npz):

* the filtered illuminant of all 127 literal cases word for word (C library erff), and
  the same rejections; against the Rust build's libm erff the words differ in at most
  2 samples by at most 6 ulp, as the reference's own fixtures record;
* the preflash raw integral of all 19 cases word for word, and the same rejections;
* the print balance of the 42 characterization cases and the 60 product records:
  raw R, G, B words, the two mid-grey factors, the normaliser, the illuminant hash and
  the balance hash, and the same rejections with the same diagnostic field;
* the TH-KG3 enlarger lamp built from the KG3 transmission rows, filtered by each
  product record's main and preflash C, M, Y, reproduces the products' illuminant
  words exactly."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def cases():
    import os

    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "print_cases.npz"))


@pytest.fixture(scope="module")
def pp():
    from film_juicer_b200 import print_prep

    return print_prep


def _f(a):
    return np.asarray(a, dtype=np.uint32).view(np.float32)


def test_filtered_illuminant_words(cases, pp):
    n = len(cases["illum_id"])
    assert n == 127
    rust_words = []
    for i in range(n):
        args = (_f(cases["illum_cmy_cc"][i]), _f(cases["illum_source"][i]), _f(cases["illum_edges_nm"][i]),
                _f(cases["illum_transitions_nm"][i]))
        if not cases["illum_success"][i]:
            with pytest.raises(pp.PrintPrepError) as e:
                pp.filtered_illuminant(*args)
            assert e.value.field == "filtered_print_illuminant"
            continue
        got = pp.filtered_illuminant(*args).view(np.uint32)
        assert np.array_equal(got, cases["illum_samples"][i]), cases["illum_id"][i]
        rust = cases["illum_rust_samples"][i]
        diff = np.nonzero(got != rust)[0]
        rust_words.append(len(diff))
        if len(diff):
            ulp = np.abs(got[diff].astype(np.int64) - rust[diff].astype(np.int64))
            assert int(ulp.max()) <= 6
    assert sum(rust_words) <= 2


def test_preflash_raw_words(cases, pp):
    n = len(cases["preflash_id"])
    assert n == 19
    for i in range(n):
        args = (_f(cases["preflash_film_base_density"][i]), _f(cases["preflash_filtered_illuminant"][i]),
                _f(cases["preflash_sensitivity_cmy"][i]))
        if not cases["preflash_success"][i]:
            with pytest.raises(pp.PrintPrepError) as e:
                pp.preflash_raw(*args)
            assert e.value.field == "preflash_raw"
            continue
        got = pp.preflash_raw(*args).view(np.uint32)
        assert np.array_equal(got, cases["preflash_raw"][i]), cases["preflash_id"][i]


def test_balance_words_and_hashes(cases, pp):
    n = len(cases["balance_id"])
    assert n == 102
    failures = 0
    for i in range(n):
        args = (_f(cases["balance_baseline_density_cmy"][i]), _f(cases["balance_compensated_density_cmy"][i]),
                int(cases["balance_reference_hash"][i]), int(cases["balance_mode"][i]),
                _f(cases["balance_film_base_density"][i]), _f(cases["balance_film_channel_density_cmy"][i]),
                _f(cases["balance_print_sensitivity_rgb"][i]), _f(cases["balance_filtered_main_illuminant"][i]))
        if not cases["balance_success"][i]:
            failures += 1
            with pytest.raises(pp.PrintPrepError) as e:
                pp.Balance(*args)
            assert e.value.field == str(cases["balance_field"][i]), cases["balance_id"][i]
            continue
        b = pp.Balance(*args)
        assert np.array_equal(b.baseline_raw_rgb.view(np.uint32), cases["balance_baseline_raw"][i])
        assert np.array_equal(b.compensated_raw_rgb.view(np.uint32), cases["balance_compensated_raw"][i])
        assert [pp.f32_bits(v) for v in b.scalars] == list(cases["balance_scalars"][i]), cases["balance_id"][i]
        assert b.filtered_main_illuminant_hash == int(cases["balance_illuminant_hash"][i])
        assert b.hash == int(cases["balance_hash"][i]), cases["balance_id"][i]
    assert failures == 20


def test_enlarger_lamp_and_product_illuminants(cases, pp):
    lamp = pp.tungsten_kg3(pp.parse_csv_rows(str(cases["kg3_csv"])))
    assert abs(float(np.mean(lamp.astype(np.float64))) - 1.0) < 1e-6
    for i in range(len(cases["product_main"])):
        main = pp.filtered_illuminant(_f(cases["product_main_cmy"][i]), lamp)
        assert np.array_equal(main.view(np.uint32), cases["product_main"][i]), i
        if cases["product_preflash"][i].any():  # records with a preflash illuminant
            pre = pp.filtered_illuminant(_f(cases["product_preflash_cmy"][i]), lamp)
            assert np.array_equal(pre.view(np.uint32), cases["product_preflash"][i]), i


def test_filters_and_hash_helpers(pp):
    main, pre = pp.filters((0.0, 65.0, 55.0), ui_ymc_cc=(1.0, 2.0, 3.0), preflash_m_cc=4.0, preflash_y_cc=5.0)
    assert [float(v) for v in main] == [3.0, 67.0, 56.0]
    assert [float(v) for v in pre] == [0.0, 69.0, 60.0]
    assert pp.normalization_mode(True, True) == 3 and pp.normalization_mode(False, True) == 1
    assert pp.hash_finite_f32s([0.0]) == pp.hash_finite_f32s([-0.0])
    assert pp.hash_finite_f32s([1.0, np.nan]) is None
    assert pp.hash_u64s([]) == pp.FNV_OFFSET
    assert pp.f32_bits(pp.f32_from_decimal("0.1")) == 0x3DCCCCCD


def test_print_recipe_tables_are_the_reference_products(cases, pp, recipes):
    """kodak_portra_400 -> kodak_portra_endura (tests/golden/recipe_print.npz): the print
    tables film_juicer_b200.prepare builds are the ones in the reference's balance
    product records word for word (film base and dye densities, the paper's linear
    sensitivity, the filtered TH-KG3 main illuminant at the calibrated neutral), the
    balance of a product's reference densities on them is the product's balance word
    for word, and the recipe's own normaliser (a metered grey at log exposure 0) is
    within 2e-4 of that of the products at 0 EV whose reference densities lie within
    2e-4 of the recipe's (the other products differ in reconstruction or
    development settings)."""
    rec = recipes["print"]
    w = lambda a: np.ascontiguousarray(np.asarray(a, np.float32)).reshape(-1).view(np.uint32)  # noqa: E731
    fields = (("film_base_density", "print_film_base_density"), ("film_channel_density_cmy", "print_film_density_cmy"),
              ("print_sensitivity_rgb", "print_sensitivity_cmy"), ("filtered_main_illuminant", "print_main_illuminant"))
    match = [i for i in range(len(cases["balance_id"]))
             if cases["balance_success"][i] and int(cases["balance_mode"][i]) == 3
             and all(np.array_equal(cases[f"balance_{k}"][i], w(rec.arrays[r])) for k, r in fields)]
    assert len(match) >= 10
    assert [float(v) for v in rec.scalars["print_main_cc_cmy"]] == [float(v) for v in _f(cases["product_main_cmy"][0])]
    checked = 0
    for i in match:
        b = pp.Balance(_f(cases["balance_baseline_density_cmy"][i]), _f(cases["balance_compensated_density_cmy"][i]),
                       int(cases["balance_reference_hash"][i]), 3, rec.arrays["print_film_base_density"],
                       rec.arrays["print_film_density_cmy"], rec.arrays["print_sensitivity_cmy"],
                       rec.arrays["print_main_illuminant"])
        assert [pp.f32_bits(v) for v in b.scalars] == list(cases["balance_scalars"][i])
        assert b.hash == int(cases["balance_hash"][i])
        ours = np.asarray(rec.scalars["print_reference_density_cmy"][0])
        theirs = _f(cases["balance_baseline_density_cmy"][i]).astype(np.float64)
        if (np.array_equal(cases["balance_baseline_density_cmy"][i], cases["balance_compensated_density_cmy"][i])
                and np.abs(ours - theirs).max() <= 2e-4):
            checked += 1  # a product at 0 EV on the recipe's own reference densities
            ref = float(_f(cases["balance_scalars"][i])[2])
            assert abs(rec.scalars["print_normalizer"] - ref) <= 2e-4 * ref
    assert checked >= 4


def test_enlarger_lamp_choice(pp):
    assert pp.enlarger_illuminant() == "TH-KG3"
    assert pp.enlarger_illuminant(4) == "TH-KG3-L" and pp.enlarger_illuminant(0) == "D65"
    assert pp.enlarger_illuminant(99) == "TH-KG3"
