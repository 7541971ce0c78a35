"""The correlation-matrix random fields (nonstationary_random_2D / _3D,
CPP_17-3-Nonstationary-RF.cpp, flspv 3; nonstationary_correlated_random_2D /
_3D and random_variable_generate, CPP_17-5-Nonstationary-Correlated-RF.cpp,
flspv 4 and 5): the oracle's restatement against the reference's own
routines, with the normals injected in place of its time-seeded generator --
from the committed fixtures made by the reference (tests/golden/make_golden.py
RF_CASES, RF_CORR_CASES, RV_CASES) and, where the reference is built here,
live.  Both run the same FP64 operations in the same order with one thread, so
the fields must be bit-identical."""
import os

import numpy as np
import pytest

import make_golden
import scenes
from checkers import (have_reference, rf_oracle, rf_oracle_corr, rf_reference, rf_reference_corr, rv_oracle,
                      rv_reference)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _same(a, b):
    return bool(((a == b) | (np.isnan(a) & np.isnan(b))).all())


@pytest.mark.parametrize("name", list(make_golden.RF_CASES))
def test_rf_oracle_matches_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    field = make_golden.RF_CASES[name][1]
    dom = {"nb_min": g["nb_min"], "nb_max": g["nb_max"], "soil_max": float(g["soil_max"]),
           "water_max": float(g["water_max"])}
    err, out, ncell = rf_oracle(int(g["ndim"]), g["xp"], g["type"], float(g["dr"]), field, dom, g["zeta"])
    assert err == 0 and ncell == len(g["zeta"])
    assert _same(out, g["out"])
    assert np.isfinite(out).sum() > 100


@pytest.mark.skipif(not have_reference(), reason="reference not built here (oracle/_ref)")
def test_rf_error_codes_match_reference():
    """41: cells of a tenth of a spacing make 15,000 cells or more; 42: cells
    of ten spacings hold more than 39 particles."""
    sc = scenes.slope_2d(H=5.0, dx=0.1)
    dom = scenes.kl_domain(sc)
    base = {"no": 1, "type": 1, "mean": 1.0, "sd": 0.1, "rl": [1.0, 1.0, 0.0], "flag_auto": 1}
    for ndx, code in ((0.5, 41), (10.0, 42)):
        f = dict(base, cell_ndx=ndx)
        z = np.zeros(20000)
        assert rf_oracle(2, sc.xp, sc.ptype, sc.dr, f, dom, z)[0] == code
        assert rf_reference(2, sc.xp, sc.ptype, sc.dr, f, dom, z)[0] == code


def _dom(g):
    return {"nb_min": g["nb_min"], "nb_max": g["nb_max"], "soil_max": float(g["soil_max"]),
            "water_max": float(g["water_max"])}


@pytest.mark.parametrize("name", list(make_golden.RF_CORR_CASES))
def test_rf_corr_oracle_matches_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    _, pair, coe, _ = make_golden.RF_CORR_CASES[name]
    err, out, ncell = rf_oracle_corr(int(g["ndim"]), g["xp"], g["type"], float(g["dr"]), pair, coe, _dom(g), g["u2"])
    assert err == 0 and ncell == len(g["u2"])
    assert _same(out, g["out"])
    assert (np.isfinite(out).sum(axis=1) > 100).all()
    # the two members are correlated, not copies
    both = np.isfinite(out[0]) & np.isfinite(out[1])
    assert both.sum() > 100 and not np.allclose(out[0][both] / out[0][both].mean(), out[1][both] / out[1][both].mean())


@pytest.mark.parametrize("name", list(make_golden.RV_CASES))
def test_rv_oracle_matches_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    _, pair, coe, _ = make_golden.RV_CASES[name]
    out = rv_oracle(g["type"], pair, coe, g["u2"])
    assert _same(out, g["out"])
    assert np.isfinite(out).sum() > 0


@pytest.mark.skipif(not have_reference(), reason="reference not built here (oracle/_ref)")
def test_rf_corr_live_and_error_codes():
    """A fresh correlated field and the 41 / 42 codes against the reference."""
    sc = scenes.slope_2d(H=5.0, dx=0.1)
    dom = scenes.kl_domain(sc)
    _, pair, coe, _ = make_golden.RF_CORR_CASES["rfc_slope_2d_soil_lognormal"]
    u2 = np.random.default_rng(5).standard_normal((15000, 2))
    e0, a, nc = rf_oracle_corr(2, sc.xp, sc.ptype, sc.dr, pair, coe, dom, u2)
    e1, b = rf_reference_corr(2, sc.xp, sc.ptype, sc.dr, pair, coe, dom, u2[:nc])
    assert e0 == e1 == 0 and _same(a, b)
    for ndx, code in ((0.5, 41), (10.0, 42)):
        p = (dict(pair[0], cell_ndx=ndx), pair[1])
        assert rf_oracle_corr(2, sc.xp, sc.ptype, sc.dr, p, coe, dom, u2)[0] == code
        assert rf_reference_corr(2, sc.xp, sc.ptype, sc.dr, p, coe, dom, u2)[0] == code
