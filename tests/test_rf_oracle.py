"""The correlation-matrix random field (nonstationary_random_2D / _3D,
CPP_17-3-Nonstationary-RF.cpp; flspv 3): the oracle's restatement against the
reference's own routine, with the cell normals injected in place of its
time-seeded generator -- from the committed fixtures made by the reference
(tests/golden/make_golden.py RF_CASES) and, where the reference is built
here, live.  Both run the same FP64 operations in the same order with one
thread, so the fields must be bit-identical."""
import os

import numpy as np
import pytest

import make_golden
import scenes
from checkers import have_reference, rf_oracle, rf_reference

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
