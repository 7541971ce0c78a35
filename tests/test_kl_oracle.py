"""The K-L random field restatement (oracle/kl_oracle.c) pinned to the
reference (CPP_17-1_K-L_expansion_non.cpp, CPP_17-2_K-L_expansion_corr.cpp).

The reference draws its standard normals from a time-seeded engine; its own
solve_wi / solve_ramdai / solve_h_2D / solve_h_3D are called here with
injected normals (oracle/ref_driver.cpp: ref_kl_field).  The golden fixtures
tests/golden/kl_*.npz hold those reference outputs (tests/golden/make_golden.py)
so that the check also runs where the reference tree is absent.  Every value
is compared bit for bit: roots, eigenvalues, their order, and the field.
"""
import glob
import os

import numpy as np
import pytest

import scenes
from checkers import have_reference, kl_correlate, kl_oracle, kl_reference

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "kl_*.npz")))


def _field_from(z):
    no, typ = (int(v) for v in z["field"])
    mean, sd, dep, *rl = (float(v) for v in z["field_vals"])
    return {"no": no, "type": typ, "mean": mean, "sd": sd, "coe_depth": dep, "rl": rl}


def _dom_from(z):
    return {"a": z["a"], "x_trans": z["x_trans"], "soil_max": float(z["soil_max"]),
            "water_max": float(z["water_max"])}


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_matches_reference_fixture(path):
    z = np.load(path)
    nd = int(z["ndim"])
    out, written, wi, eig, order = kl_oracle(nd, z["xp"], z["type"], _field_from(z), _dom_from(z), z["xi"])
    assert np.array_equal(wi[:, :nd], z["wi"])
    assert np.array_equal(eig, z["eigval"])
    assert np.array_equal(order[:, :nd], z["order"])
    ref = z["out"]
    assert np.array_equal(np.isnan(ref), written == 0)
    assert np.array_equal(out[written == 1], ref[written == 1])
    assert written.sum() > 0


def test_fixture_set_covers_both_dimensions_and_distributions():
    kinds = set()
    for p in FIXTURES:
        z = np.load(p)
        kinds.add((int(z["ndim"]), int(z["field"][1])))
    assert {(2, 1), (2, 2), (3, 1), (3, 2)} <= kinds


@pytest.mark.skipif(not have_reference(), reason="reference solver not built here")
@pytest.mark.parametrize("no,typ,dep", [(2, 2, 0.0), (3, 1, 0.01), (4, 1, 0.0)])
def test_oracle_matches_live_reference_2d(no, typ, dep):
    sc = scenes.dam_break_2d(dx=0.04, steps=10)
    sc.ptype[::7] = np.where(sc.ptype[::7] == 1, 2, sc.ptype[::7])   # some soil among the water
    dom = scenes.kl_domain(sc)
    field = {"no": no, "type": typ, "mean": 1.0e-4 if no == 2 else 0.3, "sd": 2.0e-5 if no == 2 else 0.03,
             "rl": [0.3, 0.2, 0.0], "coe_depth": dep}
    xi = np.random.default_rng(no * 10 + typ).standard_normal(200)
    out, written, wi, eig, order = kl_oracle(2, sc.xp, sc.ptype, field, dom, xi)
    ref, rwi, reig, rorder = kl_reference(2, sc.xp, sc.ptype, field, dom, xi)
    assert np.array_equal(wi[:, :2], rwi[:, :2]) and np.array_equal(eig, reig)
    assert np.array_equal(order[:, :2], rorder[:, :2])
    assert np.array_equal(np.isnan(ref), written == 0)
    assert np.array_equal(out[written == 1], ref[written == 1])


def test_domain_quirk_last_particle_not_maximum():
    """input_par's fmax(running min, x) leaves soil_max at the last soil
    particle's coordinate (CPP_2-initialf.cpp:961)."""
    sc = scenes.slope_2d(H=5.0, dx=0.1)
    dom = scenes.kl_domain(sc)
    soil = np.flatnonzero(sc.ptype == 2)
    assert dom["soil_max"] == sc.xp[soil[-1], 1]


def test_correlated_normals():
    """zeta = u (K x 2) [1, rho; 0, sqrt(1 - rho^2)] (CPP_17-2:120-168): the
    friction normals are u[:, 0], the cohesion normals rho u0 + sqrt(1-rho^2) u1."""
    u = np.random.default_rng(5).standard_normal((200, 2))
    a, b = kl_correlate(u, 0.5)
    assert np.array_equal(a, u[:, 0] * 1.0 + u[:, 1] * 0.0)
    assert np.array_equal(b, u[:, 0] * 0.5 + u[:, 1] * np.sqrt(1.0 - 0.25))
