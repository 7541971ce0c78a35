"""The engine's K-L random fields (sphgpu_kl_generate / _corr) against the
reference's own output (golden fixtures made by the reference with injected
normals) and the oracle.

The roots, eigenvalues and their order are formed exactly as the reference
forms them; the per-particle eigenfunctions call the device's cos / sin, which
may differ from the C library's by an ulp, so fields are held to KL_REL_TOL
relative to their magnitude.  A field then enters the step through the
material records: an oracle given the engine's field values steps bit for bit
with the engine.
"""
import glob
import os

import numpy as np
import pytest

import scenes
import sphgpu
from checkers import ORC_JACOBI, ORC_POW_CR, STATE_FIELDS, Oracle, kl_correlate, kl_oracle

pytestmark = pytest.mark.gpu

KL_REL_TOL = 1e-12
HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "kl_*.npz")))
SCENE_OF = {"slope_2d": lambda: scenes.slope_2d(H=5.0, dx=0.1),
            "column_3d": lambda: scenes.soil_column_3d(dx=0.05, steps=100)}


def _scene_for(name):
    for k, f in SCENE_OF.items():
        if k in name:
            return f()
    raise KeyError(name)


def _engine(sc):
    st = scenes.initialise(sc)
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    return st, eng


def _domain(sc):
    dom = scenes.kl_domain(sc)
    return dom, sphgpu.kl_domain(dom["nb_min"], dom["nb_max"], dom["soil_max"], dom["water_max"])


def _close(a, b, tol=KL_REL_TOL):
    assert np.array_equal(np.isnan(a), np.isnan(b))
    m = ~np.isnan(b)
    scale = np.abs(b[m]).max()
    err = np.abs(a[m] - b[m]).max() / scale
    assert err <= tol, err
    return err


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_field_matches_reference(path):
    z = np.load(path)
    sc = _scene_for(os.path.basename(path))
    assert np.array_equal(sc.xp, z["xp"]) and np.array_equal(sc.ptype, z["type"])
    no, typ = (int(v) for v in z["field"])
    mean, sd, dep, *rl = (float(v) for v in z["field_vals"])
    _, eng = _engine(sc)
    _, d = _domain(sc)
    got = eng.kl_generate(d, [sphgpu.kl_field(no, typ, mean, sd, rl, dep)], z["xi"][None, :])[0]
    err = _close(got, z["out"])
    print(os.path.basename(path), "max relative error", err)


def test_fields_enter_the_step():
    """Cohesion and friction fields on the slope, then steps: an oracle given
    the engine's material values is bit-identical to the engine."""
    sc = scenes.slope_2d(H=5.0, dx=0.1)
    st, eng = _engine(sc)
    _, d = _domain(sc)
    rng = np.random.default_rng(9)
    xi = rng.standard_normal((2, 200))
    fields = [sphgpu.kl_field(1, 2, 10.0e3, 3.0e3, [10.0, 1.0]), sphgpu.kl_field(0, 1, 25.0, 2.0, [8.0, 2.0], 0.3)]
    vals = eng.kl_generate(d, fields, xi)
    soil = st.soil.copy()
    m_c, m_f = ~np.isnan(vals[0]), ~np.isnan(vals[1])
    soil["c"][m_c] = vals[0][m_c]
    soil["fai"][m_f] = vals[1][m_f]
    orc = Oracle(st.params, ORC_JACOBI, ORC_POW_CR)
    orc.load_state(st.fields, st.fluid, soil)
    eng.step(10)
    assert orc.step(10) == 0
    for k in STATE_FIELDS:
        a, b = eng.get_field(k), orc.get_field(k)
        assert np.array_equal(a, b) or np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(
            a[~np.isnan(a)], b[~np.isnan(b)]), k


def test_correlated_pair_matches_oracle():
    sc = scenes.slope_2d(H=5.0, dx=0.1)
    st, eng = _engine(sc)
    dom, d = _domain(sc)
    u2 = np.random.default_rng(12).standard_normal((200, 2))
    fai = {"no": 0, "type": 2, "mean": 25.0, "sd": 2.5, "rl": [10.0, 1.0, 0.0], "coe_depth": 0.0}
    coh = {"no": 1, "type": 2, "mean": 10.0e3, "sd": 3.0e3, "rl": [10.0, 1.0, 0.0], "coe_depth": 0.0}
    rho = -0.5
    got = eng.kl_generate_corr(d, sphgpu.kl_field(0, 2, 25.0, 2.5, [10.0, 1.0]),
                               sphgpu.kl_field(1, 2, 10.0e3, 3.0e3, [10.0, 1.0]), rho, u2)
    # the correlation coefficient of the underlying normals (CPP_17-2:123-129)
    c = np.log(1.0 + rho * (2.5 / 25.0) * (3.0e3 / 10.0e3))
    c = c / np.sqrt(np.log(1.0 + 2.5 * 2.5 / 25.0 / 25.0) * np.log(1.0 + 3.0e3 * 3.0e3 / 10.0e3 / 10.0e3))
    xa, xb = kl_correlate(u2, c)
    ra = kl_oracle(2, sc.xp, sc.ptype, fai, dom, xa)[0]
    rb = kl_oracle(2, sc.xp, sc.ptype, coh, dom, xb)[0]
    _close(got[0], ra)
    _close(got[1], rb)


def test_error_codes():
    sc = scenes.slope_2d(H=5.0, dx=0.1)
    _, eng = _engine(sc)
    dom, d = _domain(sc)
    with pytest.raises(sphgpu.SPHError) as e:
        eng.kl_generate(d, [sphgpu.kl_field(1, 3, 10.0, 1.0, [1.0, 1.0])], np.zeros((1, 200)))
    assert e.value.code == 14
    flat = sphgpu.kl_domain([0.0, 1.0, 0.0], [0.0, 2.0, 0.0], 1.0, 1.0)
    with pytest.raises(sphgpu.SPHError) as e:
        eng.kl_generate(flat, [sphgpu.kl_field(1, 1, 10.0, 1.0, [1.0, 1.0])], np.zeros((1, 200)))
    assert e.value.code == 13
