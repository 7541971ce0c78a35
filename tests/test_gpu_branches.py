"""GPU engine vs the oracle on the branches of the step the other parity tests
do not reach, and on the 2-D dam break at its full stated size.

Each case is one of the golden cases of tests/golden/make_golden.py: the
oracle's run of it is bit-identical to the reference's (tests/test_oracle.py),
so engine == oracle here means engine == reference up to the libm functions
named per case.

* three phases (fla 1): pore air (type 3) with the air equation of state as
  the reference writes it (CPP_7-1-eos_CR.cpp:34), fluid_acceleration_air
  (CPP_9-4-derivation_stress.cpp:98) and the soil-air drag of interact1
  (CPP_10-interact1.cpp:74-91), with unsaturated Cam-clay soil;
* the minor momentum forms of water and air (acc_type 1,
  CPP_9-4-derivation_stress.cpp:183, 268);
* a Bingham water (bhtype 1, CPP_7-2-constitutive.cpp:40-48);
* moving walls (if_move 1, CPP_11-xsph.cpp:61-84, CPP_12-1-update.cpp:38-47);
* a geostatic stage (inip > 0) crossing l == inip: elastic stresses before it
  (CPP_7-2-constitutive.cpp:104-115), soil_damping_geostress
  (CPP_9-4-derivation_stress.cpp:850-897), the strain reset
  (CPP_7-1-strain.cpp:35-39) and the displacement restart
  (CPP_12-1-update.cpp:19-28), with Drucker-Prager soil (cd = 0) and with
  Cam-clay under TSSMP (cd > 0) and regularisation every 4 steps;
* rainfall (flr 1): three rows of rain particles released on the device every
  lp steps (rainpro, CPP_15-1-rain.cpp:43-85) and a water particle taken out
  past the domain's left end (partidel, CPP_15-2-partidel.cpp:19-58);
* the 3-D rainfall slope, reduced: soil with co-located pore air (fla 1),
  rain rows over the crest falling as water onto it, Darcy drag between all
  three phases.
"""
import numpy as np
import pytest

import make_golden
import scenes
import sphgpu
from checkers import ORC_JACOBI, ORC_POW_CR, STATE_FIELDS, Oracle

pytestmark = pytest.mark.gpu

# tolerance relative to each field's magnitude: 0 = bit-identical.  The
# unsaturated Cam-clay (pow in its hardening term, tan / exp / log in the
# suction), the Bingham viscosity (tan of the friction angle) and subloading
# Cam-clay (log of p0 / p) call double-precision functions whose CUDA and C
# library results may differ in the last bit.
CASES = {
    "three_phase_column_3d_dx0.1_unsat": 1e-12,
    "three_phase_column_3d_dx0.1_minor": 0.0,
    "dam_break_2d_dx0.04_minor": 0.0,
    "dam_break_2d_dx0.04_bingham": 1e-12,
    "dam_break_2d_dx0.04_moving_wall": 0.0,
    "soil_column_3d_dx0.1_moving_wall": 0.0,
    "soil_column_3d_dx0.1_geostatic": 0.0,
    "soil_column_3d_dx0.1_geostatic_camclay": 1e-12,
    "slope_2d_H1_dx0.05_geostatic": 0.0,
    "dam_break_2d_dx0.04_rain": 0.0,
    "rain_slope_3d_dx0.25": 0.0,
}
RATIO_FIELDS = {"divr"}


def _compare(eng, orc, tol):
    worst = 0.0
    for name in STATE_FIELDS:
        a, b = eng.get_field(name), orc.get_field(name)
        if a.dtype.kind != "f":
            assert np.array_equal(a, b), name
            continue
        nan_a, nan_b = np.isnan(a), np.isnan(b)
        assert np.array_equal(nan_a, nan_b), name
        if tol == 0.0:
            same = (a == b) | (nan_a & nan_b)
            assert same.all(), (name, int((~same).sum()))
            continue
        if name in RATIO_FIELDS or not b.size:
            continue
        scale = max(float(np.nanmax(np.abs(b))), 1e-300)
        err = float(np.nanmax(np.abs(a - b))) / scale
        worst = max(worst, err)
        assert err <= tol, (name, err)
    return worst


@pytest.mark.parametrize("name", list(CASES))
def test_branch_against_oracle(name):
    factory, steps = make_golden.CASES[name]
    st = scenes.initialise(factory())
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil, st.rain)
    orc = Oracle(st.params, ORC_JACOBI, ORC_POW_CR)
    orc.load_state(st.fields, st.fluid, st.soil, st.rain)
    for chunk in (1, steps - 1):
        eng.step(chunk)
        assert orc.step(chunk) == 0
    assert eng.step_index == orc.step_index
    if st.rain is not None:
        assert eng.rain()["nrain"] == orc.rain()["nrain"] == 0
    worst = _compare(eng, orc, CASES[name])
    print(f"{name}: worst relative error {worst:.3g}")
    n1, i1 = eng.nnps()
    err, n2, i2, _ = orc.nnps()
    assert err == 0 and np.array_equal(n1, n2)
    mask = np.arange(100)[None, :] <= np.minimum(n1, 99)[:, None]
    mask[:, 0] = False
    assert np.array_equal(np.where(mask, i1, 0), np.where(mask, i2[:, :100], 0))
    eng.close()


def test_dam_break_full_size_2000_steps():
    """The 2-D dam break at its stated size (dx = 5 mm: 12,800 water and 2,178
    wall particles) for its full 2,000 steps: every field bit-identical to the
    oracle, and the neighbour lists of the last step identical."""
    st = scenes.initialise(scenes.dam_break_2d(dx=0.005, steps=2000))
    assert int((st.fields["type"] == 1).sum()) == 12800
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    orc = Oracle(st.params, ORC_JACOBI, ORC_POW_CR)
    orc.load_state(st.fields, st.fluid, st.soil)
    for chunk in (1, 999, 1000):
        eng.step(chunk)
        assert orc.step(chunk) == 0
    assert eng.step_index == orc.step_index == 2001
    _compare(eng, orc, 0.0)
    n1, i1 = eng.nnps()
    err, n2, i2, _ = orc.nnps()
    assert err == 0 and np.array_equal(n1, n2)
    x = eng.get_field("xp")
    water = st.fields["type"] == 1
    assert x[water, 0].max() > 1.0          # the front has run most of the tank
    eng.close()
