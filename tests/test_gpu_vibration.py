"""Vibration loading (flv 1 and 2) on the GPU engine against the oracle, whose
run of each case is bit-identical to the reference's own
(tests/test_oracle.py, fixtures of tests/golden/make_golden.py).

The cases shake a Drucker-Prager block through its floor: with flv 1 the
floor walls (matype 3, and matype 5 under the free-field columns and at the
sides) take the load of the step's time as their acceleration
(vibration_acceleration, CPP_9-1-acceleration_vibration.cpp:10-78), with flv 2
the walls of matype 4 and 5 take it as their velocity (vibration_velocity,
:80-160).  The load table holds an entry of 1500 (the reference's cut-off,
which zeroes the walls' interf and interfss) and a window that starts after
step 2 and ends at step 30.  Soil and structure are damped by
soil_damping_vibration (:162-224, from the largest diagonal entry of the
constitutive matrix of the step); the soil feels the free-field columns
(matype 52, CPP_19-FreeFieldParticles_soil.cpp) and the walls of matype 5
(CPP_19-FreeFieldParticles.cpp, whose elastic constants are the reference's
default-constructed pFFBound).  No double-precision library function enters
these terms beyond sqrt, so every field must be bit-identical, compared
after several chunks so that states inside and outside the load window are
both checked.
"""
import os
import tempfile

import numpy as np
import pytest

import make_golden
import scenes
import sphgpu
from checkers import ORC_JACOBI, ORC_POW_CR, STATE_FIELDS, Oracle

pytestmark = pytest.mark.gpu

CASES = ["shaking_box_2d_flv1", "shaking_box_2d_flv2", "shaking_box_3d_flv1", "shaking_box_3d_flv2"]


def _same_all(eng, orc):
    for name in STATE_FIELDS:
        a, b = eng.get_field(name), orc.get_field(name)
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        assert same.all(), (name, int((~same).sum()))


def _pair(name):
    factory, steps = make_golden.CASES[name]
    st = scenes.initialise(factory())
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil, vibration=st.vibration)
    orc = Oracle(st.params, ORC_JACOBI, ORC_POW_CR)
    orc.load_state(st.fields, st.fluid, st.soil, vibration=st.vibration)
    return st, steps, eng, orc


@pytest.mark.parametrize("name", CASES)
def test_vibration_against_oracle(name):
    st, steps, eng, orc = _pair(name)
    walls = st.fields["type"] == 0
    moved = False
    done = 0
    for chunk in (1, 4, 5, 9, steps - 19):
        eng.step(chunk)
        assert orc.step(chunk) == 0
        done += chunk
        _same_all(eng, orc)
        moved |= bool(np.abs(eng.get_field("interfss")[walls]).max() > 0.0)
    assert done == steps and moved
    n1, i1 = eng.nnps()
    err, n2, i2, _ = orc.nnps()
    assert err == 0 and np.array_equal(n1, n2)
    eng.close()


def test_vibration_checkpoint_restart():
    """A checkpoint inside the load window keeps the table and the stiffness
    the damping reads: the restarted run equals the uninterrupted one."""
    st, steps, eng, orc = _pair("shaking_box_2d_flv1")
    eng.step(10)
    path = os.path.join(tempfile.mkdtemp(), "vib.ck")
    eng.checkpoint_save(path)
    eng.step(12)
    want = {k: eng.get_field(k) for k in STATE_FIELDS}
    eng.close()
    two = sphgpu.Engine(st.params, device=0)
    two.checkpoint_load(path)
    two.step(12)
    for k in STATE_FIELDS:
        a, b = two.get_field(k), want[k]
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        assert same.all(), k
    two.close()


def test_vibration_errors():
    """Steps before the table is set are refused; nsteps < 1 is the
    reference's error 7; a flv 0 context takes no table."""
    sc = scenes.shaking_box(ndim=2, flv=1, dx=0.1)
    st = scenes.initialise(sc)
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    with pytest.raises(sphgpu.SPHError) as e:
        eng.step(1)
    assert e.value.code == 104
    bad = dict(st.vibration, nsteps=0, loads=np.zeros((1, 3)))
    with pytest.raises(sphgpu.SPHError) as e:
        eng.set_vibration(bad)
    assert e.value.code == 7
    eng.set_vibration(st.vibration)
    eng.step(2)
    eng.close()
    p0 = dict(st.params, flv=0)
    eng = sphgpu.Engine(p0, device=0)
    with pytest.raises(sphgpu.SPHError) as e:
        eng.set_vibration(st.vibration)
    assert e.value.code == 104
    eng.close()
