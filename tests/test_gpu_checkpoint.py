"""Checkpoint and restart (sphgpu_checkpoint_save / _load): a run saved
between steps and continued in a new context from the file goes on bit for
bit as the run that was not interrupted (every state field after the same
further steps)."""
import os
import tempfile

import numpy as np
import pytest

import make_golden
import scenes
import sphgpu
from checkers import STATE_FIELDS

pytestmark = pytest.mark.gpu


def _same(a, b):
    if a.dtype.kind != "f":
        return np.array_equal(a, b)
    return bool(((a == b) | (np.isnan(a) & np.isnan(b))).all())


@pytest.mark.parametrize("label,factory,before,after,cfl", [
    ("column_no_slip_walls", make_golden.CASES["soil_column_3d_dx0.1_no_slip_vsd"][0], 6, 6, 0.0),
    ("dam_break_tm_boundary", make_golden.CASES["dam_break_2d_dx0.04_tm_boundary"][0], 7, 8, 0.0),
    ("dam_break_rain", make_golden.CASES["dam_break_2d_dx0.04_rain"][0], 12, 12, 0.0),
    ("dam_break_cfl", lambda: scenes.dam_break_2d(dx=0.02, steps=100), 8, 8, 0.2),
])
def test_restart_continues_bit_for_bit(label, factory, before, after, cfl):
    st = scenes.initialise(factory())
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil, st.rain)
    if cfl > 0.0:
        eng.set_cfl(cfl)
    eng.step(before)
    path = os.path.join(tempfile.mkdtemp(), "run.ck")
    eng.checkpoint_save(path)
    eng.step(after)
    want = {k: eng.get_field(k) for k in STATE_FIELDS}
    want_l = eng.step_index
    want_dt = eng.dt()
    want_rain = eng.rain()["nrain"] if st.rain is not None else None
    eng.close()
    again = sphgpu.Engine(st.params, device=0)
    again.checkpoint_load(path)
    assert again.step_index == want_l - after
    again.step(after)
    assert again.step_index == want_l
    assert again.dt() == want_dt
    for k in STATE_FIELDS:
        assert _same(again.get_field(k), want[k]), (label, k)
    if st.rain is not None:
        assert again.rain()["nrain"] == want_rain < st.rain["nrain"]
    again.close()


def test_checkpoint_rejects_another_system():
    st = scenes.initialise(scenes.dam_break_2d(dx=0.04, steps=10))
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    eng.step(2)
    path = os.path.join(tempfile.mkdtemp(), "run.ck")
    eng.checkpoint_save(path)
    other = scenes.initialise(scenes.dam_break_2d(dx=0.05, steps=10))
    e2 = sphgpu.Engine(other.params, device=0)
    with pytest.raises(sphgpu.SPHError) as e:
        e2.checkpoint_load(path)
    assert e.value.code == 100
