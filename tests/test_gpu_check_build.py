"""The bounds-checked build (libsphgpu_check.so, SPHGPU_CHECK=1): after every
neighbour search a pass checks each index the later passes take from it --
list slots within [0, N) and not the particle itself, slot masks marking
exactly the slots of their type, the sorted order a permutation, the cell
ranges within the sorted positions -- and sets SPHGPU_E_CHECK (106) rather
than trapping.  On valid runs it must report nothing and change no result:
every field bit-identical to the plain build's, step for step.  The plain
build is also bitwise deterministic: two runs of the same input agree."""
import numpy as np
import pytest

import make_golden
import scenes
import sphgpu
from checkers import STATE_FIELDS

pytestmark = pytest.mark.gpu


def _run(sc, steps, library=None):
    st = scenes.initialise(sc)
    eng = sphgpu.Engine(st.params, device=0, library=library)
    eng.load_state(st.fields, st.fluid, st.soil, st.rain, st.vibration)
    for chunk in (1, steps - 1):
        eng.step(chunk)
    out = {k: eng.get_field(k) for k in STATE_FIELDS}
    nn, nb = eng.nnps()
    eng.close()
    return out, nn, nb


def _same(a, b):
    if a.dtype.kind != "f":
        return np.array_equal(a, b)
    return bool(((a == b) | (np.isnan(a) & np.isnan(b))).all())


@pytest.mark.parametrize("label,factory,steps", [
    ("dam_break_2d", lambda: scenes.dam_break_2d(dx=0.02, steps=100), 20),
    ("soil_column_3d", lambda: scenes.soil_column_3d(dx=0.1, steps=200), 12),
    ("footing_penalty", make_golden.CASES["footing_2d_penalty_coupled"][0], 10),
    ("rain_slope_3d", make_golden.CASES["rain_slope_3d_dx0.25"][0], 20),
])
def test_checked_build_agrees_with_plain_build(label, factory, steps):
    plain, n1, b1 = _run(factory(), steps)
    checked, n2, b2 = _run(factory(), steps, library=sphgpu.CHECK_LIB_PATH)
    for k in STATE_FIELDS:
        assert _same(plain[k], checked[k]), (label, k)
    assert np.array_equal(n1, n2) and np.array_equal(b1, b2)


def test_plain_build_is_deterministic():
    a, n1, b1 = _run(scenes.soil_column_3d(dx=0.05, steps=100), 15)
    b, n2, b2 = _run(scenes.soil_column_3d(dx=0.05, steps=100), 15)
    for k in STATE_FIELDS:
        assert _same(a[k], b[k]), k
    assert np.array_equal(n1, n2) and np.array_equal(b1, b2)
