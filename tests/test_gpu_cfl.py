"""The adaptive time step (sphgpu_set_cfl), an addition of this library: the
reference's dt is constant (CPP_12-2-dt.cpp:13-20).  After every step the
device reduces min(cfl h / (c + |v|), cfl_force sqrt(h / |a|)) over the water,
soil, air and structure particles, and the next step runs with it, capped at
the input dt.  The reduction is checked bit for bit against the same
expression evaluated here on the downloaded state (IEEE division and square
root round identically on both sides; the minimum is exact)."""
import numpy as np
import pytest

import scenes
import sphgpu

pytestmark = pytest.mark.gpu


def _expected_dt(eng, st, cfl, cfl_f):
    nd = int(st.params["ndim"])
    t = eng.get_field("type")
    v, a, h = eng.get_field("vxp"), eng.get_field("axp"), eng.get_field("hl")
    c = np.where((t == 1) | (t == 3), st.fluid["vpu"], np.where(t == 2, st.soil["vpu"],
                                                                 st.params["structure"]["vpu"]))
    v2 = np.zeros(len(t))
    a2 = np.zeros(len(t))
    for k in range(nd):
        v2 = v2 + v[:, k] * v[:, k]
        a2 = a2 + a[:, k] * a[:, k]
    lim = cfl * (h / (c + np.sqrt(v2)))
    with np.errstate(divide="ignore"):
        lf = cfl_f * np.sqrt(h / np.sqrt(a2))
    lim = np.where((a2 > 0.0) & (lf < lim), lf, lim)
    act = (t >= 1) & (t <= 4)
    return min(float(lim[act].min()), float(st.params["dt"]))


@pytest.mark.parametrize("factory", [lambda: scenes.dam_break_2d(dx=0.01, steps=100),
                                     lambda: scenes.soil_column_3d(dx=0.05, steps=100)])
def test_cfl_dt_is_the_reduced_limit(factory):
    st = scenes.initialise(factory())
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    assert eng.dt() == st.params["dt"]
    cfl, cfl_f = 0.2, 0.25
    eng.set_cfl(cfl, cfl_f)
    assert eng.dt() == st.params["dt"]          # the first step runs with the input dt
    seen = []
    for _ in range(15):
        eng.step(1)
        want = _expected_dt(eng, st, cfl, cfl_f)
        got = eng.dt()
        assert got == want, (got, want)
        seen.append(got)
    assert min(seen) < st.params["dt"]           # the limit bites once the particles move
    assert all(np.isfinite(eng.get_field("vx")).ravel())
    eng.set_cfl(0.0)
    assert eng.dt() == st.params["dt"]
    eng.close()


def test_cfl_off_is_the_constant_step():
    """Turning the adaptive step on and off again leaves a run identical to one
    that never had it."""
    sc = scenes.dam_break_2d(dx=0.02, steps=100)
    outs = []
    for toggle in (False, True):
        st = scenes.initialise(sc)
        eng = sphgpu.Engine(st.params, device=0)
        eng.load_state(st.fields, st.fluid, st.soil)
        if toggle:
            eng.set_cfl(0.2)
            eng.set_cfl(0.0)
        eng.step(10)
        outs.append(eng.get_field("xp"))
        eng.close()
    assert np.array_equal(outs[0], outs[1])
