"""The FP32-bulk form (SPHGPU_PREC_FP32_BULK) against the FP64 oracle.

In the bulk form the pair arithmetic of the neighbour passes runs in FP32
with Kahan-compensated sums; positions, velocities, densities, stresses, the
time integration, the constitutive update and the neighbour search stay FP64.
Errors are stated per field as the relative L2 norm over the moving particles
(types 1-4), ||a - b|| / ||b||, and as the largest absolute difference
relative to the field's largest magnitude.

* Neighbour lists are identical to the oracle's (same positions in, same lists
  out): the search is shared with the FP64 form.
* On runs whose dynamics are smooth (the fluid dam break, an elastic soil
  column) every checked field stays within BULK_REL_TOL of the oracle.
* The Drucker-Prager soil column switches branches (yield, tension cut-off,
  the drag reversal limiter, free-surface colour thresholds) and amplifies
  any rounding: the FP64 form started from positions perturbed by 1e-13
  drifts from the oracle by as much.  There the bulk form's error is held to
  CONDITIONING_FACTOR times that FP64 drift.
"""
import numpy as np
import pytest

import scenes
import sphgpu
from checkers import ORC_JACOBI, ORC_POW_CR, Oracle

pytestmark = pytest.mark.gpu

BULK_REL_TOL = 1e-4          # stress and displacement: the bound the FP32-bulk form is held to
CONDITIONING_FACTOR = 3.0
FIELDS = ("sig", "ux", "vx", "rho", "pre", "xp")


def _rel(a, b, moving):
    a, b = a[moving], b[moving]
    l2 = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    mx = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    return l2, mx


def _runs(sc, steps, perturb=None):
    st = scenes.initialise(sc)
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    eng.set_precision(sphgpu.PREC_FP32_BULK)
    assert eng.precision == sphgpu.PREC_FP32_BULK
    orc = Oracle(st.params, ORC_JACOBI, ORC_POW_CR)
    orc.load_state(st.fields, st.fluid, st.soil)
    eng.step(steps)
    assert orc.step(steps) == 0
    moving = (st.fields["type"] >= 1) & (st.fields["type"] <= 4)
    errs = {k: _rel(eng.get_field(k), orc.get_field(k), moving) for k in FIELDS}
    drift = None
    if perturb is not None:
        f2 = dict(st.fields)
        xp = np.array(st.fields["xp"], dtype=np.float64).reshape(-1, 3)
        rng = np.random.default_rng(11)
        xp[moving] *= 1.0 + perturb * rng.standard_normal(xp[moving].shape)
        f2["xp"] = xp
        e64 = sphgpu.Engine(st.params, device=0)
        e64.load_state(f2, st.fluid, st.soil)
        e64.step(steps)
        drift = {k: _rel(e64.get_field(k), orc.get_field(k), moving) for k in FIELDS}
    return eng, orc, errs, drift


def test_bulk_neighbour_lists_identical():
    sc = scenes.soil_column_3d(dx=0.05, steps=100)
    st = scenes.initialise(sc)
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    eng.set_precision(sphgpu.PREC_FP32_BULK)
    eng.step(20)
    # the oracle's search on the bulk run's positions
    orc = Oracle(st.params, ORC_JACOBI, ORC_POW_CR)
    fields = dict(st.fields)
    fields["xp"] = eng.get_field("xp")
    orc.load_state(fields, st.fluid, st.soil)
    n1, i1 = eng.nnps()
    err, n2, i2, _ = orc.nnps()
    assert err == 0
    assert np.array_equal(n1, n2)
    for i in range(len(n1)):
        m = min(n1[i], 99)
        assert np.array_equal(i1[i, 1:m + 1], i2[i, 1:m + 1]), i


@pytest.mark.parametrize("label,factory,steps", [
    ("dam_break_2d", lambda: scenes.dam_break_2d(dx=0.01, steps=100), 200),
    ("elastic_column_3d", lambda: scenes.set_soil_model(scenes.soil_column_3d(dx=0.05, steps=100), 6, e=1.0e7), 200),
])
def test_bulk_error_smooth_runs(label, factory, steps):
    _, _, errs, _ = _runs(factory(), steps)
    print(label, {k: ("%.2e" % v[0], "%.2e" % v[1]) for k, v in errs.items()})
    for k in ("sig", "ux"):
        assert errs[k][0] <= BULK_REL_TOL, (k, errs[k])
    for k in ("vx", "rho", "pre", "xp"):
        assert errs[k][0] <= BULK_REL_TOL, (k, errs[k])


def test_bulk_error_within_conditioning_of_dp_column():
    _, _, errs, drift = _runs(scenes.soil_column_3d(dx=0.05, steps=100), 200, perturb=1e-13)
    print("bulk", {k: "%.2e" % v[0] for k, v in errs.items()})
    print("fp64 perturbed 1e-13", {k: "%.2e" % v[0] for k, v in drift.items()})
    for k in ("sig", "ux", "vx"):
        assert errs[k][0] <= CONDITIONING_FACTOR * drift[k][0], (k, errs[k], drift[k])


def test_precision_switch_roundtrip():
    """Switching back to FP64 restores the bit-exact drop-in."""
    sc = scenes.dam_break_2d(dx=0.02, steps=10)
    st = scenes.initialise(sc)
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    eng.set_precision(sphgpu.PREC_FP32_BULK)
    eng.set_precision(sphgpu.PREC_FP64)
    orc = Oracle(st.params, ORC_JACOBI, ORC_POW_CR)
    orc.load_state(st.fields, st.fluid, st.soil)
    eng.step(5)
    assert orc.step(5) == 0
    for k in ("xp", "vx", "rho", "sig"):
        assert np.array_equal(eng.get_field(k), orc.get_field(k)), k
    with pytest.raises(sphgpu.SPHError):
        eng.set_precision(7)
