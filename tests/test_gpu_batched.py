"""Batched contexts (sphgpu_create_batched): several systems of uneven size in
one particle array, stepped by the same kernel launches, driven by the
per-instance table of particle ranges and cell grids.

Each instance must evolve exactly as a context of its own: every field and
its neighbour lists bit-identical to a single-system run of the same scene
(which the other parity tests hold to the oracle and the reference).  The
reference runs such instances as separate projects (CPP_0-main.cpp, one
SPH_Calculation per directory)."""
import numpy as np
import pytest

import scenes
import sphgpu
from checkers import STATE_FIELDS

pytestmark = pytest.mark.gpu


def _slopes(heights, dx=0.05):
    return [scenes.slope_2d(H=h, dx=dx) for h in heights]


def _dam_breaks(widths, flbndy):
    out = []
    for w in widths:
        sc = scenes.dam_break_2d(dx=0.04, water=(w, 0.6), steps=200)
        sc.flags["flbndy"] = flbndy
        out.append(sc)
    return out


def _columns(heights):
    return [scenes.soil_column_3d(dx=0.1, block=(1.0, 0.5, h), steps=200) for h in heights]


def _run_single(st, steps, bulk):
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    if bulk:
        eng.set_precision(sphgpu.PREC_FP32_BULK)
    eng.step(steps)
    out = {k: eng.get_field(k) for k in STATE_FIELDS}
    nn, nb = eng.nnps()
    eng.close()
    return out, nn, nb


def _same(a, b):
    if a.dtype.kind != "f":
        return np.array_equal(a, b)
    return bool(((a == b) | (np.isnan(a) & np.isnan(b))).all())


@pytest.mark.parametrize("label,make,steps,bulk", [
    ("slopes_2d", lambda: _slopes([1.0, 1.75, 1.3]), 25, False),
    ("slopes_2d_bulk", lambda: _slopes([1.0, 1.75, 1.3]), 25, True),
    ("dam_breaks_tm_boundary", lambda: _dam_breaks([0.24, 0.4, 0.32], 2), 20, False),
    ("dam_breaks_no_slip", lambda: _dam_breaks([0.24, 0.4], 13), 20, False),
    ("columns_3d", lambda: _columns([0.3, 0.5]), 12, False),
])
def test_batched_instances_match_single_runs(label, make, steps, bulk):
    states = [scenes.initialise(sc) for sc in make()]
    shared, insts, fields, fluid, soil = sphgpu.batch(states)
    eng = sphgpu.Engine(shared, device=0, instances=insts)
    assert eng.lib.sphgpu_instance_count(eng.h) == len(states)
    eng.load_state(fields, fluid, soil)
    if bulk:
        eng.set_precision(sphgpu.PREC_FP32_BULK)
    for chunk in (1, steps - 1):
        eng.step(chunk)
    got = {k: eng.get_field(k) for k in STATE_FIELDS}
    nn, nb = eng.nnps()
    eng.close()
    for q, st in enumerate(states):
        a, cnt = int(insts[q].first), int(insts[q].count)
        want, wn, wb = _run_single(st, steps, bulk)
        for k in STATE_FIELDS:
            assert _same(got[k][a:a + cnt], want[k]), (label, q, k)
        assert np.array_equal(nn[a:a + cnt], wn), (label, q)
        rows = nb[a:a + cnt]
        mask = np.arange(100)[None, :] <= np.minimum(wn, 99)[:, None]
        mask[:, 0] = False
        assert np.array_equal(np.where(mask, rows - a, 0), np.where(mask, wb, 0)), (label, q)


def test_batched_kl_fields_match_single_runs():
    """One lognormal cohesion field per slope, each with its own normals and
    domain, in one call: the same values (and the same steps after them) as
    sphgpu_kl_generate on a context of the slope alone."""
    scs = _slopes([1.0, 1.6])
    states = [scenes.initialise(sc) for sc in scs]
    shared, insts, fields, fluid, soil = sphgpu.batch(states)
    eng = sphgpu.Engine(shared, device=0, instances=insts)
    eng.load_state(fields, fluid, soil)
    field = sphgpu.kl_field(1, 2, 10.0e3, 3.0e3, [10.0, 1.0, 0.0])
    doms, xis = [], []
    for q, sc in enumerate(scs):
        d = scenes.kl_domain(sc)
        doms.append(sphgpu.kl_domain(d["nb_min"], d["nb_max"], d["soil_max"], d["water_max"]))
        xis.append(np.random.default_rng(100 + q).standard_normal(200))
    got = eng.kl_generate_batched(doms, field, np.array(xis))
    eng.step(10)
    sig = eng.get_field("sig")
    eng.close()
    for q, st in enumerate(states):
        a, cnt = int(insts[q].first), int(insts[q].count)
        one = sphgpu.Engine(st.params, device=0)
        one.load_state(st.fields, st.fluid, st.soil)
        want = one.kl_generate(doms[q], [field], xis[q][None, :])[0]
        assert _same(got[a:a + cnt], want), q
        one.step(10)
        assert _same(sig[a:a + cnt], one.get_field("sig")), q
        one.close()


def test_batched_rejects_a_broken_table():
    """Instances must follow one another from particle 0 with their own
    complete grids."""
    states = [scenes.initialise(sc) for sc in _slopes([1.0, 1.2])]
    shared, insts, _, _, _ = sphgpu.batch(states)
    insts[1].first += 1
    with pytest.raises(sphgpu.SPHError) as e:
        sphgpu.Engine(shared, device=0, instances=insts)
    assert e.value.code == 100
