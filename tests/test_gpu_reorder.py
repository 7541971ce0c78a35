"""Re-sorted state (sphgpu_set_reorder): the engine holds the particle state
in a spatial order (rows of a lattice of spacing dr), re-sorted on the device
every R steps, and maps back to the caller's order at every exchange with the
host.

The reference keeps its particle array in input order (Binary_Sort,
CPP_3-NNPS.cpp:561-630, sorts an index list only), so a re-sorted run must
give exactly the caller's-order run: every field, the neighbour lists, the
rain bookkeeping and the result files bit for bit.  The cases cover every
pass whose result depends on the particle numbering: the search's order
inside a cell, the rain rows (rainpro), check_domain's first wall of matype
> 2 (the shaking boxes), tm_boundary's default wall (flbndy 2), the order of
a structure particle's contact reactions (the footings) and the batched
instances' tables.
"""
import filecmp
import glob
import os
import tempfile

import numpy as np
import pytest

import make_golden
import scenes
import sphgpu
from checkers import ORC_JACOBI, ORC_POW_CR, STATE_FIELDS, Oracle

pytestmark = pytest.mark.gpu


def _same(a, b):
    if a.dtype.kind != "f":
        return np.array_equal(a, b)
    return bool(((a == b) | (np.isnan(a) & np.isnan(b))).all())


def _engine(st, reorder, bulk=False, instances=None, fields=None, fluid=None, soil=None):
    eng = sphgpu.Engine(st.params if instances is None else st, device=0, instances=instances)
    if instances is None:
        eng.load_state(st.fields, st.fluid, st.soil, st.rain, vibration=st.vibration)
    else:
        eng.load_state(fields, fluid, soil)
    if bulk:
        eng.set_precision(sphgpu.PREC_FP32_BULK)
    eng.set_reorder(reorder)
    return eng


def _run(eng, chunks):
    for c in chunks:
        eng.step(c)


def _assert_equal_runs(a, b, label):
    assert a.step_index == b.step_index
    for k in STATE_FIELDS:
        assert _same(a.get_field(k), b.get_field(k)), (label, k)
    n1, i1 = a.nnps()
    n2, i2 = b.nnps()
    assert np.array_equal(n1, n2), label
    mask = np.arange(100)[None, :] <= np.minimum(n1, 99)[:, None]
    assert np.array_equal(np.where(mask, i1, 0), np.where(mask, i2, 0)), label


def _held_out_of_order(eng):
    """The map the device holds, read before any call that restores the
    caller's order: a permutation, and not the identity."""
    o = eng.order()
    assert np.array_equal(np.sort(o), np.arange(eng.n))
    return not np.array_equal(o, np.arange(eng.n))


@pytest.mark.parametrize("name", list(make_golden.CASES))
def test_every_golden_case_resorted_each_step(name):
    factory, steps = make_golden.CASES[name]
    st = scenes.initialise(factory())
    plain, sorted_ = _engine(st, 0), _engine(st, 1)
    _run(plain, (1, steps - 1))
    _run(sorted_, (1, steps - 1))
    assert _held_out_of_order(sorted_)
    if st.rain is not None:
        assert sorted_.rain()["nrain"] == plain.rain()["nrain"]
    _assert_equal_runs(plain, sorted_, name)
    plain.close()
    sorted_.close()


@pytest.mark.parametrize("name,every", [("soil_column_3d_dx0.1", 3), ("dam_break_2d_dx0.04_rain", 4),
                                        ("footing_3d_deformable_coupled", 5), ("shaking_box_2d_flv2", 7)])
def test_resorted_every_few_steps_against_the_oracle(name, every):
    """Re-sorts every few steps, the steps run in uneven chunks (a re-sort
    falls inside a sphgpu_step call and across calls): bit-identical to the
    oracle, which runs the caller's order."""
    factory, steps = make_golden.CASES[name]
    st = scenes.initialise(factory())
    eng = _engine(st, every)
    orc = Oracle(st.params, ORC_JACOBI, ORC_POW_CR)
    orc.load_state(st.fields, st.fluid, st.soil, st.rain, vibration=st.vibration)
    for c in (2, 5, steps - 7):
        eng.step(c)
        assert orc.step(c) == 0
    assert _held_out_of_order(eng)
    for k in STATE_FIELDS:
        assert _same(eng.get_field(k), orc.get_field(k)), (name, k)
    eng.close()


def _shuffled(st, seed):
    """The same scene with its particles in a random order (every per-particle
    input permuted alike); waiting rain particles stay at the end, in their
    rows."""
    n = int(st.params["ntotal"])
    tail = st.rain["nrain"] if st.rain else 0
    p = np.concatenate([np.random.default_rng(seed).permutation(n - tail), np.arange(n - tail, n)])
    fields = {k: np.ascontiguousarray(v[p]) for k, v in st.fields.items()}
    fluid = None if st.fluid is None else np.ascontiguousarray(st.fluid[p])
    soil = None if st.soil is None else np.ascontiguousarray(st.soil[p])
    return scenes.InitialState(params=st.params, fields=fields, fluid=fluid, soil=soil, rain=st.rain,
                               vibration=st.vibration)


@pytest.mark.parametrize("factory,steps", [
    (lambda: scenes.soil_column_3d(dx=0.05, steps=200), 12),
    (lambda: scenes.dam_break_2d(dx=0.01, steps=200), 30),
    (make_golden.CASES["footing_3d_deformable"][0], 10),
])
def test_random_input_order(factory, steps):
    """Particles given in a random order: the re-sorted run equals the run
    held in that order, in both precision forms."""
    st = _shuffled(scenes.initialise(factory()), 5)
    for bulk in (False, True):
        plain, sorted_ = _engine(st, 0, bulk), _engine(st, 2, bulk)
        _run(plain, (3, steps - 3))
        _run(sorted_, (3, steps - 3))
        assert _held_out_of_order(sorted_)
        _assert_equal_runs(plain, sorted_, ("bulk" if bulk else "fp64"))
        plain.close()
        sorted_.close()


def test_dam_break_full_size_long_run():
    """The 2-D dam break at dx = 5 mm for 1,500 steps, re-sorted every 25
    steps while the water runs across the tank: identical to the run in the
    caller's order."""
    st = scenes.initialise(scenes.dam_break_2d(dx=0.005, steps=2000))
    plain, sorted_ = _engine(st, 0), _engine(st, 25)
    _run(plain, (700, 800))
    _run(sorted_, (700, 800))
    assert _held_out_of_order(sorted_)
    _assert_equal_runs(plain, sorted_, "dam break")
    plain.close()
    sorted_.close()


def test_batched_instances_resorted():
    states = [scenes.initialise(sc) for sc in (scenes.slope_2d(H=h, dx=0.05) for h in (1.0, 1.75, 1.3))]
    shared, insts, fields, fluid, soil = sphgpu.batch(states)
    plain = _engine(shared, 0, instances=insts, fields=fields, fluid=fluid, soil=soil)
    sorted_ = _engine(shared, 1, instances=insts, fields=fields, fluid=fluid, soil=soil)
    _run(plain, (1, 19))
    _run(sorted_, (1, 19))
    assert _held_out_of_order(sorted_)
    _assert_equal_runs(plain, sorted_, "batched")
    plain.close()
    sorted_.close()


def test_host_exchanges_between_resorted_steps():
    """Field reads and writes, a record download and upload, the method
    entries and a checkpoint between re-sorted steps: each sees and changes
    the caller's order, and the run goes on as the plain one does."""
    st = scenes.initialise(scenes.soil_column_3d(dx=0.1, steps=200))
    plain, sorted_ = _engine(st, 0), _engine(st, 1)
    for eng in (plain, sorted_):
        eng.step(4)
    assert _held_out_of_order(sorted_)
    # a field written in the caller's order
    for eng in (plain, sorted_):
        v = eng.get_field("vxp")
        v[::7, 2] += 1.0e-3
        eng.set_field("vxp", v)
        eng.step(3)
    assert _held_out_of_order(sorted_)
    # records out and back in
    for eng in (plain, sorted_):
        rec = np.zeros(eng.n * sphgpu.PARTICLE_BYTES, dtype=np.uint8)
        eng.download_particles(rec)
        eng.upload_particles(rec)
        eng.step(2)
    # the method entries for one step
    for eng in (plain, sorted_):
        assert eng.parttocell() == 0
        assert eng.partisearching() == 0
        assert eng.update() == 0
        eng.step(3)
    assert _held_out_of_order(sorted_)
    # a checkpoint of the re-sorted state, loaded into a fresh context
    path = tempfile.mktemp(prefix="sphck", suffix=".bin", dir="/tmp")
    sorted_.checkpoint_save(path)
    fresh = _engine(st, 1)
    fresh.checkpoint_load(path)
    os.remove(path)
    for eng in (plain, sorted_, fresh):
        eng.step(5)
    _assert_equal_runs(plain, sorted_, "exchanges")
    _assert_equal_runs(plain, fresh, "checkpoint")
    for eng in (plain, sorted_, fresh):
        eng.close()


def test_result_files_from_the_resorted_state():
    """The result-file snapshot writes its rows through the map: the files of
    a re-sorted run are byte-identical to the plain run's."""
    sc = scenes.shaking_box(ndim=2, flv=1, dx=0.05)
    sc.problem["if_cal"] = 1
    st = scenes.initialise(sc)
    dirs = []
    for every in (0, 1):
        eng = _engine(st, every)
        d = tempfile.mkdtemp(prefix="sphro", dir="/tmp")
        eng.output_begin(d)
        done = 0
        for l in (2, 5, 9):
            eng.step(l - done)
            done = l
            eng.output_step(d, sphgpu.OUT_ODB | sphgpu.OUT_FLOWDIST | sphgpu.OUT_IMPACT | sphgpu.OUT_MGF)
        if every:
            assert _held_out_of_order(eng)
        eng.output_wait()
        eng.close()
        dirs.append(d)
    names = sorted(os.path.basename(p) for p in glob.glob(os.path.join(dirs[0], "*")))
    assert len(names) >= 5
    assert names == sorted(os.path.basename(p) for p in glob.glob(os.path.join(dirs[1], "*")))
    for f in names:
        assert filecmp.cmp(os.path.join(dirs[0], f), os.path.join(dirs[1], f), shallow=False), f


def test_step_profiled_resorts_and_reports():
    st = scenes.initialise(scenes.soil_column_3d(dx=0.05, steps=200))
    plain, sorted_ = _engine(st, 0), _engine(st, 2)
    plain.step(6)
    prof = sorted_.step_profiled(6)
    assert prof["reorder"] > 0.0
    assert _held_out_of_order(sorted_)
    _assert_equal_runs(plain, sorted_, "profiled")
    plain.close()
    sorted_.close()


@pytest.mark.parametrize("shuffle", [False, True])
def test_reorder_autotuner_keeps_results(shuffle):
    """sphgpu_autotune_reorder times both orders over real steps and keeps
    one; whichever it keeps, the run stays the plain run bit for bit, and with
    0 chosen the state is back in the caller's order."""
    st = scenes.initialise(scenes.soil_column_3d(dx=0.05, steps=200))
    if shuffle:
        st = _shuffled(st, 11)
    plain, tuned = _engine(st, 0), _engine(st, 0)
    got = tuned.autotune_reorder(steps=2, every=5)
    assert got["every_steps"] in (0, 5)
    assert got["caller_order_ms"] > 0 and got["resorted_ms"] > 0 and got["resort_ms_per_step"] > 0
    assert tuned.reorder == got["every_steps"]
    if got["every_steps"] == 0:
        assert not _held_out_of_order(tuned)
    plain.step(4)               # the autotuner's own 2 + 2 steps
    tuned.step(7)
    plain.step(7)
    _assert_equal_runs(plain, tuned, "autotuned")
    plain.close()
    tuned.close()


@pytest.mark.parametrize("every", [0, 3])
@pytest.mark.parametrize("factory,steps", [
    (lambda: scenes.dam_break_2d(dx=0.02, steps=100), 25),
    (lambda: scenes.soil_column_3d(dx=0.05, steps=100), 12),
    (make_golden.CASES["footing_3d_deformable"][0], 10),
    (make_golden.CASES["shaking_box_2d_flv1"][0], 20),
    (make_golden.CASES["dam_break_2d_dx0.04_rain"][0], 35),
])
def test_random_order_against_the_oracle(factory, steps, every):
    """Particles in a random order (whose results the oracle pins to the
    reference's on the same order, tests/test_oracle.py): the engine, held in
    that order or re-sorted, is bit-identical to the oracle."""
    st = _shuffled(scenes.initialise(factory()), 7)
    eng = _engine(st, every)
    orc = Oracle(st.params, ORC_JACOBI, ORC_POW_CR)
    orc.load_state(st.fields, st.fluid, st.soil, st.rain, vibration=st.vibration)
    for c in (1, steps - 1):
        eng.step(c)
        assert orc.step(c) == 0
    if every:
        assert _held_out_of_order(eng)
    for k in STATE_FIELDS:
        assert _same(eng.get_field(k), orc.get_field(k)), k
    if st.rain:
        assert eng.rain()["nrain"] == orc.rain()["nrain"] == 0
    eng.close()
