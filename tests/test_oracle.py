"""The oracle (C restatement of the reference's step loop) pinned against the
reference solver: against the committed golden fixtures made by the reference
(tests/golden/make_golden.py) and, where the reference is built here
(oracle/_ref), against live runs of it.  CPU only."""
import os
import tempfile

import numpy as np
import pytest

import make_golden
import scenes
import sphgpu
from checkers import (ORC_INPLACE, ORC_JACOBI, ORC_POW_CR, ORC_POW_LIBM, STATE_FIELDS, Oracle,
                      Params, Reference, have_reference)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["dam_break_2d_dx0.04", "soil_column_3d_dx0.1", "soil_column_3d_dx0.1_kgc_regu",
         "slope_2d_H1_dx0.05_art_stress", "soil_column_3d_dx0.1_art_stress",
         "soil_column_3d_dx0.1_drag_tsuji_dilute", "soil_column_3d_dx0.1_drag_peng",
         "soil_column_3d_dx0.1_camclay", "soil_column_3d_dx0.1_mohr_coulomb", "soil_column_3d_dx0.1_visco_elastic",
         "dam_break_2d_dx0.04_tm_boundary", "soil_column_3d_dx0.1_tm_boundary",
         "footing_2d_rigid", "footing_2d_deformable", "footing_2d_penalty", "footing_3d_deformable",
         "footing_3d_penalty", "dam_break_2d_dx0.04_no_slip", "dam_break_2d_dx0.04_free_slip_vsd",
         "soil_column_3d_dx0.1_free_slip", "soil_column_3d_dx0.1_no_slip_vsd",
         "dam_break_2d_dx0.04_free_solid", "soil_column_3d_dx0.1_free_solid",
         "footing_2d_penalty_coupled", "footing_3d_deformable_coupled",
         "soil_column_3d_dx0.1_unsat", "soil_column_3d_dx0.1_amcc", "soil_column_3d_dx0.1_focc",
         "soil_column_3d_dx0.1_tssmp",
         "three_phase_column_3d_dx0.1_unsat", "three_phase_column_3d_dx0.1_minor",
         "dam_break_2d_dx0.04_minor", "dam_break_2d_dx0.04_bingham", "dam_break_2d_dx0.04_moving_wall",
         "soil_column_3d_dx0.1_moving_wall", "soil_column_3d_dx0.1_geostatic",
         "soil_column_3d_dx0.1_geostatic_camclay", "slope_2d_H1_dx0.05_geostatic",
         "dam_break_2d_dx0.04_rain", "shaking_box_2d_flv1", "shaking_box_2d_flv2", "shaking_box_3d_flv1",
         "shaking_box_3d_flv2", "rain_slope_3d_dx0.25"]


def _golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    p = Params.from_buffer_copy(g["params"].tobytes())
    return g, p


def golden_rain(g):
    """The rainfall record a golden case was made with (None without rain)."""
    if "rain" not in g:
        return None
    r = g["rain"]
    return dict(rtype=int(r[0]), nrain=int(r[1]), nhor=int(r[2]), press_factor=float(r[3]),
                drop_velocity=float(r[4]))


def golden_vibration(g):
    """The vibration table a golden case was made with (None without)."""
    if "vib_par" not in g:
        return None
    v = g["vib_par"]
    return dict(ttime=float(v[0]), nsteps=int(v[1]), sttime=float(v[2]), edtime=float(v[3]), loads=g["vib_loads"])


def _oracle_from_golden(g, p, mode=ORC_INPLACE, pow_mode=ORC_POW_LIBM):
    orc = Oracle(p, mode, pow_mode)
    orc.load_state({k: g["init_" + k] for k in STATE_FIELDS}, g["fluid"], g["soil"], golden_rain(g),
                   golden_vibration(g))
    return orc


@pytest.mark.parametrize("name", CASES)
def test_golden_neighbour_lists(name):
    """parttocell + partisearching: same neighbours, same order, same kernel
    values (bit for bit) as the reference."""
    g, p = _golden(name)
    orc = _oracle_from_golden(g, p)
    err, ninflu, influ, wij = orc.nnps(with_wij=True)
    assert err == 0
    assert np.array_equal(ninflu, g["nnps_ninflu"])
    mask = np.arange(100)[None, :] <= ninflu[:, None]
    assert np.array_equal(np.where(mask, influ, 0), g["nnps_influ"])
    assert np.array_equal(np.where(mask[:, :, None], wij, 0.0), g["nnps_wij"])


@pytest.mark.parametrize("name", CASES)
def test_golden_steps_bit_identical(name):
    """N full steps in the reference's own (sequential in-place) order and
    with the C library's pow: every state field bit-identical."""
    g, p = _golden(name)
    orc = _oracle_from_golden(g, p)
    assert orc.step(int(g["steps"])) == 0
    if "final_nrain" in g:
        assert orc.rain()["nrain"] == int(g["final_nrain"])
    for k in STATE_FIELDS:
        a, b = orc.get_field(k), g["final_" + k]
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        assert same.all(), (k, int((~same).sum()))


@pytest.mark.parametrize("name", CASES)
def test_golden_initial_state_from_scene(name):
    """scenes.initialise (the engine's host-side set-up) reproduces the
    reference's own initialisation bit for bit."""
    g, p = _golden(name)
    import make_golden
    sc = make_golden.CASES[name][0]()
    st = scenes.initialise(sc)
    assert bytes(sphgpu.params_from_dict(st.params)) == bytes(p)
    assert np.array_equal(st.fluid, g["fluid"]) and np.array_equal(st.soil, g["soil"])
    for k in STATE_FIELDS:
        assert np.array_equal(np.asarray(st.fields[k]).reshape(g["init_" + k].shape), g["init_" + k]), k


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("name,factor", [("soil_column_3d_dx0.1", 2.0), ("dam_break_2d_dx0.04", 6.0)])
def test_jacobi_order_vs_reference_numbering_sensitivity(name, factor):
    """The reference's Shepard pass updates densities in place in particle
    order (CPP_6-density.cpp:168-188), so its result depends on how the
    particles are numbered.  The engine uses the order-free (Jacobi) form.
    Measured on the golden cases: the Jacobi result differs from the
    reference by at most `factor` times what merely reversing the particle
    numbering changes in the reference itself (density, velocity,
    displacement; relative L2 over the moving particles)."""
    g, p = _golden(name)
    n = int(p.ntotal)
    steps = int(g["steps"])
    init = {k: g["init_" + k] for k in STATE_FIELDS}
    rev = np.arange(n)[::-1].copy()
    o_rev = Oracle(p, ORC_INPLACE)
    o_rev.load_state({k: np.asarray(v)[rev] for k, v in init.items()}, g["fluid"][rev], g["soil"][rev])
    assert o_rev.step(steps) == 0
    o_jac = _oracle_from_golden(g, p, ORC_JACOBI)
    assert o_jac.step(steps) == 0
    t = g["init_type"]
    act = (t >= 1) & (t <= 4)
    for k in ("rho", "vxp", "ux"):
        ref = g["final_" + k][act]
        d_rev = _rel_l2(o_rev.get_field(k)[rev.argsort()][act], ref)
        d_jac = _rel_l2(o_jac.get_field(k)[act], ref)
        assert d_rev > 0.0
        assert d_jac <= factor * d_rev, (k, d_jac, d_rev)


def test_pow7_correctly_rounded():
    """The CR evaluation of x^7 used by the engine (and ORC_POW_CR) is the
    correctly rounded power: checked against exact rational arithmetic."""
    from fractions import Fraction
    lib = Oracle.__init__.__globals__["oracle_lib"]()
    rng = np.random.default_rng(7)
    xs = np.concatenate([1.0 + (rng.random(4000) - 0.5) * 0.02, rng.random(1000) * 3.0])
    for x in xs:
        x = float(x)
        assert lib.orc_pow7(x) == float(Fraction(x) ** 7), x


def test_pow7_vs_libm_rate():
    """glibc's pow(x, 7) differs from the correctly rounded value on a small
    fraction of inputs near 1 (measured ~0.1%); this is the only arithmetic
    difference between the engine and the reference's FP64 path."""
    lib = Oracle.__init__.__globals__["oracle_lib"]()
    rng = np.random.default_rng(11)
    xs = 1.0 + (rng.random(200000) - 0.5) * 0.02
    diff = sum(lib.orc_pow7(float(x)) != float(x) ** 7.0 for x in xs)
    assert diff / len(xs) < 0.01


def test_oracle_error_codes():
    """parttocell's code 3 (particle outside the cell grid) and
    partisearching's code 5 (more than 99 neighbours)."""
    sc = scenes.dam_break_2d(dx=0.04, steps=10)
    st = scenes.initialise(sc)
    f = dict(st.fields)
    xp = f["xp"].copy()
    xp[3, 0] = st.params["xmax"] + 100.0
    f["xp"] = xp
    orc = Oracle(st.params)
    orc.load_state(f, st.fluid, st.soil)
    assert orc.step(1) == 3
    sc = scenes.dam_break_2d(dx=0.04, steps=10)
    water = np.flatnonzero(sc.ptype == 1)[:120]
    sc.xp[water, 0] = 0.2 + 0.001 * (np.arange(120) % 10)
    sc.xp[water, 1] = 0.2 + 0.001 * (np.arange(120) // 10)
    st = scenes.initialise(sc)
    orc = Oracle(st.params)
    orc.load_state(st.fields, st.fluid, st.soil)
    assert orc.step(1) == 5


# --------------------------------------------------------------------------
# live reference runs (where oracle/_ref was built from the reference sources)

needs_ref = pytest.mark.skipif(not have_reference(), reason="reference not built here (oracle/_ref)")


def _live(sc, nthreads=1):
    d = tempfile.mkdtemp()
    path = os.path.join(d, "input.dat")
    scenes.write_input_dat(sc, path)
    return Reference(path, nthreads)


def _variant(factory, flknl, step_regu):
    sc = factory()
    sc.flags["flknl"] = flknl
    sc.problem["step_regu"] = step_regu
    return sc


@needs_ref
@pytest.mark.parametrize("flknl,step_regu", [(2, 100000000), (3, 4), (4, 3), (1, 1)])
@pytest.mark.parametrize("factory,steps", [
    (lambda: scenes.dam_break_2d(dx=0.02, steps=100), 12),
    (lambda: scenes.soil_column_3d(dx=0.05, steps=100), 8),
])
def test_live_reference_kernel_and_regularisation_variants(factory, steps, flknl, step_regu):
    """Yang-Liu kernel (flknl 2/4), kernel gradient correction (flknl 3/4,
    CPP_3-NNPS.cpp:376-496) and strain/stress regularisation every step_regu
    steps (CPP_7-2-constitutive.cpp:385-450): bit-identical to the reference."""
    sc = _variant(factory, flknl, step_regu)
    ref = _live(sc)
    fl, so = ref.materials()
    orc = Oracle(ref.params, ORC_INPLACE)
    orc.load_state({k: ref.get_field(k) for k in STATE_FIELDS}, fl, so)
    assert ref.step(steps) == 0
    assert orc.step(steps) == 0
    for k in STATE_FIELDS:
        assert np.array_equal(orc.get_field(k), ref.get_field(k)), k


@needs_ref
@pytest.mark.parametrize("factory,steps", [
    (lambda: scenes.dam_break_2d(dx=0.02, steps=100), 40),
    (lambda: scenes.soil_column_3d(dx=0.05, steps=100), 20),
])
def test_live_reference_bit_identical(factory, steps):
    sc = factory()
    ref = _live(sc)
    fl, so = ref.materials()
    orc = Oracle(ref.params, ORC_INPLACE)
    orc.load_state({k: ref.get_field(k) for k in STATE_FIELDS}, fl, so)
    for chunk in (1, steps - 1):
        assert ref.step(chunk) == 0
        assert orc.step(chunk) == 0
    for k in STATE_FIELDS:
        a, b = orc.get_field(k), ref.get_field(k)
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        assert same.all(), k


def _shuffled_scene(sc, seed):
    """The scene's particles in a random order (every per-particle input
    permuted alike); waiting rain particles stay at the end of the array, in
    their rows, where rainpro releases them from."""
    tail = sc.rain["nrain"] if sc.rain else 0
    p = np.concatenate([np.random.default_rng(seed).permutation(sc.n - tail), np.arange(sc.n - tail, sc.n)])
    for k in ("xp", "vxp", "ptype", "matype", "permtype", "etype"):
        setattr(sc, k, np.ascontiguousarray(getattr(sc, k)[p]))
    return sc


@needs_ref
@pytest.mark.parametrize("factory,steps", [
    (lambda: scenes.dam_break_2d(dx=0.02, steps=100), 25),
    (lambda: scenes.soil_column_3d(dx=0.05, steps=100), 12),
    (make_golden.CASES["footing_3d_deformable"][0], 10),
    (make_golden.CASES["shaking_box_2d_flv1"][0], 20),
    (make_golden.CASES["dam_break_2d_dx0.04_rain"][0], 35),
])
def test_live_reference_random_particle_order(factory, steps):
    """The reference on its particles in a random order, where its neighbour
    order inside a cell (Binary_Sort), its in-place Shepard sweep, the order
    a structure particle takes its contact reactions in (the footing) and
    check_domain's first wall of matype > 2 (the shaking box) follow the
    numbering: the oracle in the reference's in-place order follows it bit for
    bit, so parity is pinned for any order a caller gives."""
    sc = _shuffled_scene(factory(), 7)
    ref = _live(sc)
    fl, so = ref.materials()
    orc = Oracle(ref.params, ORC_INPLACE)
    orc.load_state({k: ref.get_field(k) for k in STATE_FIELDS}, fl, so, sc.rain, vibration=sc.vibration)
    for chunk in (1, steps - 1):
        assert ref.step(chunk) == 0
        assert orc.step(chunk) == 0
    for k in STATE_FIELDS:
        a, b = orc.get_field(k), ref.get_field(k)
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        assert same.all(), k
    if sc.rain:
        assert orc.rain()["nrain"] == 0


def _stretched_column(dx):
    sc = scenes.soil_column_3d(dx=dx, steps=100)
    sc.soils[2]["c"] = 20.0e3
    sc.problem["art_stre_coe"] = 0.5
    return scenes.uplift(sc, 2, 0.25)


def _stretched_slope(dx):
    return scenes.uplift(scenes.slope_2d(H=1.0, dx=dx, art_stre_coe=0.5), 1, 0.5)


@needs_ref
@pytest.mark.parametrize("factory,steps", [
    (lambda: _stretched_slope(0.025), 20),
    (lambda: _stretched_column(0.05), 12),
])
def test_live_reference_artificial_stress(factory, steps):
    """Artificial stress (CPP_9-5-artificialstress.cpp) on soil in tension:
    bit-identical to the reference, and the tensile branch is reached."""
    sc = factory()
    ref = _live(sc)
    fl, so = ref.materials()
    orc = Oracle(ref.params, ORC_INPLACE)
    orc.load_state({k: ref.get_field(k) for k in STATE_FIELDS}, fl, so)
    assert ref.step(steps) == 0
    assert orc.step(steps) == 0
    for k in STATE_FIELDS:
        assert np.array_equal(orc.get_field(k), ref.get_field(k)), k
    strep, t = ref.get_field("strep"), ref.get_field("type")
    assert (strep[t == 2] > 0.0).any()


@needs_ref
@pytest.mark.parametrize("fli,eps0,vw", [(2, 0.6667, 0.05), (2, 5.0, 1.0), (3, 0.6667, 0.05), (3, 0.6667, 0.0)])
def test_live_reference_drag_forms(fli, eps0, vw):
    """interact2 (Tsuji/Shi: Ergun below porosity 0.8, Wen-Yu above) and
    interact3 (Peng: laminar below Re 60, turbulent above), CPP_10-interact1.cpp:
    114-405, bit-identical to the reference."""
    sc = scenes.soil_column_3d(dx=0.05, steps=100)
    sc.flags["fli"], sc.soils[2]["eps0"] = fli, eps0
    w = np.flatnonzero(sc.ptype == 1)
    sc.vxp[w, 0] = vw * (np.arange(len(w)) % 4)
    ref = _live(sc)
    fl, so = ref.materials()
    orc = Oracle(ref.params, ORC_INPLACE)
    orc.load_state({k: ref.get_field(k) for k in STATE_FIELDS}, fl, so)
    assert ref.step(10) == 0
    assert orc.step(10) == 0
    for k in STATE_FIELDS:
        assert np.array_equal(orc.get_field(k), ref.get_field(k)), k
    assert np.abs(ref.get_field("interf")).max() > 0.0


MCC = dict(ramda=0.2, kapa=0.04, zmf=1.2, eps0=0.9, poi=0.3, sme0=50.0e3, ann=1.0, ocr=1.5, e=0.0, fs=1.0)


@needs_ref
@pytest.mark.parametrize("label,factory,steps", [
    ("camclay", lambda: scenes.set_soil_model(scenes.soil_column_3d(dx=0.05, steps=100), 1, **MCC), 20),
    ("camclay_2d", lambda: scenes.set_soil_model(scenes.slope_2d(H=1.0, dx=0.05), 1, **MCC), 30),
    ("mohr_coulomb", lambda: scenes.set_soil_model(scenes.soil_column_3d(dx=0.05, steps=100), 9,
                                                   c=0.0, fai=30.0, e=1.0e7), 20),
    ("mohr_coulomb_cohesive", lambda: scenes.set_soil_model(scenes.soil_column_3d(dx=0.05, steps=100), 9,
                                                            c=5.0e3, fai=25.0, e=1.0e7), 20),
    ("visco_elastic", lambda: scenes.set_soil_model(scenes.soil_column_3d(dx=0.05, steps=100), 7,
                                                    c=1.0e5, e=1.0e7), 20),
])
def test_live_reference_soil_models(label, factory, steps):
    """sub_camclay, elastic_plastic (M-C) and viscous_elastic
    (CPP_8-1-consfactor.cpp:88-281, 618-777): bit-identical to the reference;
    the plastic branch is reached for the Cam-clay and cohesionless M-C
    cases."""
    sc = factory()
    ref = _live(sc)
    fl, so = ref.materials()
    orc = Oracle(ref.params, ORC_INPLACE)
    orc.load_state({k: ref.get_field(k) for k in STATE_FIELDS}, fl, so)
    assert ref.step(steps) == 0
    assert orc.step(steps) == 0
    for k in STATE_FIELDS:
        assert np.array_equal(orc.get_field(k), ref.get_field(k)), k
    if label in ("camclay", "camclay_2d", "mohr_coulomb"):
        t = ref.get_field("type")
        assert (np.abs(ref.get_field("adps")[t == 2]).sum(axis=1) > 0).any()


@needs_ref
def test_live_reference_dam_break_full_size():
    """The 2-D dam break at its stated size (dx = 5 mm, 12,800 water and 2,178
    wall particles) for 200 steps: the oracle in the reference's sequential
    order is bit-identical to the reference."""
    sc = scenes.dam_break_2d(dx=0.005, steps=2000)
    ref = _live(sc)
    fl, so = ref.materials()
    orc = Oracle(ref.params, ORC_INPLACE)
    orc.load_state({k: ref.get_field(k) for k in STATE_FIELDS}, fl, so)
    assert ref.n == 14978
    assert ref.step(200) == 0
    assert orc.step(200) == 0
    for k in STATE_FIELDS:
        a, b = orc.get_field(k), ref.get_field(k)
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        assert same.all(), k
