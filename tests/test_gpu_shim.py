"""The reference's own step loop on the GPU through the shim classes.

multiphase-sph-solver_b200/shim/sph_shim.cpp defines the reference's step
classes (clNNPS_Fun, clDensity_Fun, clStraStre_Fun, clInterFor_Fun,
clAcce_Fun, clVel_Fun, clUpdate_Fun::update, clBndy_Fun, clSoilStruct_Fun)
with the signatures of its Class_Functions.h over the sphgpu C ABI.
oracle/Makefile links it, in place of the reference's hot-path translation
units, into

* oracle/_ref/libsphshim.so: the reference's initialisation and the step body
  of ref_driver.cpp, which calls the classes in SPH_Calculation's order
  (CPP_1-SPHLoops.cpp:523-753);
* oracle/_ref/sph_shim: the reference's own executable, CPP_0-main.cpp and
  SPH_Calculation unchanged, beside oracle/_ref/sph_ref, the same executable
  with the reference's classes.

Through the shim the state must equal the oracle's (Jacobi order, correctly
rounded x^7, the engine's arithmetic) bit for bit, and the engine's when it is
driven directly; the executable's result files must hold the engine's values
as printed.  (The reference's own classes differ from all three by the order
of their in-place Shepard pass, which the engine and the oracle replace with
the order-free form.)
"""
import glob
import os
import subprocess
import tempfile

import numpy as np
import pytest

import make_golden
import scenes
import sphgpu
from checkers import (ORC_JACOBI, ORC_POW_CR, REPO, SHIM_SO, STATE_FIELDS, Oracle, Reference, have_reference,
                      have_shim)

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_shim(), reason="oracle/_ref/libsphshim.so not built (reference tree)")]

LIBM_REL_TOL = 1e-9
SPH_REF_EXE = os.path.join(REPO, "oracle", "_ref", "sph_ref")
SPH_SHIM_EXE = os.path.join(REPO, "oracle", "_ref", "sph_shim")

# name: (scene factory, steps, tolerance against the CR oracle; 0 = bit-identical)
CASES = {
    "dam_break_2d": (lambda: scenes.dam_break_2d(dx=0.02, steps=100), 15, 0.0),
    "soil_column_3d": (lambda: scenes.soil_column_3d(dx=0.1, steps=200), 10, 0.0),
    "dam_break_2d_tm_boundary": (make_golden.CASES["dam_break_2d_dx0.04_tm_boundary"][0], 12, 0.0),
    "soil_column_3d_no_slip_vsd": (make_golden.CASES["soil_column_3d_dx0.1_no_slip_vsd"][0], 10, 0.0),
    "footing_2d_penalty_coupled": (make_golden.CASES["footing_2d_penalty_coupled"][0], 12, 0.0),
    "three_phase_minor": (make_golden.CASES["three_phase_column_3d_dx0.1_minor"][0], 10, 0.0),
    "geostatic": (make_golden.CASES["soil_column_3d_dx0.1_geostatic"][0], 10, 0.0),
    "drag_peng": (make_golden.CASES["soil_column_3d_dx0.1_drag_peng"][0], 8, 1e-12),
    "kgc_regu": (make_golden.CASES["soil_column_3d_dx0.1_kgc_regu"][0], 8, 0.0),
    "shaking_box_2d_flv1": (make_golden.CASES["shaking_box_2d_flv1"][0], 20, 0.0),
    "shaking_box_3d_flv2": (make_golden.CASES["shaking_box_3d_flv2"][0], 15, 0.0),
}


def _deck(sc, steps, fop):
    sc.problem["fop"] = fop
    d = tempfile.mkdtemp(prefix="sph", dir="/tmp")
    path = os.path.join(d, "input.dat")
    scenes.write_input_dat(sc, path)
    return path


def _compare(a_obj, b_obj, tol):
    worst = 0.0
    for name in STATE_FIELDS:
        a, b = a_obj.get_field(name), b_obj.get_field(name)
        if a.dtype.kind != "f":
            assert np.array_equal(a, b), name
            continue
        assert np.array_equal(np.isnan(a), np.isnan(b)), name
        if tol == 0.0:
            same = (a == b) | (np.isnan(a) & np.isnan(b))
            assert same.all(), (name, int((~same).sum()))
            continue
        if name == "divr" or not b.size:
            continue
        scale = max(float(np.nanmax(np.abs(b))), 1e-300)
        err = float(np.nanmax(np.abs(a - b))) / scale
        worst = max(worst, err)
        assert err <= tol, (name, err)
    return worst


@pytest.mark.parametrize("sync", ["output", "always"])
@pytest.mark.parametrize("name", list(CASES))
def test_shim_step_loop_matches_oracle(name, sync, monkeypatch):
    """ref_driver.cpp's step body (SPH_Calculation's call order) with the
    shim classes: every field the host copy holds after the last step equals
    the oracle's.  sync 'output': the shim downloads only on output steps
    (the last step is one here); 'always': upload and download every step."""
    factory, steps, tol = CASES[name]
    sc = factory()
    if sync == "always":
        monkeypatch.setenv("SPHGPU_SHIM_SYNC", "always")
        path = _deck(sc, steps, 100000)
    else:
        monkeypatch.delenv("SPHGPU_SHIM_SYNC", raising=False)
        path = _deck(sc, steps, steps)
    shim = Reference(path, 1, so=SHIM_SO)
    fl, so = shim.materials()
    orc = Oracle(shim.params, ORC_JACOBI, ORC_POW_CR)
    orc.load_state({k: shim.get_field(k) for k in STATE_FIELDS}, fl, so,
                   vibration=sc.vibration if sc.flags.get("flv", 0) >= 1 else None)
    for chunk in (1, steps - 1):
        assert shim.step(chunk) == 0
        assert orc.step(chunk) == 0
    _compare(shim, orc, tol)
    del shim


@pytest.mark.parametrize("name", ["dam_break_2d", "soil_column_3d", "footing_2d_penalty_coupled"])
def test_shim_step_loop_matches_direct_engine(name):
    """The same loop against the engine driven directly through its C ABI
    from the same initial state: the shim adds nothing to the arithmetic, so
    every field is bit-identical."""
    factory, steps, _ = CASES[name]
    path = _deck(factory(), steps, steps)
    shim = Reference(path, 1, so=SHIM_SO)
    fl, so = shim.materials()
    init = {k: shim.get_field(k) for k in STATE_FIELDS}
    params = shim.params
    assert shim.step(steps) == 0
    got = {k: shim.get_field(k) for k in STATE_FIELDS}
    del shim
    eng = sphgpu.Engine(params, device=0)
    eng.load_state(init, fl, so)
    eng.step(steps)
    for k in STATE_FIELDS:
        a, b = got[k], eng.get_field(k)
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        assert same.all(), (name, k)
    eng.close()


def _read_odb(path):
    """A data-*.odb file of output_total (CPP_14-2-output.cpp:15-136): the step
    number and the particle rows as numbers."""
    rows = []
    with open(path) as fh:
        for line in fh:
            if line.startswith("*"):
                continue
            rows.append([float(v) for v in line.split()])
    return int(rows[0][0]), np.array(rows[1:])


def _odb_rows(eng):
    """The rows output_total prints for the engine's state, each value passed
    through the same %14.6e conversion."""
    t = eng.get_field("type")
    ux = eng.get_field("ux")
    umag = np.sqrt(ux[:, 0] * ux[:, 0] + ux[:, 1] * ux[:, 1] + ux[:, 2] * ux[:, 2])
    moving = (t != 0)[:, None]
    a3 = np.where(moving, eng.get_field("ax"), eng.get_field("interfss"))
    v3 = np.where(moving, eng.get_field("vx"), eng.get_field("interf"))
    one = lambda k: eng.get_field(k)[:, None]
    cols = [eng.get_field("xp"), ux, umag[:, None], a3, v3, one("pre"), one("prea"), one("prew"),
            eng.get_field("sig"), eng.get_field("strep"), eng.get_field("eps"), eng.get_field("adps"),
            one("vsig"), one("veps"), one("meps"), one("divq"), one("divr"), one("satu"), one("suct"),
            eng.get_field("interfss")]
    vals = np.concatenate(cols, axis=1)
    printed = np.vectorize(lambda v: float("%14.6e" % v))(vals)
    n = len(t)
    return np.concatenate([np.arange(1, n + 1)[:, None], printed, t[:, None], eng.get_field("matype")[:, None]],
                          axis=1)


@pytest.mark.skipif(not os.path.exists(SPH_SHIM_EXE), reason="reference executables not built")
@pytest.mark.parametrize("name", ["dam_break_2d", "soil_column_3d"])
def test_sph_calculation_links_unchanged(name):
    """The reference's executable (CPP_0-main.cpp and SPH_Calculation,
    unchanged) linked against the shim: its result files (data-*.odb of
    output_total, written at steps 1, 4, 8 and 12) hold exactly the values the
    engine reaches when driven directly from the same deck, as printed."""
    factory, steps, _ = CASES[name]
    sc = factory()
    sc.loop = 12
    sc.problem["dttype"] = 1
    sc.dt = 0.25 * sc.dr / 600.0
    sc.problem["fop"] = 4
    d = tempfile.mkdtemp(prefix="sphx", dir="/tmp")
    scenes.write_input_dat(sc, os.path.join(d, "input.dat"))
    r = subprocess.run([SPH_SHIM_EXE, "-p", d], stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, timeout=600)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    files = sorted(glob.glob(os.path.join(d, "data-*.odb")))
    assert [os.path.basename(f) for f in files] == ["data-0000000001.odb", "data-0000000004.odb",
                                                    "data-0000000008.odb", "data-0000000012.odb"]
    st = scenes.initialise(sc)
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    done = 0
    for f in files:
        l, rows = _read_odb(f)
        eng.step(l - done)
        done = l
        want = _odb_rows(eng)
        assert rows.shape == want.shape, f
        assert np.array_equal(rows, want), (f, int((rows != want).sum()))
    eng.close()
