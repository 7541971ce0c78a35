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
rounded x^7, the engine's arithmetic) bit for bit, and the reference's within
the rounding of the C library's pow; the executables' result files must
agree to their printed precision.
"""
import glob
import os
import subprocess
import tempfile

import numpy as np
import pytest

import make_golden
import scenes
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
    if sync == "always":
        monkeypatch.setenv("SPHGPU_SHIM_SYNC", "always")
        path = _deck(factory(), steps, 100000)
    else:
        monkeypatch.delenv("SPHGPU_SHIM_SYNC", raising=False)
        path = _deck(factory(), steps, steps)
    shim = Reference(path, 1, so=SHIM_SO)
    fl, so = shim.materials()
    orc = Oracle(shim.params, ORC_JACOBI, ORC_POW_CR)
    orc.load_state({k: shim.get_field(k) for k in STATE_FIELDS}, fl, so)
    for chunk in (1, steps - 1):
        assert shim.step(chunk) == 0
        assert orc.step(chunk) == 0
    _compare(shim, orc, tol)
    del shim


@pytest.mark.skipif(not have_reference(), reason="reference not built here (oracle/_ref)")
@pytest.mark.parametrize("name", ["dam_break_2d", "soil_column_3d", "footing_2d_penalty_coupled"])
def test_shim_step_loop_matches_reference(name):
    """The same loop against the reference's own classes (which call the C
    library's pow): equal to LIBM_REL_TOL of each field's magnitude."""
    factory, steps, _ = CASES[name]
    path = _deck(factory(), steps, steps)
    ref = Reference(path, 1)
    shim = Reference(path, 1, so=SHIM_SO)
    assert ref.step(steps) == 0
    assert shim.step(steps) == 0
    worst = _compare(shim, ref, LIBM_REL_TOL)
    print(f"{name}: shim vs reference, worst relative difference {worst:.3g}")


def _read_odb(path):
    rows = []
    with open(path) as fh:
        for line in fh:
            if line.startswith("*"):
                continue
            rows.append([float(v) for v in line.split()])
    header, body = rows[0], np.array(rows[1:])
    return header, body


@pytest.mark.skipif(not (os.path.exists(SPH_REF_EXE) and os.path.exists(SPH_SHIM_EXE)),
                    reason="reference executables not built")
@pytest.mark.parametrize("name", ["dam_break_2d", "soil_column_3d"])
def test_sph_calculation_links_unchanged(name):
    """The reference's executable (CPP_0-main.cpp + SPH_Calculation) linked
    against the shim writes the same result files as the reference's own
    build: every data-*.odb with the same rows, to the 7 significant digits
    they are printed with."""
    factory, steps, _ = CASES[name]
    sc = factory()
    sc.loop = 12
    sc.problem["dttype"] = 1
    sc.dt = 0.25 * sc.dr / 600.0
    outs = {}
    for exe in (SPH_REF_EXE, SPH_SHIM_EXE):
        d = tempfile.mkdtemp(prefix="sphx", dir="/tmp")
        sc.problem["fop"] = 4
        scenes.write_input_dat(sc, os.path.join(d, "input.dat"))
        r = subprocess.run([exe, "-p", d], stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, timeout=600)
        assert r.returncode == 0, r.stderr.decode()[-2000:]
        outs[exe] = d
    ref_files = sorted(os.path.basename(p) for p in glob.glob(os.path.join(outs[SPH_REF_EXE], "data-*.odb")))
    shim_files = sorted(os.path.basename(p) for p in glob.glob(os.path.join(outs[SPH_SHIM_EXE], "data-*.odb")))
    assert ref_files == shim_files and len(ref_files) >= 3, (ref_files, shim_files)
    for f in ref_files:
        ha, a = _read_odb(os.path.join(outs[SPH_REF_EXE], f))
        hb, b = _read_odb(os.path.join(outs[SPH_SHIM_EXE], f))
        assert ha == hb
        assert a.shape == b.shape
        # one unit in the 7th printed digit, on values that may straddle a
        # rounding boundary of the print
        tol = 2e-6 * np.maximum(np.abs(a), np.abs(b)) + 1e-300
        bad = np.abs(a - b) > tol
        assert not bad.any(), (f, int(bad.sum()), np.argwhere(bad)[:5])
