"""Result files written while the steps go on (sphgpu_output_total,
sphgpu_output_step): the engine's data-*.odb files, and the appended "Flowing
distance.dat", AVS_MGF.mgf and Total_Force.dat with the Impact-force files,
must equal, byte for byte, the ones the reference's own output_total,
output_flowdist, mgf and output_impact (CPP_14-2-output.cpp, CPP_14-1-outmgf.cpp)
write from the same state -- here through the reference's executable linked
against the shim, which hands those functions the engine's state -- and a
file must hold the state of the step it was asked for even when later steps
run before it is written."""
import glob
import os
import subprocess
import tempfile

import numpy as np
import pytest

import scenes
import sphgpu
from checkers import REPO
from test_gpu_shim import _odb_rows, _read_odb

pytestmark = pytest.mark.gpu
SPH_SHIM_EXE = os.path.join(REPO, "oracle", "_ref", "sph_shim")


def _deck(sc):
    sc.loop = 12
    sc.problem["dttype"] = 1
    sc.dt = 0.25 * sc.dr / 600.0
    sc.problem["fop"] = 4
    return sc


def _impact(sc):
    sc.problem["if_cal"] = 1
    return sc


@pytest.mark.skipif(not os.path.exists(SPH_SHIM_EXE), reason="reference executables not built")
@pytest.mark.parametrize("factory", [lambda: scenes.dam_break_2d(dx=0.02, steps=100),
                                     lambda: _impact(scenes.soil_column_3d(dx=0.1, steps=200)),
                                     lambda: _impact(scenes.shaking_box(ndim=2, flv=1, dx=0.05))])
def test_output_files_equal_the_references(factory):
    sc = _deck(factory())
    ref_dir = tempfile.mkdtemp(prefix="sphr", dir="/tmp")
    scenes.write_input_dat(sc, os.path.join(ref_dir, "input.dat"))
    r = subprocess.run([SPH_SHIM_EXE, "-p", ref_dir], stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                       timeout=600)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    st = scenes.initialise(sc)
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil, vibration=st.vibration)
    out_dir = tempfile.mkdtemp(prefix="sphg", dir="/tmp")
    eng.output_begin(out_dir)
    done = 0
    impact = sc.problem["if_cal"] == 1
    for l in (1, 4, 8, 12):
        eng.step(l - done)
        done = l
        # what SPH_Calculation writes at an output step (CPP_1-SPHLoops.cpp:761-773)
        what = sphgpu.OUT_ODB | sphgpu.OUT_FLOWDIST | (sphgpu.OUT_IMPACT if impact else 0) | \
            (sphgpu.OUT_MGF if l != 1 else 0)
        eng.output_step(out_dir, what)
    eng.output_wait()
    eng.close()
    names = sorted(os.path.basename(p) for p in glob.glob(os.path.join(ref_dir, "data-*.odb")))
    assert names == sorted(os.path.basename(p) for p in glob.glob(os.path.join(out_dir, "data-*.odb")))
    assert len(names) == 4
    others = ["Flowing distance.dat", "AVS_MGF.mgf"]
    if impact:
        imp = sorted(os.path.basename(p) for p in glob.glob(os.path.join(ref_dir, "Impact-force*.inp")))
        assert len(imp) == 4
        others += ["Total_Force.dat"] + imp
    for f in names + others:
        a = open(os.path.join(ref_dir, f), "rb").read()
        b = open(os.path.join(out_dir, f), "rb").read()
        assert len(a) > 0 and a == b, f


def test_output_holds_its_step_while_later_steps_run():
    st = scenes.initialise(scenes.soil_column_3d(dx=0.05, steps=100))
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    out_dir = tempfile.mkdtemp(prefix="spho", dir="/tmp")
    eng.step(3)
    eng.output_total(out_dir)
    want = _odb_rows(eng)
    eng.step(10)
    eng.output_total(out_dir)
    eng.step(1)
    eng.output_total(out_dir)          # a third file waits for the first slot
    eng.output_wait()
    l, rows = _read_odb(os.path.join(out_dir, "data-0000000003.odb"))
    assert l == 3
    assert np.array_equal(rows, want)
    assert len(glob.glob(os.path.join(out_dir, "data-*.odb"))) == 3
    eng.close()
