"""The C ABI library without a GPU: it loads, exports every entry point
include/sphgpu.h declares, reports no device and refuses to create a context
(there is no CPU fallback), and its Particle record layout matches the
reference's Particle class."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import sphgpu
from checkers import have_reference

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "sphgpu.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sphgpu_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = sphgpu.load_library()
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_error_strings():
    lib = sphgpu.load_library()
    assert lib.sphgpu_abi_version() == 1
    for code in (0, 3, 5, 100, 101, 102, 103, 104):
        assert lib.sphgpu_error_string(code)


@pytest.mark.skipif(sphgpu.load_library().sphgpu_device_count() > 0, reason="a GPU is present")
def test_no_device_no_context():
    lib = sphgpu.load_library()
    import scenes
    st = scenes.initialise(scenes.dam_break_2d(dx=0.04, steps=10))
    p = sphgpu.params_from_dict(st.params)
    assert not lib.sphgpu_create(C.byref(p), 0)
    assert lib.sphgpu_last_create_error() == 102
    with pytest.raises(sphgpu.SPHError):
        sphgpu.Engine(st.params)


def test_unsupported_flags_rejected():
    """Flag combinations outside the engine's set fail loudly at create
    (checked before the device query)."""
    lib = sphgpu.load_library()
    import scenes
    st = scenes.initialise(scenes.dam_break_2d(dx=0.04, steps=10))
    for key, val in (("flbndy", 6), ("ss_type", 4), ("flv", 3), ("flv", -1), ("if_move", 4), ("flknl", 5)):
        d = dict(st.params)
        d[key] = val
        p = sphgpu.params_from_dict(d)
        assert not lib.sphgpu_create(C.byref(p), 0)
        assert lib.sphgpu_last_create_error() == 103, key


def test_field_table_matches_python_binding():
    lib = sphgpu.load_library()
    for name, nc in sphgpu.FIELDS.items():
        n, t = C.c_int(), C.c_int()
        assert lib.sphgpu_field_info(name.encode(), C.byref(n), C.byref(t)) == 0, name
        assert n.value == nc and t.value == (1 if name in sphgpu.INT_FIELDS else 0), name


@pytest.mark.skipif(not have_reference(), reason="reference not built here (oracle/_ref)")
def test_particle_layout_matches_reference_class():
    """Every member the record upload/download touches sits at the offset the
    reference's compiled Particle class puts it (sizeof(Particle) == 1064)."""
    import tempfile
    import scenes
    from checkers import Reference
    lib = sphgpu.load_library()
    sc = scenes.soil_column_3d(dx=0.1, steps=10)
    d = tempfile.mkdtemp()
    scenes.write_input_dat(sc, os.path.join(d, "input.dat"))
    ref = Reference(os.path.join(d, "input.dat"), 1)
    ref.step(2)
    size, raw = ref.particles_bytes()
    assert size == 1064
    recs = np.frombuffer(raw, dtype=np.uint8).reshape(ref.n, size)
    checked = 0
    for name, nc in sphgpu.FIELDS.items():
        off, ncomp = C.c_size_t(), C.c_int()
        assert lib.sphgpu_particle_layout(name.encode(), C.byref(off), C.byref(ncomp)) == 0, name
        assert ncomp.value == nc
        dt = np.int32 if name in sphgpu.INT_FIELDS else np.float64
        width = nc * np.dtype(dt).itemsize
        got = recs[:, off.value:off.value + width].copy().view(dt).reshape(ref.n, nc)
        want = ref.get_field(name).reshape(ref.n, nc)
        assert np.array_equal(got, want), name
        checked += 1
    assert checked == len(sphgpu.FIELDS)


def test_header_compiles_as_c_and_links(tmp_path):
    """include/sphgpu.h is plain C: a C99 program that takes the address of
    every entry point it declares compiles, links against libsphgpu.so and
    runs without a GPU (no device, no context)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    names = _declared()
    src = tmp_path / "abi.c"
    lines = ['#include <stdio.h>', '#include "sphgpu.h"', "int main(void) {",
             "    void* const table[] = {"]
    lines += ["        (void*)&%s," % n for n in names]
    lines += ["    };",
              '    printf("%d %d %zu\\n", sphgpu_abi_version(), sphgpu_device_count(), sizeof(table) / sizeof(table[0]));',
              "    return sphgpu_create(NULL, 0) == NULL ? 0 : 1;", "}"]
    src.write_text("\n".join(lines) + "\n")
    lib_dir = os.path.dirname(sphgpu.LIB_PATH)
    exe = tmp_path / "abi"
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"), str(src), "-o",
                    str(exe), "-L", lib_dir, "-lsphgpu", "-Wl,-rpath," + lib_dir], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert int(out[0]) == sphgpu.load_library().sphgpu_abi_version()
    assert int(out[2]) == len(names)
