"""ctypes bindings of the two checkers (test infrastructure only):

* ``Oracle``    -- oracle/liboracle.so, the C restatement of the reference's
                   step loop (sph_oracle.c);
* ``Reference`` -- oracle/_ref/libsphref.so, the reference solver compiled
                   from its own sources with ref_driver.cpp.  Present only
                   where it was built (from the reference tree).
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "multiphase-sph-solver_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)

import sphgpu  # noqa: E402
from sphgpu import FIELDS, INT_FIELDS, Params  # noqa: E402

ORACLE_SO = os.path.join(REPO, "oracle", "liboracle.so")
REF_SO = os.path.join(REPO, "oracle", "_ref", "libsphref.so")

ORC_JACOBI, ORC_INPLACE = 0, 1
ORC_POW_LIBM, ORC_POW_CR = 0, 1

ORACLE_FIELDS = dict(FIELDS)
ORACLE_FIELDS.update({"divx": 9, "deps": 6, "dsig": 6, "weps": 9,
                      "cd": 1, "beta": 9, "beta_ts": 9, "vel_bndy": 3, "vb_water": 3, "vb_soil": 3,
                      "vb_air": 3, "vb_struct": 3})


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


_olib = None


def oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_SO):
            raise FileNotFoundError(f"{ORACLE_SO} missing: run make -C oracle")
        lib = C.CDLL(ORACLE_SO)
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.POINTER(Params)]
        lib.orc_destroy.argtypes = [C.c_void_p]
        lib.orc_set_field.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_size_t]
        lib.orc_get_field.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_size_t]
        lib.orc_set_materials.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        lib.orc_kl_solve_wi.argtypes = [C.c_void_p, C.c_double * 3, C.c_double * 3, C.c_int, C.c_int]
        lib.orc_kl_ramdai.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double * 3, C.c_int, C.c_int]
        lib.orc_set_mode.argtypes = [C.c_void_p, C.c_int]
        lib.orc_set_pow_mode.argtypes = [C.c_void_p, C.c_int]
        lib.orc_pow7.restype = C.c_double
        lib.orc_pow7.argtypes = [C.c_double]
        lib.orc_get_step.argtypes = [C.c_void_p]
        lib.orc_nnps.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.orc_step.argtypes = [C.c_void_p, C.c_int]
        lib.orc_set_rain.argtypes = [C.c_void_p, C.c_void_p]
        lib.orc_rf_cholesky.restype = C.c_int
        lib.orc_get_rain.argtypes = [C.c_void_p, C.c_void_p]
        _olib = lib
    return _olib


class Oracle:
    def __init__(self, params: dict | Params, mode: int = ORC_JACOBI, pow_mode: int = ORC_POW_LIBM):
        self.lib = oracle_lib()
        self.params = params if isinstance(params, Params) else sphgpu.params_from_dict(params)
        self.h = C.c_void_p(self.lib.orc_create(C.byref(self.params)))
        if not self.h:
            raise RuntimeError("orc_create failed")
        self.n = int(self.params.ntotal)
        self.lib.orc_set_mode(self.h, mode)
        self.lib.orc_set_pow_mode(self.h, pow_mode)

    @property
    def step_index(self):
        return int(self.lib.orc_get_step(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def set_field(self, name, values):
        nc = ORACLE_FIELDS[name]
        dt = np.int32 if name in INT_FIELDS else np.float64
        a = np.ascontiguousarray(np.asarray(values, dtype=dt).reshape(self.n * nc))
        assert self.lib.orc_set_field(self.h, name.encode(), _ptr(a), a.size) == 0, name

    def get_field(self, name):
        nc = ORACLE_FIELDS[name]
        dt = np.int32 if name in INT_FIELDS else np.float64
        a = np.empty(self.n * nc, dtype=dt)
        assert self.lib.orc_get_field(self.h, name.encode(), _ptr(a), a.size) == 0, name
        return a if nc == 1 else a.reshape(self.n, nc)

    def set_materials(self, fluid, soil):
        fp = _ptr(np.ascontiguousarray(fluid)) if fluid is not None else None
        sp = _ptr(np.ascontiguousarray(soil)) if soil is not None else None
        assert self.lib.orc_set_materials(self.h, fp, sp, self.n) == 0

    def load_state(self, fields, fluid=None, soil=None, rain=None, vibration=None):
        for name, v in fields.items():
            if name in ORACLE_FIELDS:
                self.set_field(name, v)
        self.set_materials(fluid, soil)
        if rain is not None:
            self.set_rain(rain)
        if vibration is not None:
            self.set_vibration(vibration)

    def set_vibration(self, vib: dict) -> int:
        loads = np.ascontiguousarray(np.asarray(vib["loads"], dtype=np.float64).reshape(-1))
        return self.lib.orc_set_vibration(self.h, C.c_double(vib["ttime"]), C.c_int(int(vib["nsteps"])),
                                          C.c_double(vib["sttime"]), C.c_double(vib["edtime"]), _ptr(loads))

    def step(self, nsteps=1):
        return self.lib.orc_step(self.h, int(nsteps))

    def set_rain(self, rain: dict):
        r = sphgpu.rain_record(rain)
        assert self.lib.orc_set_rain(self.h, C.byref(r)) == 0

    def rain(self) -> dict:
        r = sphgpu.Rain()
        assert self.lib.orc_get_rain(self.h, C.byref(r)) == 0
        return {k: getattr(r, k) for k, _ in sphgpu.Rain._fields_}

    def nnps(self, with_wij=False):
        ninflu = np.zeros(self.n, np.int32)
        influ = np.zeros(self.n * 100, np.int32)
        wij = np.zeros(self.n * 400) if with_wij else None
        err = self.lib.orc_nnps(self.h, _ptr(ninflu), _ptr(influ), _ptr(wij) if with_wij else None)
        return err, ninflu, influ.reshape(self.n, 100), (wij.reshape(self.n, 100, 4) if with_wij else None)


SHIM_SO = os.path.join(REPO, "oracle", "_ref", "libsphshim.so")
_rlibs = {}


def have_reference() -> bool:
    return os.path.exists(REF_SO)


def have_shim() -> bool:
    return os.path.exists(SHIM_SO)


def reference_lib(so: str = REF_SO):
    """The reference driver library: REF_SO (the reference's own classes) or
    SHIM_SO (the same driver with the step classes of the engine's shim)."""
    if so not in _rlibs:
        lib = C.CDLL(so)
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.c_char_p, C.c_int]
        lib.ref_last_error.restype = C.c_int
        lib.ref_set_threads.argtypes = [C.c_void_p, C.c_int]
        lib.ref_get_params.argtypes = [C.c_void_p, C.POINTER(Params)]
        lib.ref_get_materials.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_get_field.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        lib.ref_particles.restype = C.c_void_p
        lib.ref_particles.argtypes = [C.c_void_p]
        lib.ref_particle_size.restype = C.c_size_t
        lib.ref_nnps.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_step.argtypes = [C.c_void_p, C.c_int]
        lib.ref_get_step.argtypes = [C.c_void_p]
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_get_rain.argtypes = [C.c_void_p, C.c_void_p]
        _rlibs[so] = lib
    return _rlibs[so]


class Reference:
    """The reference solver, initialised from an input.dat by its own code
    (with so=SHIM_SO: its step methods run on the GPU through the shim)."""

    def __init__(self, input_dat: str, nthreads: int = 1, so: str = REF_SO):
        self.lib = reference_lib(so)
        h = self.lib.ref_create(input_dat.encode(), int(nthreads))
        if not h:
            raise RuntimeError(f"ref_create failed: {self.lib.ref_last_error()}")
        self.h = C.c_void_p(h)
        self.params = Params()
        self.lib.ref_get_params(self.h, C.byref(self.params))
        self.n = int(self.params.ntotal)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    def get_field(self, name):
        nc = ORACLE_FIELDS[name]
        dt = np.int32 if name in INT_FIELDS else np.float64
        a = np.empty(self.n * nc, dtype=dt)
        assert self.lib.ref_get_field(self.h, name.encode(), _ptr(a)) == 0, name
        return a if nc == 1 else a.reshape(self.n, nc)

    def materials(self):
        from scenes import FLUID_DTYPE, SOIL_DTYPE
        fl = np.zeros(self.n, FLUID_DTYPE)
        so = np.zeros(self.n, SOIL_DTYPE)
        self.lib.ref_get_materials(self.h, _ptr(fl), _ptr(so))
        return fl, so

    def rain(self) -> dict:
        r = sphgpu.Rain()
        self.lib.ref_get_rain(self.h, C.byref(r))
        return {k: getattr(r, k) for k, _ in sphgpu.Rain._fields_}

    def set_threads(self, n):
        self.lib.ref_set_threads(self.h, int(n))

    def step(self, nsteps=1):
        return self.lib.ref_step(self.h, int(nsteps))

    def nnps(self, with_wij=False):
        ninflu = np.zeros(self.n, np.int32)
        influ = np.zeros(self.n * 100, np.int32)
        wij = np.zeros(self.n * 400) if with_wij else None
        err = self.lib.ref_nnps(self.h, _ptr(ninflu), _ptr(influ), _ptr(wij) if with_wij else None)
        return err, ninflu, influ.reshape(self.n, 100), (wij.reshape(self.n, 100, 4) if with_wij else None)

    def particles_bytes(self):
        size = self.lib.ref_particle_size()
        ptr = self.lib.ref_particles(self.h)
        return size, C.string_at(ptr, size * self.n)


STATE_FIELDS = ("x", "xp", "vx", "vxp", "ax", "axp", "ux", "strep", "interf", "interfss", "rho",
                "rhop", "mass", "hl", "pre", "prep", "e", "eps", "sig", "adps", "tssig", "tsqc", "satu", "dsatu", "suct", "cop",
                "vsig", "veps", "divq", "divr", "meps", "prew", "prea", "porosity", "poro_cop",
                "type", "matype", "permtype", "etype")


def snapshot(obj, names=STATE_FIELDS):
    return {k: obj.get_field(k) for k in names}


# --------------------------------------------------------------------------
# K-L random fields (CPP_17-1_K-L_expansion_non.cpp)

class OrcKLSpec(C.Structure):
    _fields_ = [("no", C.c_int), ("type", C.c_int), ("mean_value", C.c_double), ("sd_value", C.c_double),
                ("coe_depth", C.c_double), ("rl", C.c_double * 3), ("a", C.c_double * 3),
                ("x_trans", C.c_double * 3), ("soil_max", C.c_double), ("water_max", C.c_double)]


def kl_spec(field: dict, dom: dict) -> OrcKLSpec:
    s = OrcKLSpec()
    s.no, s.type = int(field["no"]), int(field["type"])
    s.mean_value, s.sd_value, s.coe_depth = field["mean"], field["sd"], field.get("coe_depth", 0.0)
    for d in range(3):
        s.rl[d] = field["rl"][d]
        s.a[d] = dom["a"][d]
        s.x_trans[d] = dom["x_trans"][d]
    s.soil_max, s.water_max = dom["soil_max"], dom["water_max"]
    return s


def kl_oracle(ndim, xp, ptype, field, dom, xi, K=200):
    """The oracle's field: (out, written, wi, eigval, order)."""
    lib = oracle_lib()
    n = len(ptype)
    xp = np.ascontiguousarray(xp, dtype=np.float64).reshape(n, 3)
    ptype = np.ascontiguousarray(ptype, dtype=np.int32)
    s = kl_spec(field, dom)
    wi = np.zeros((K, 3))
    lib.orc_kl_solve_wi(_ptr(wi), s.a, s.rl, C.c_int(ndim), C.c_int(K))
    eig = np.zeros(K)
    order = np.zeros((K, 3), np.int32)
    assert lib.orc_kl_ramdai(_ptr(eig), _ptr(order), _ptr(wi), s.rl, C.c_int(ndim), C.c_int(K)) == 0
    out = np.full(n, np.nan)
    written = np.zeros(n, np.int32)
    xi = np.ascontiguousarray(xi, dtype=np.float64)
    err = lib.orc_kl_field(C.c_int(ndim), C.c_int(n), _ptr(xp), _ptr(ptype), C.byref(s), _ptr(wi), _ptr(eig),
                           _ptr(order), _ptr(xi), C.c_int(K), _ptr(out), _ptr(written))
    assert err == 0
    out[written == 0] = np.nan
    return out, written, wi, eig, order


def kl_correlate(u2, coefficient, K=200):
    lib = oracle_lib()
    u2 = np.ascontiguousarray(u2, dtype=np.float64).reshape(K, 2)
    a, b = np.zeros(K), np.zeros(K)
    lib.orc_kl_correlate(_ptr(u2), C.c_double(coefficient), _ptr(a), _ptr(b), C.c_int(K))
    return a, b


def kl_reference(ndim, xp, ptype, field, dom, xi):
    """The reference's own solve_wi / solve_ramdai / solve_h (klterm = 200)."""
    lib = reference_lib()
    n = len(ptype)
    xp = np.ascontiguousarray(xp, dtype=np.float64).reshape(n, 3)
    ptype = np.ascontiguousarray(ptype, dtype=np.int32)
    out = np.zeros(n)
    wi, eig, order = np.zeros((200, 3)), np.zeros(200), np.zeros((200, 3), np.int32)
    rl = np.ascontiguousarray(field["rl"], dtype=np.float64)
    a = np.ascontiguousarray(dom["a"], dtype=np.float64)
    xt = np.ascontiguousarray(dom["x_trans"], dtype=np.float64)
    xi = np.ascontiguousarray(xi, dtype=np.float64)
    f = lib.ref_kl_field
    f.restype = C.c_int
    err = f(C.c_int(ndim), C.c_int(n), _ptr(xp), _ptr(ptype), C.c_int(int(field["no"])), C.c_int(int(field["type"])),
            C.c_double(field["mean"]), C.c_double(field["sd"]), C.c_double(field.get("coe_depth", 0.0)),
            _ptr(rl), _ptr(a), _ptr(xt), C.c_double(dom["soil_max"]), C.c_double(dom["water_max"]),
            _ptr(xi), _ptr(out), _ptr(wi), _ptr(eig), _ptr(order))
    assert err == 0
    return out, wi, eig, order


# --------------------------------------------------------------------------
# correlation-matrix (Cholesky) random fields (CPP_17-3-Nonstationary-RF.cpp)

class OrcRFSpec(C.Structure):
    _fields_ = [("no", C.c_int), ("type", C.c_int), ("mean_value", C.c_double), ("sd_value", C.c_double),
                ("coe_depth", C.c_double), ("rl", C.c_double * 3), ("cell_ndx", C.c_double),
                ("flag_auto", C.c_int), ("beta", C.c_double), ("beta_1", C.c_double),
                ("nb_min", C.c_double * 3), ("nb_max", C.c_double * 3), ("soil_max", C.c_double),
                ("water_max", C.c_double)]


def rf_spec(field: dict, dom: dict) -> OrcRFSpec:
    s = OrcRFSpec()
    s.no, s.type = int(field["no"]), int(field["type"])
    s.mean_value, s.sd_value, s.coe_depth = field["mean"], field["sd"], field.get("coe_depth", 0.0)
    for d in range(3):
        s.rl[d] = field["rl"][d]
        s.nb_min[d] = dom["nb_min"][d]
        s.nb_max[d] = dom["nb_max"][d]
    s.cell_ndx, s.flag_auto = field["cell_ndx"], int(field["flag_auto"])
    s.beta, s.beta_1 = field.get("beta", 0.0), field.get("beta_1", 0.0)
    s.soil_max, s.water_max = dom["soil_max"], dom["water_max"]
    return s


def rf_oracle(ndim, xp, ptype, dr, field, dom, zeta):
    """The oracle's correlation-matrix field: (code, out, number of cells)."""
    lib = oracle_lib()
    n = len(ptype)
    xp = np.ascontiguousarray(xp, dtype=np.float64).reshape(n, 3)
    ptype = np.ascontiguousarray(ptype, dtype=np.int32)
    zeta = np.ascontiguousarray(zeta, dtype=np.float64)
    out = np.zeros(n)
    ncell = C.c_int(0)
    s = rf_spec(field, dom)
    err = lib.orc_rf_cholesky(C.c_int(ndim), C.c_int(n), _ptr(xp), _ptr(ptype), C.c_double(dr), C.byref(s),
                              _ptr(zeta), C.c_int(len(zeta)), _ptr(out), C.byref(ncell))
    return err, out, ncell.value


def rf_oracle_corr(ndim, xp, ptype, dr, pair, coe, dom, u2):
    """The oracle's correlated field (flspv 4): (code, out 2 x n, cells).
    pair: the friction and cohesion field dicts; the cell and kernel keys are
    read from pair[0]."""
    lib = oracle_lib()
    n = len(ptype)
    xp = np.ascontiguousarray(xp, dtype=np.float64).reshape(n, 3)
    ptype = np.ascontiguousarray(ptype, dtype=np.int32)
    u2 = np.ascontiguousarray(u2, dtype=np.float64).reshape(-1, 2)
    out = np.zeros(2 * n)
    ncell = C.c_int(0)
    cells = {k: pair[0][k] for k in ("cell_ndx", "flag_auto", "beta", "beta_1") if k in pair[0]}
    s0, s1 = rf_spec(pair[0], dom), rf_spec(dict(pair[1], **cells), dom)
    lib.orc_rf_cholesky_corr.restype = C.c_int
    err = lib.orc_rf_cholesky_corr(C.c_int(ndim), C.c_int(n), _ptr(xp), _ptr(ptype), C.c_double(dr), C.byref(s0),
                                   C.byref(s1), C.c_double(coe), _ptr(u2), C.c_int(len(u2)), _ptr(out),
                                   C.byref(ncell))
    return err, out.reshape(2, n), ncell.value


def rv_oracle(ptype, pair, coe, u2):
    """The oracle's correlated random variables (flspv 5): out 2 x n."""
    lib = oracle_lib()
    n = len(ptype)
    ptype = np.ascontiguousarray(ptype, dtype=np.int32)
    u2 = np.ascontiguousarray(u2, dtype=np.float64)
    out = np.zeros(2 * n)
    dom = {"nb_min": [0, 0, 0], "nb_max": [0, 0, 0], "soil_max": 0.0, "water_max": 0.0}
    s0, s1 = rf_spec(dict(pair[0], cell_ndx=1.0, flag_auto=1), dom), rf_spec(dict(pair[1], cell_ndx=1.0, flag_auto=1), dom)
    lib.orc_rv_corr.restype = C.c_int
    err = lib.orc_rv_corr(C.c_int(n), _ptr(ptype), C.byref(s0), C.byref(s1), C.c_double(coe), _ptr(u2), _ptr(out))
    assert err == 0
    return out.reshape(2, n)


def _pair_arrays(pair):
    mean = np.array([pair[0]["mean"], pair[1]["mean"]], dtype=np.float64)
    sd = np.array([pair[0]["sd"], pair[1]["sd"]], dtype=np.float64)
    cd = np.array([pair[0].get("coe_depth", 0.0), pair[1].get("coe_depth", 0.0)], dtype=np.float64)
    return mean, sd, cd


def rf_reference_corr(ndim, xp, ptype, dr, pair, coe, dom, u2):
    """The reference's nonstationary_correlated_random_2D / _3D with the pair
    normals u2: (code, out 2 x n)."""
    lib = reference_lib()
    n = len(ptype)
    xp = np.ascontiguousarray(xp, dtype=np.float64).reshape(n, 3)
    ptype = np.ascontiguousarray(ptype, dtype=np.int32)
    u2 = np.ascontiguousarray(u2, dtype=np.float64).reshape(-1, 2)
    out = np.zeros(2 * n)
    f0 = pair[0]
    mean, sd, cd = _pair_arrays(pair)
    rl = np.ascontiguousarray(f0["rl"], dtype=np.float64)
    lo = np.ascontiguousarray(dom["nb_min"], dtype=np.float64)
    hi = np.ascontiguousarray(dom["nb_max"], dtype=np.float64)
    f = lib.ref_rf_cholesky_corr
    f.restype = C.c_int
    err = f(C.c_int(ndim), C.c_int(n), _ptr(xp), _ptr(ptype), C.c_double(dr), C.c_int(int(f0["no"])),
            C.c_int(int(f0["type"])), _ptr(mean), _ptr(sd), _ptr(cd), _ptr(rl), C.c_double(f0["cell_ndx"]),
            C.c_int(int(f0["flag_auto"])), C.c_double(f0.get("beta", 0.0)), C.c_double(f0.get("beta_1", 0.0)),
            C.c_double(coe), _ptr(lo), _ptr(hi), C.c_double(dom["soil_max"]), C.c_double(dom["water_max"]),
            _ptr(u2), C.c_int(len(u2)), _ptr(out))
    return err, out.reshape(2, n)


def rv_reference(ptype, pair, coe, u2):
    """The reference's random_variable_generate with the normals u2."""
    lib = reference_lib()
    n = len(ptype)
    ptype = np.ascontiguousarray(ptype, dtype=np.int32)
    u2 = np.ascontiguousarray(u2, dtype=np.float64)
    out = np.zeros(2 * n)
    mean, sd, _ = _pair_arrays(pair)
    f = lib.ref_rv_corr
    f.restype = C.c_int
    err = f(C.c_int(n), _ptr(ptype), C.c_int(int(pair[0]["no"])), C.c_int(int(pair[0]["type"])), _ptr(mean), _ptr(sd),
            C.c_double(coe), _ptr(u2), _ptr(out))
    assert err == 0
    return out.reshape(2, n)


def rf_reference(ndim, xp, ptype, dr, field, dom, zeta):
    """The reference's nonstationary_random_2D / _3D with the normals zeta."""
    lib = reference_lib()
    n = len(ptype)
    xp = np.ascontiguousarray(xp, dtype=np.float64).reshape(n, 3)
    ptype = np.ascontiguousarray(ptype, dtype=np.int32)
    zeta = np.ascontiguousarray(zeta, dtype=np.float64)
    out = np.zeros(n)
    rl = np.ascontiguousarray(field["rl"], dtype=np.float64)
    lo = np.ascontiguousarray(dom["nb_min"], dtype=np.float64)
    hi = np.ascontiguousarray(dom["nb_max"], dtype=np.float64)
    f = lib.ref_rf_cholesky
    f.restype = C.c_int
    err = f(C.c_int(ndim), C.c_int(n), _ptr(xp), _ptr(ptype), C.c_double(dr), C.c_int(int(field["no"])),
            C.c_int(int(field["type"])), C.c_double(field["mean"]), C.c_double(field["sd"]),
            C.c_double(field.get("coe_depth", 0.0)), _ptr(rl), C.c_double(field["cell_ndx"]),
            C.c_int(int(field["flag_auto"])), C.c_double(field.get("beta", 0.0)), C.c_double(field.get("beta_1", 0.0)),
            _ptr(lo), _ptr(hi), C.c_double(dom["soil_max"]), C.c_double(dom["water_max"]), _ptr(zeta),
            C.c_int(len(zeta)), _ptr(out))
    return err, out
