"""Python host binding of the sphgpu C ABI (include/sphgpu.h).

This is the call a Python user makes: build a parameter record, create an
engine on a device, upload the particle state and the per-particle material
records, and step.  The shared library is the in-tree
``multiphase-sph-solver_b200/libsphgpu.so`` built by ``build.py``; importing
this module does not load it, constructing an ``Engine`` does, and raises if
it is missing or no CUDA device is present (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SPHGPU_LIB", os.path.join(HERE, "libsphgpu.so"))

FLUID_FIELDS = ("vis", "vpu", "dens", "paa0", "porosity", "fai", "c",
                "bhtype", "press_type", "acc_type", "pre_coe", "strain_min")
_FLUID_INTS = {"bhtype", "press_type", "acc_type"}


class Fluid(C.Structure):
    _fields_ = [(k, C.c_int if k in _FLUID_INTS else C.c_double) for k in FLUID_FIELDS]


SOIL_FIELDS = ("e", "poi", "eps0", "dens", "damp1", "damp2", "cop", "ramda", "kapa", "zmf",
               "ann", "bnn", "beta", "sitas", "sitar", "epsr", "epss", "sd", "sw", "kse",
               "c1", "c2", "c3", "fai", "c", "ocr", "sme0", "mzm", "azm", "r0",
               "bl", "bz", "zet", "vpu", "porosity", "fs", "etao", "g0", "ds", "damp_coe")


class Soil(C.Structure):
    _fields_ = [(k, C.c_double) for k in SOIL_FIELDS]


class Structure(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("dens", "eps0", "e", "poi", "vpu", "porosity", "cop")]


class Params(C.Structure):
    _fields_ = [
        ("ndim", C.c_int), ("ntotal", C.c_int),
        ("fla", C.c_int), ("fls", C.c_int), ("flr", C.c_int), ("fli", C.c_int), ("flv", C.c_int),
        ("fleob", C.c_int), ("flts", C.c_int), ("flspv", C.c_int), ("flknl", C.c_int), ("flbndy", C.c_int),
        ("inip", C.c_int), ("step_regu", C.c_int), ("loop", C.c_int), ("fop", C.c_int),
        ("dr", C.c_double), ("dt", C.c_double),
        ("xsph", C.c_double * 3),
        ("art_vis", (C.c_double * 2) * 3),
        ("art_stre_coe", C.c_double),
        ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double),
        ("threshold_min", C.c_double), ("threshold_max", C.c_double),
        ("interc", C.c_double), ("permtype", C.c_int),
        ("pers", C.c_double), ("perl", C.c_double), ("perm", C.c_double),
        ("ss_type", C.c_int), ("ss_myu", C.c_double), ("ss_zeta", C.c_double), ("ss_acc_type", C.c_int),
        ("coe_bndy", C.c_double), ("if_cal", C.c_int), ("if_move", C.c_int),
        ("move_vx", C.c_double * 3),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
        ("zmin", C.c_double), ("zmax", C.c_double),
        ("cxm", C.c_int), ("cym", C.c_int), ("czm", C.c_int), ("ctotal", C.c_int),
        ("flagum", C.c_int), ("alphats", C.c_double),
        ("water_acc_type", C.c_int), ("air_acc_type", C.c_int),
        ("structure", Structure),
    ]


class Instance(C.Structure):
    """sphgpu_instance: one instance of a batched context."""
    _fields_ = [("first", C.c_int), ("count", C.c_int),
                ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
                ("zmin", C.c_double), ("zmax", C.c_double),
                ("cxm", C.c_int), ("cym", C.c_int), ("czm", C.c_int), ("ctotal", C.c_int)]


class Rain(C.Structure):
    """sphgpu_rain: the reference's Para_Rain as the step uses it."""
    _fields_ = [("rtype", C.c_int), ("nrain", C.c_int), ("nhor", C.c_int),
                ("press_factor", C.c_double), ("drop_velocity", C.c_double)]


def rain_record(d: dict) -> Rain:
    return Rain(int(d["rtype"]), int(d["nrain"]), int(d["nhor"]), float(d["press_factor"]),
                float(d["drop_velocity"]))


def params_from_dict(d: dict) -> Params:
    p = Params()
    for name, ctype in Params._fields_:
        if name not in d:
            continue
        v = d[name]
        if name == "xsph" or name == "move_vx":
            for k in range(3):
                getattr(p, name)[k] = float(v[k])
        elif name == "art_vis":
            for a in range(3):
                for b in range(2):
                    p.art_vis[a][b] = float(v[a][b])
        elif name == "structure":
            for k, _ in Structure._fields_:
                setattr(p.structure, k, float(v.get(k, 0.0)))
        else:
            setattr(p, name, v if ctype is C.c_int else float(v))
    return p


def params_to_dict(p: Params) -> dict:
    d = {}
    for name, ctype in Params._fields_:
        v = getattr(p, name)
        if name in ("xsph", "move_vx"):
            v = tuple(v[k] for k in range(3))
        elif name == "art_vis":
            v = tuple(tuple(v[a][b] for b in range(2)) for a in range(3))
        elif name == "structure":
            v = {k: getattr(v, k) for k, _ in Structure._fields_}
        d[name] = v
    return d


# Particle members the engine transfers: name -> components.  Integers are
# the four trailing members of Particle (Class_particle.h:87-94).
FIELDS = {
    "x": 3, "xp": 3, "vx": 3, "vxp": 3, "ax": 3, "axp": 3, "ux": 3, "strep": 3,
    "interf": 3, "interfss": 3, "rho": 1, "rhop": 1, "mass": 1, "hl": 1, "pre": 1, "prep": 1,
    "e": 1, "eps": 6, "sig": 6, "adps": 6, "tssig": 6, "tsqc": 1, "satu": 1, "dsatu": 1,
    "suct": 1, "cop": 1, "vsig": 1, "veps": 1,
    "divq": 1, "divr": 1, "meps": 1, "prew": 1, "prea": 1, "porosity": 1, "poro_cop": 1,
    "cd": 1, "type": 1, "matype": 1, "permtype": 1, "etype": 1,
}
INT_FIELDS = {"type", "matype", "permtype", "etype"}

PARTICLE_BYTES = 1064  # sizeof(Particle) of the reference (Class_particle.h)


def particle_records(fields: dict, n: int, stride: int = PARTICLE_BYTES) -> np.ndarray:
    """Particle records (n x stride bytes, zero elsewhere) holding `fields`
    at the offsets sphgpu_particle_layout reports, as the reference's own
    Particle array would hold them."""
    lib = load_library()
    buf = np.zeros(n * stride, np.uint8)
    for name, v in fields.items():
        if name not in FIELDS:
            continue
        off, nc = C.c_size_t(), C.c_int()
        if lib.sphgpu_particle_layout(name.encode(), C.byref(off), C.byref(nc)) != 0:
            continue
        dt = np.int32 if name in INT_FIELDS else np.float64
        a = np.ascontiguousarray(np.asarray(v, dtype=dt).reshape(n, nc.value))
        view = np.lib.stride_tricks.as_strided(buf[off.value:], shape=(n, a.itemsize * nc.value),
                                               strides=(stride, 1))
        view[:] = a.view(np.uint8).reshape(n, a.itemsize * nc.value)
    return buf


PREC_FP64 = 0          # SPHGPU_PREC_FP64
PREC_FP32_BULK = 1     # SPHGPU_PREC_FP32_BULK

class KLField(C.Structure):
    """sphgpu_kl_field: Para_SpatialVariability's members the K-L generators read."""
    _fields_ = [("no", C.c_int), ("type", C.c_int), ("mean_value", C.c_double), ("sd_value", C.c_double),
                ("rl_value", C.c_double * 3), ("coe_depth", C.c_double)]


class KLDomain(C.Structure):
    """sphgpu_kl_domain: the Cell_Con members the K-L generators read."""
    _fields_ = [("xmin_nb", C.c_double), ("xmax_nb", C.c_double), ("ymin_nb", C.c_double),
                ("ymax_nb", C.c_double), ("zmin_nb", C.c_double), ("zmax_nb", C.c_double),
                ("soil_max", C.c_double * 3), ("water_max", C.c_double * 3)]


def kl_field(no: int, type: int, mean: float, sd: float, rl, coe_depth: float = 0.0) -> KLField:
    f = KLField()
    f.no, f.type, f.mean_value, f.sd_value, f.coe_depth = int(no), int(type), float(mean), float(sd), float(coe_depth)
    for d in range(3):
        f.rl_value[d] = float(rl[d]) if d < len(rl) else 0.0
    return f


def kl_domain(nb_min, nb_max, soil_max, water_max) -> KLDomain:
    """soil_max / water_max: 3 values each, or one value for the depth axis
    (y in 2-D, z in 3-D), which is the only component the generators read."""
    d = KLDomain()
    d.xmin_nb, d.ymin_nb, d.zmin_nb = (float(v) for v in nb_min)
    d.xmax_nb, d.ymax_nb, d.zmax_nb = (float(v) for v in nb_max)
    for k in range(3):
        d.soil_max[k] = float(soil_max[k]) if hasattr(soil_max, "__len__") else float(soil_max)
        d.water_max[k] = float(water_max[k]) if hasattr(water_max, "__len__") else float(water_max)
    return d


OUT_ODB, OUT_FLOWDIST, OUT_IMPACT, OUT_MGF = 1, 2, 4, 8


class Vibration(C.Structure):
    """sphgpu_vibration: Para_Vibra without its loads."""
    _fields_ = [("ttime", C.c_double), ("nsteps", C.c_int), ("sttime", C.c_double), ("edtime", C.c_double)]


class RFFlags(C.Structure):
    """sphgpu_rf_flags: the Flag_SpatialVariability members the correlation-
    matrix generators read."""
    _fields_ = [("cell_ndx", C.c_double), ("flag_auto", C.c_int), ("beta", C.c_double), ("beta_1", C.c_double),
                ("coe_frict_cohesion", C.c_double)]


def rf_flags(cell_ndx: float, flag_auto: int = 1, beta: float = 0.0, beta_1: float = 0.0,
             coe_frict_cohesion: float = 0.0) -> RFFlags:
    f = RFFlags()
    f.cell_ndx, f.flag_auto, f.beta, f.beta_1 = float(cell_ndx), int(flag_auto), float(beta), float(beta_1)
    f.coe_frict_cohesion = float(coe_frict_cohesion)
    return f


ERRORS = {0: "ok", 3: "particle outside the cell grid", 41: "no random-field cells, or 15,000 or more",
          42: "a random-field cell holds more than 39 particles", 5: "more than 99 neighbours",
          100: "bad argument", 101: "CUDA error", 102: "no CUDA device", 103: "unsupported flags",
          104: "call order", 105: "tensor-core wait expired", 106: "index check failed (bounds-checked build)"}


class SPHError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: error {code} ({ERRORS.get(code, 'unknown')})")
        self.code = code


_lib = None


CHECK_LIB_PATH = os.path.join(HERE, "libsphgpu_check.so")
_libs: dict = {}


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libsphgpu.so, or another build of it such as the bounds-checked
    libsphgpu_check.so (raises if it was not built)."""
    global _lib
    if path == LIB_PATH and _lib is not None:
        return _lib
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built; run __graft_entry__.build()")
    lib = C.CDLL(path)
    lib.sphgpu_abi_version.restype = C.c_int
    lib.sphgpu_device_count.restype = C.c_int
    lib.sphgpu_error_string.restype = C.c_char_p
    lib.sphgpu_error_string.argtypes = [C.c_int]
    lib.sphgpu_create.restype = C.c_void_p
    lib.sphgpu_create.argtypes = [C.POINTER(Params), C.c_int]
    lib.sphgpu_last_create_error.restype = C.c_int
    lib.sphgpu_destroy.argtypes = [C.c_void_p]
    lib.sphgpu_get_params.argtypes = [C.c_void_p, C.POINTER(Params)]
    lib.sphgpu_get_step.argtypes = [C.c_void_p]
    lib.sphgpu_set_step.argtypes = [C.c_void_p, C.c_int]
    lib.sphgpu_field_info.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.sphgpu_set_field.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_size_t]
    lib.sphgpu_get_field.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_size_t]
    lib.sphgpu_set_materials.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    lib.sphgpu_upload_particles.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_size_t]
    lib.sphgpu_particle_layout.argtypes = [C.c_char_p, C.POINTER(C.c_size_t), C.POINTER(C.c_int)]
    lib.sphgpu_download_particles.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_size_t]
    lib.sphgpu_step.argtypes = [C.c_void_p, C.c_int]
    lib.sphgpu_nnps.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.sphgpu_synchronize.argtypes = [C.c_void_p]
    lib.sphgpu_last_step_ms.restype = C.c_double
    lib.sphgpu_last_step_ms.argtypes = [C.c_void_p]
    lib.sphgpu_last_step_launches.restype = C.c_long
    lib.sphgpu_last_step_launches.argtypes = [C.c_void_p]
    lib.sphgpu_stream.restype = C.c_void_p
    lib.sphgpu_stream.argtypes = [C.c_void_p]
    lib.sphgpu_stage_count.restype = C.c_int
    lib.sphgpu_stage_name.restype = C.c_char_p
    lib.sphgpu_stage_name.argtypes = [C.c_int]
    lib.sphgpu_step_profiled.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    lib.sphgpu_set_precision.argtypes = [C.c_void_p, C.c_int]
    lib.sphgpu_set_cfl.argtypes = [C.c_void_p, C.c_double, C.c_double]
    lib.sphgpu_get_dt.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    lib.sphgpu_kl_generate.argtypes = [C.c_void_p, C.POINTER(KLDomain), C.POINTER(KLField), C.c_int, C.c_void_p,
                                       C.c_int, C.c_void_p]
    lib.sphgpu_set_vibration.argtypes = [C.c_void_p, C.POINTER(Vibration), C.c_void_p]
    lib.sphgpu_rf_cells.argtypes = [C.c_void_p, C.POINTER(KLDomain), C.POINTER(RFFlags), C.POINTER(C.c_int)]
    lib.sphgpu_rf_generate.argtypes = [C.c_void_p, C.POINTER(KLDomain), C.POINTER(KLField), C.c_int,
                                       C.POINTER(RFFlags), C.c_void_p, C.c_int, C.c_void_p]
    lib.sphgpu_rf_generate_corr.argtypes = [C.c_void_p, C.POINTER(KLDomain), C.POINTER(KLField), C.POINTER(RFFlags),
                                            C.c_void_p, C.c_int, C.c_void_p]
    lib.sphgpu_rv_generate_corr.argtypes = [C.c_void_p, C.POINTER(KLField), C.c_double, C.c_void_p, C.c_void_p]
    lib.sphgpu_kl_synthesize.argtypes = [C.c_void_p, C.POINTER(KLDomain), C.POINTER(KLField), C.c_void_p, C.c_int,
                                         C.c_int, C.c_void_p, C.POINTER(C.c_double)]
    lib.sphgpu_kl_generate_corr.argtypes = [C.c_void_p, C.POINTER(KLDomain), C.POINTER(KLField), C.c_double,
                                            C.c_void_p, C.c_int, C.c_void_p]
    lib.sphgpu_get_precision.argtypes = [C.c_void_p]
    lib.sphgpu_create_batched.restype = C.c_void_p
    lib.sphgpu_create_batched.argtypes = [C.POINTER(Params), C.POINTER(Instance), C.c_int, C.c_int]
    lib.sphgpu_instance_count.argtypes = [C.c_void_p]
    lib.sphgpu_kl_generate_batched.argtypes = [C.c_void_p, C.POINTER(KLDomain), C.POINTER(KLField), C.c_void_p,
                                               C.c_int, C.c_void_p]
    lib.sphgpu_update_params.argtypes = [C.c_void_p, C.POINTER(Params)]
    lib.sphgpu_pipe_peaks.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.sphgpu_set_reorder.argtypes = [C.c_void_p, C.c_int]
    lib.sphgpu_get_reorder.argtypes = [C.c_void_p]
    lib.sphgpu_get_order.argtypes = [C.c_void_p, C.c_void_p]
    lib.sphgpu_autotune_reorder.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_void_p]
    lib.sphgpu_last_reorder_ms.restype = C.c_double
    lib.sphgpu_last_reorder_ms.argtypes = [C.c_void_p]
    lib.sphgpu_parttocell.argtypes = [C.c_void_p]
    lib.sphgpu_partisearching.argtypes = [C.c_void_p]
    lib.sphgpu_update.argtypes = [C.c_void_p]
    lib.sphgpu_kl_wait_check.argtypes = [C.c_void_p, C.c_longlong]
    lib.sphgpu_set_rain.argtypes = [C.c_void_p, C.POINTER(Rain)]
    lib.sphgpu_set_launch.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.sphgpu_get_launch.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.sphgpu_autotune.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_void_p]
    lib.sphgpu_output_total.argtypes = [C.c_void_p, C.c_char_p]
    lib.sphgpu_output_wait.argtypes = [C.c_void_p]
    lib.sphgpu_output_begin.argtypes = [C.c_void_p, C.c_char_p]
    lib.sphgpu_output_step.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
    lib.sphgpu_checkpoint_save.argtypes = [C.c_void_p, C.c_char_p]
    lib.sphgpu_checkpoint_load.argtypes = [C.c_void_p, C.c_char_p]
    lib.sphgpu_get_rain.argtypes = [C.c_void_p, C.POINTER(Rain)]
    if path == LIB_PATH:
        _lib = lib
    _libs[path] = lib
    return lib


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def pipe_peaks(device: int = 0) -> tuple:
    """sphgpu_pipe_peaks: the device's measured FP64 and FP32 multiply-add
    rates, TFLOP/s."""
    lib = load_library()
    f64, f32 = C.c_double(), C.c_double()
    rc = lib.sphgpu_pipe_peaks(int(device), C.byref(f64), C.byref(f32))
    if rc:
        raise SPHError(rc, "sphgpu_pipe_peaks")
    return f64.value, f32.value


class Engine:
    """One particle system on one GPU (sphgpu_ctx); with `instances`, a
    batched context of several systems that share `params` but for their
    particle ranges and cell grids (sphgpu_create_batched)."""

    def __init__(self, params: dict | Params, device: int = 0, instances=None, library: str | None = None):
        self.lib = load_library(library) if library else load_library()
        if self.lib.sphgpu_device_count() <= 0:
            raise SPHError(102, "sphgpu_device_count")
        self.params = params if isinstance(params, Params) else params_from_dict(params)
        if instances is None:
            h = self.lib.sphgpu_create(C.byref(self.params), int(device))
            what = "sphgpu_create"
        else:
            arr = (Instance * len(instances))(*instances)
            h = self.lib.sphgpu_create_batched(C.byref(self.params), arr, len(instances), int(device))
            what = "sphgpu_create_batched"
            if h:
                self.params.ntotal = sum(int(q.count) for q in instances)
        if not h:
            raise SPHError(self.lib.sphgpu_last_create_error(), what)
        self.h = C.c_void_p(h)
        self.n = int(self.params.ntotal)
        self.instances = instances

    def close(self):
        if getattr(self, "h", None):
            self.lib.sphgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code: int, what: str):
        if code != 0:
            raise SPHError(code, what)

    def set_field(self, name: str, values) -> None:
        nc = FIELDS[name]
        dt = np.int32 if name in INT_FIELDS else np.float64
        a = np.ascontiguousarray(np.asarray(values, dtype=dt).reshape(self.n * nc))
        self._check(self.lib.sphgpu_set_field(self.h, name.encode(), _ptr(a), a.size), f"set_field({name})")

    def get_field(self, name: str) -> np.ndarray:
        nc = FIELDS[name]
        dt = np.int32 if name in INT_FIELDS else np.float64
        a = np.empty(self.n * nc, dtype=dt)
        self._check(self.lib.sphgpu_get_field(self.h, name.encode(), _ptr(a), a.size), f"get_field({name})")
        return a if nc == 1 else a.reshape(self.n, nc)

    def set_materials(self, fluid: np.ndarray | None, soil: np.ndarray | None) -> None:
        fp = _ptr(np.ascontiguousarray(fluid)) if fluid is not None else None
        sp = _ptr(np.ascontiguousarray(soil)) if soil is not None else None
        self._check(self.lib.sphgpu_set_materials(self.h, fp, sp, self.n), "set_materials")

    def upload_particles(self, records: np.ndarray, stride: int = PARTICLE_BYTES) -> None:
        """sphgpu_upload_particles: whole Particle records (n x stride bytes)."""
        self._check(self.lib.sphgpu_upload_particles(self.h, _ptr(records), self.n, stride), "upload_particles")

    def download_particles(self, records: np.ndarray, stride: int = PARTICLE_BYTES) -> None:
        """sphgpu_download_particles: the device-owned members of each record."""
        self._check(self.lib.sphgpu_download_particles(self.h, _ptr(records), self.n, stride), "download_particles")

    def load_state(self, fields: dict, fluid=None, soil=None, rain=None, vibration=None) -> None:
        for name, v in fields.items():
            if name in FIELDS:
                self.set_field(name, v)
        if fluid is not None or soil is not None:
            self.set_materials(fluid, soil)
        if rain is not None:
            self.set_rain(rain)
        if vibration is not None:
            self.set_vibration(vibration)

    def set_vibration(self, vib: dict) -> None:
        """sphgpu_set_vibration: Para_Vibra of a run with flv 1 or 2 (ttime,
        nsteps, sttime, edtime and nsteps x 3 loads)."""
        v = Vibration()
        v.ttime, v.nsteps, v.sttime, v.edtime = float(vib["ttime"]), int(vib["nsteps"]), float(vib["sttime"]), \
            float(vib["edtime"])
        loads = np.ascontiguousarray(np.asarray(vib["loads"], dtype=np.float64).reshape(-1))
        self._check(self.lib.sphgpu_set_vibration(self.h, C.byref(v), _ptr(loads)), "sphgpu_set_vibration")

    def kl_generate(self, domain: KLDomain, fields, xi, K: int = 200) -> np.ndarray:
        """SpatialVariables_Generate_2D / _3D with the standard normals xi
        (len(fields) x K); returns the fields (len(fields) x ntotal, NaN where a
        field writes none), which also become the particles' material values."""
        fields = list(fields)
        arr = (KLField * len(fields))(*fields)
        x = np.ascontiguousarray(np.asarray(xi, dtype=np.float64).reshape(len(fields) * K))
        out = np.empty(len(fields) * self.n)
        self._check(self.lib.sphgpu_kl_generate(self.h, C.byref(domain), arr, len(fields), _ptr(x), int(K), _ptr(out)),
                    "sphgpu_kl_generate")
        return out.reshape(len(fields), self.n)

    def kl_synthesize(self, domain: KLDomain, field: KLField, xi, d_out: int, K: int = 200) -> float:
        """R realisations of one field (xi: R x K normals) into the device
        buffer at address d_out (R x ntotal float32) on the tensor cores;
        returns the kernels' device time in ms."""
        x = np.ascontiguousarray(np.asarray(xi, dtype=np.float64))
        R = x.size // K
        ms = C.c_double(0.0)
        self._check(self.lib.sphgpu_kl_synthesize(self.h, C.byref(domain), C.byref(field), _ptr(x), int(R), int(K),
                                                  C.c_void_p(int(d_out)), C.byref(ms)), "sphgpu_kl_synthesize")
        return ms.value

    def kl_generate_corr(self, domain: KLDomain, friction: KLField, cohesion: KLField, coe: float, u2,
                         K: int = 200) -> np.ndarray:
        """SpatialVariables_Generate_*_corr for one phase; u2: K x 2 normals."""
        arr = (KLField * 2)(friction, cohesion)
        u = np.ascontiguousarray(np.asarray(u2, dtype=np.float64).reshape(2 * K))
        out = np.empty(2 * self.n)
        self._check(self.lib.sphgpu_kl_generate_corr(self.h, C.byref(domain), arr, float(coe), _ptr(u), int(K),
                                                     _ptr(out)), "sphgpu_kl_generate_corr")
        return out.reshape(2, self.n)

    def rf_cells(self, domain: KLDomain, flags: RFFlags) -> int:
        """The number of correlation-matrix cells (the normals each field takes)."""
        n = C.c_int(0)
        self._check(self.lib.sphgpu_rf_cells(self.h, C.byref(domain), C.byref(flags), C.byref(n)), "sphgpu_rf_cells")
        return n.value

    def rf_generate(self, domain: KLDomain, fields, flags: RFFlags, zeta) -> np.ndarray:
        """nonstationary_random_2D / _3D (flspv 3) with the cell normals zeta
        (len(fields) x cells); returns len(fields) x ntotal values (NaN where a
        field writes none), which also become the particles' material values."""
        fields = list(fields)
        arr = (KLField * len(fields))(*fields)
        z = np.ascontiguousarray(np.asarray(zeta, dtype=np.float64).reshape(len(fields), -1))
        out = np.empty(len(fields) * self.n)
        self._check(self.lib.sphgpu_rf_generate(self.h, C.byref(domain), arr, len(fields), C.byref(flags), _ptr(z),
                                                z.shape[1], _ptr(out)), "sphgpu_rf_generate")
        return out.reshape(len(fields), self.n)

    def rf_generate_corr(self, domain: KLDomain, friction: KLField, cohesion: KLField, flags: RFFlags,
                         u2) -> np.ndarray:
        """nonstationary_correlated_random_2D / _3D (flspv 4) for one phase;
        u2: cells x 2 normals; returns 2 x ntotal values."""
        arr = (KLField * 2)(friction, cohesion)
        u = np.ascontiguousarray(np.asarray(u2, dtype=np.float64).reshape(-1, 2))
        out = np.empty(2 * self.n)
        self._check(self.lib.sphgpu_rf_generate_corr(self.h, C.byref(domain), arr, C.byref(flags), _ptr(u), len(u),
                                                     _ptr(out)), "sphgpu_rf_generate_corr")
        return out.reshape(2, self.n)

    def rv_generate_corr(self, friction: KLField, cohesion: KLField, coe: float, u2) -> np.ndarray:
        """random_variable_generate (flspv 5): one correlated pair for the
        phase from two normals; returns (friction, cohesion)."""
        arr = (KLField * 2)(friction, cohesion)
        u = np.ascontiguousarray(np.asarray(u2, dtype=np.float64).reshape(2))
        out = np.empty(2)
        self._check(self.lib.sphgpu_rv_generate_corr(self.h, arr, float(coe), _ptr(u), _ptr(out)),
                    "sphgpu_rv_generate_corr")
        return out

    def set_precision(self, mode: int) -> None:
        """PREC_FP64 (the reference's arithmetic) or PREC_FP32_BULK."""
        self._check(self.lib.sphgpu_set_precision(self.h, int(mode)), "sphgpu_set_precision")

    def kl_generate_batched(self, doms, field: "KLField", xi: np.ndarray) -> np.ndarray:
        """One K-L field per instance, doms[q] its domain and xi[q] its K
        standard normals; returns the n values written (NaN where none)."""
        xi = np.ascontiguousarray(xi, dtype=np.float64)
        arr = (KLDomain * len(doms))(*doms)
        out = np.empty(self.n)
        self._check(self.lib.sphgpu_kl_generate_batched(self.h, arr, C.byref(field), _ptr(xi), xi.shape[1],
                                                        _ptr(out)), "sphgpu_kl_generate_batched")
        return out

    def update_params(self, params: dict | Params) -> None:
        p = params if isinstance(params, Params) else params_from_dict(params)
        self._check(self.lib.sphgpu_update_params(self.h, C.byref(p)), "sphgpu_update_params")
        self.params = p

    def parttocell(self) -> int:
        return int(self.lib.sphgpu_parttocell(self.h))

    def partisearching(self) -> int:
        return int(self.lib.sphgpu_partisearching(self.h))

    def update(self) -> int:
        return int(self.lib.sphgpu_update(self.h))

    TUNE_PASSES = ("k_nnps", "k_nnps_resolve", "k_pairw", "k_density", "k_shepard_eos", "k_strain", "k_stress",
                   "k_accel_a", "k_accel_b", "k_xsph_update")

    def set_launch(self, threads_per_block) -> None:
        tb = np.ascontiguousarray(threads_per_block, dtype=np.int32)
        self._check(self.lib.sphgpu_set_launch(self.h, _ptr(tb), tb.size), "sphgpu_set_launch")

    def launch(self) -> np.ndarray:
        tb = np.zeros(len(self.TUNE_PASSES), np.int32)
        self._check(self.lib.sphgpu_get_launch(self.h, _ptr(tb), tb.size), "sphgpu_get_launch")
        return tb

    def autotune(self, steps: int = 2, cache_path: str | None = None) -> np.ndarray:
        """Threads per block of each tuned pass picked by timing (runs 4 x steps
        steps of the run); returns the ms per step measured (candidates 32, 64,
        96, 128 by pass), zeros when the choice came from cache_path."""
        table = np.zeros((4, len(self.TUNE_PASSES)))
        path = cache_path.encode() if cache_path else None
        self._check(self.lib.sphgpu_autotune(self.h, int(steps), path, _ptr(table)), "sphgpu_autotune")
        return table

    def output_total(self, directory: str) -> None:
        """Write directory/data-<l>.odb (the reference's output_total format)
        for the last completed step, in the background."""
        self._check(self.lib.sphgpu_output_total(self.h, directory.encode()), "sphgpu_output_total")

    def output_begin(self, directory: str) -> None:
        """Create the run's appended result files (Flowing distance.dat,
        Total_Force.dat, AVS_MGF.mgf with its header)."""
        self._check(self.lib.sphgpu_output_begin(self.h, directory.encode()), "sphgpu_output_begin")

    def output_step(self, directory: str, what: int) -> None:
        """The result files `what` selects (OUT_* bits) for the last step."""
        self._check(self.lib.sphgpu_output_step(self.h, directory.encode(), int(what)), "sphgpu_output_step")

    def output_wait(self) -> None:
        self._check(self.lib.sphgpu_output_wait(self.h), "sphgpu_output_wait")

    def checkpoint_save(self, path: str) -> None:
        self._check(self.lib.sphgpu_checkpoint_save(self.h, path.encode()), "sphgpu_checkpoint_save")

    def checkpoint_load(self, path: str) -> None:
        self._check(self.lib.sphgpu_checkpoint_load(self.h, path.encode()), "sphgpu_checkpoint_load")

    def set_rain(self, rain: dict) -> None:
        """sphgpu_set_rain: the rainfall record of a run with flr = 1."""
        self._check(self.lib.sphgpu_set_rain(self.h, C.byref(rain_record(rain))), "sphgpu_set_rain")

    def rain(self) -> dict:
        r = Rain()
        self._check(self.lib.sphgpu_get_rain(self.h, C.byref(r)), "sphgpu_get_rain")
        return {k: getattr(r, k) for k, _ in Rain._fields_}

    def set_cfl(self, cfl: float, cfl_force: float = 0.25) -> None:
        """Adaptive dt from the CFL and force limits (cfl <= 0: off, the
        reference's constant dt)."""
        self._check(self.lib.sphgpu_set_cfl(self.h, float(cfl), float(cfl_force)), "sphgpu_set_cfl")

    def set_reorder(self, every_steps: int) -> None:
        """Hold the particle state in cell order, re-sorted every every_steps
        steps (0: the caller's order, the default); results are unchanged."""
        self._check(self.lib.sphgpu_set_reorder(self.h, int(every_steps)), "sphgpu_set_reorder")

    @property
    def reorder(self) -> int:
        return int(self.lib.sphgpu_get_reorder(self.h))

    def autotune_reorder(self, steps: int = 2, every: int = 20) -> dict:
        """sphgpu_autotune_reorder: time the caller's order against the
        re-sorted one and keep the faster; returns the choice and the times."""
        chosen = C.c_int()
        ms = np.zeros(3)
        self._check(self.lib.sphgpu_autotune_reorder(self.h, int(steps), int(every), C.byref(chosen), _ptr(ms)),
                    "sphgpu_autotune_reorder")
        return {"every_steps": int(chosen.value), "caller_order_ms": float(ms[0]), "resorted_ms": float(ms[1]),
                "resort_ms_per_step": float(ms[2])}

    def order(self) -> np.ndarray:
        """i2o: the caller's index of the particle the device holds at each
        position."""
        out = np.empty(self.n, dtype=np.int32)
        self._check(self.lib.sphgpu_get_order(self.h, _ptr(out)), "sphgpu_get_order")
        return out

    def dt(self) -> float:
        """The dt the next step uses."""
        v = C.c_double()
        self._check(self.lib.sphgpu_get_dt(self.h, C.byref(v)), "sphgpu_get_dt")
        return v.value

    @property
    def precision(self) -> int:
        return int(self.lib.sphgpu_get_precision(self.h))

    def step(self, nsteps: int = 1) -> None:
        self._check(self.lib.sphgpu_step(self.h, int(nsteps)), "sphgpu_step")

    def nnps(self):
        ninflu = np.zeros(self.n, np.int32)
        influ = np.zeros(self.n * 100, np.int32)
        self._check(self.lib.sphgpu_nnps(self.h, _ptr(ninflu), _ptr(influ)), "sphgpu_nnps")
        return ninflu, influ.reshape(self.n, 100)

    def synchronize(self) -> None:
        self._check(self.lib.sphgpu_synchronize(self.h), "sphgpu_synchronize")

    @property
    def step_index(self) -> int:
        return int(self.lib.sphgpu_get_step(self.h))

    def last_step_ms(self) -> float:
        return float(self.lib.sphgpu_last_step_ms(self.h))

    def last_step_launches(self) -> int:
        return int(self.lib.sphgpu_last_step_launches(self.h))

    def step_profiled(self, nsteps: int) -> dict:
        """Run nsteps with a CUDA event between stages; returns {stage: ms
        summed over the steps}."""
        k = self.lib.sphgpu_stage_count()
        ms = np.zeros(k)
        self._check(self.lib.sphgpu_step_profiled(self.h, int(nsteps), _ptr(ms)), "sphgpu_step_profiled")
        out = {self.lib.sphgpu_stage_name(i).decode(): float(ms[i]) for i in range(k)}
        out["reorder"] = float(self.lib.sphgpu_last_reorder_ms(self.h))
        return out


def batch(states) -> tuple:
    """Concatenate initial states (scenes.initialise results of scenes that
    share every parameter but their geometry) into the arguments of a batched
    Engine: (shared params, instances, fields, fluid records, soil records)."""
    insts, first = [], 0
    for st in states:
        p = st.params
        n = int(p["ntotal"])
        insts.append(Instance(first, n, p["xmin"], p["xmax"], p["ymin"], p["ymax"], p["zmin"], p["zmax"],
                              p["cxm"], p["cym"], p["czm"], p["ctotal"]))
        first += n
    fields = {k: np.concatenate([st.fields[k] for st in states]) for k in states[0].fields}
    fluid = np.concatenate([st.fluid for st in states])
    soil = np.concatenate([st.soil for st in states])
    shared = dict(states[0].params)
    shared["ntotal"] = first
    return shared, insts, fields, fluid, soil
