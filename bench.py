#!/usr/bin/env python3
"""Benchmark: particle-updates/s of the SPH time step on B200.

Workload (the reference's second configuration): a 3-D saturated soil column
collapse -- a 1.0 x 0.5 x 0.5 m Drucker-Prager soil block at dx = 5 mm
(2,000,000 soil particles, E = 10 MPa, nu = 0.3, phi = 30 deg, c = 0,
rho_s = 2650, porosity 0.4) overlapped by 2,000,000 pore-water particles,
Darcy drag with k = 1e-4 m/s, in a 3-layer walled box (452,072 wall
particles), dt = 0.25 dr / 600.  Synthetic lattice input, FP64 throughout.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours       K steps of the engine (CUDA graph per step) timed with CUDA events
           on the engine's stream, state resident in HBM; value =
           active particles (types 1-4) x K / time.  e2e: the same K steps
           through the C ABI from host buffers (state upload before, full
           state download after, inside the timed region).
reference  the reference solver itself (oracle/_ref, compiled from its own
           sources) on the host cores, same workload and metric.
With torchrun (N > 1) every rank runs an independent replica of the workload
(the path has no exchange step); value is the sum over ranks divided by the
slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "multiphase-sph-solver_b200")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

import scenes  # noqa: E402

METRIC = "particle-updates/s"
WORKLOAD = "3d_saturated_soil_column_collapse"

# Algorithmic bytes per particle per step: each barrier-level pass of the
# step reads its own particle's fields once and writes its outputs once,
# neighbour fields are served from cache after the cell sort, and no
# neighbour list is stored.  The per-pass figures are those of the 2-D FP64
# dam break (806 B in all); the 3-D soil column with co-located water (soil
# state sigma, eps, adps, e, n, satu, cop and its material fields) comes to
# 1,870 B by the same rule, and its per-pass figures are the 2-D ones scaled
# by 1870 / 806.  Each pass is listed with the kernels of this engine that do
# its work.  The engine's neighbour search and pair records have no
# counterpart in this count (their traffic is the engine's own choice).  The
# headline run keeps the state in the caller's order (a spatial lattice
# already), so its reorder pass does no work; the engine's re-sort
# (sphgpu_set_reorder, stage "reorder") is timed on the same particles given
# in a random order.
RESORT_EVERY = 20
PASS_BYTES_2D = {
    "key": 24.0,
    "radix sort": 32.0,
    "reorder": 196.0,
    "cell ranges": 14.0,
    "porosity + continuity": 68.0,
    "Shepard + EOS": 36.0,
    "strain + stress + free surface + eigen": 124.0,
    "stress divergence + viscosity + walls + velocity update": 132.0,
    "XSPH + walls + check_domain + update": 180.0,
}
STEP_BYTES_3D = 1870.0
PASS_KERNELS = {
    "key": ("k_cellkey",),
    "radix sort": ("radix_sort",),
    "reorder": ("reorder",),
    "cell ranges": ("k_cellreset", "k_cellrange"),
    "porosity + continuity": ("k_density",),
    "Shepard + EOS": ("k_shepard_eos",),
    "strain + stress + free surface + eigen": ("k_strain", "k_regu_eps", "k_saturation", "k_stress",
                                               "k_regu_sig", "k_stress_2", "k_art_rij"),
    "stress divergence + viscosity + walls + velocity update": ("k_accel_a", "k_accel_b", "k_ss", "k_tran_wall",
                                                                "k_coupled", "k_free_solid"),
    "XSPH + walls + check_domain + update": ("k_xsph_update", "k_tm_boundary"),
}


def pass_bytes(ndim: int = 3) -> dict:
    scale = 1.0 if ndim == 2 else STEP_BYTES_3D / sum(PASS_BYTES_2D.values())
    return {k: v * scale for k, v in PASS_BYTES_2D.items()}


def pass_roofline(stage_ms: dict, n: int, peak_gbs: float, ndim: int = 3) -> dict:
    """Per pass: its algorithmic bytes for n particles, the summed device time
    of its kernels (ms per step) and the achieved GB/s and fraction of peak."""
    out = {}
    for name, b in pass_bytes(ndim).items():
        ms = sum(stage_ms.get(k, 0.0) for k in PASS_KERNELS[name])
        gbs = b * n / (ms / 1e3) / 1e9 if ms > 0 else None
        out[name] = {"bytes_per_particle": b, "kernels": list(PASS_KERNELS[name]), "ms": ms,
                     "achieved_gbs": gbs, "frac": gbs / peak_gbs if gbs else None}
    return out


# Algorithmic FP64 flops per particle per step of the 3-D soil column with
# co-located water: about 14,000 (the pair arithmetic of the neighbour passes
# for 65 neighbours, the constitutive update and the eigenvalues), the figure
# the HBM bound is weighed against (about 7.6 flop per algorithmic byte).
STEP_FLOPS_3D = 14000.0


def fp64_roofline(device: int, n: int, step_ms: float) -> dict:
    """The whole step against the device's measured FP64 multiply-add rate
    (sphgpu_pipe_peaks), beside the HBM roofline: the drop-in form's pair and
    constitutive arithmetic runs on the FP64 pipe."""
    import sphgpu
    try:
        f64, f32 = sphgpu.pipe_peaks(device)
    except sphgpu.SPHError as e:
        return {"unavailable": str(e)}
    achieved = STEP_FLOPS_3D * n / (step_ms / 1e3) / 1e12
    return {"bound": "fp64", "algorithmic_flops_per_particle": STEP_FLOPS_3D, "achieved": achieved,
            "peak": f64, "unit": "TFLOP/s", "frac": achieved / f64, "peak_kind": "measured (sphgpu_pipe_peaks)",
            "fp32_peak": f32}


def measured_peaks() -> tuple[dict, str]:
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def ncu_traffic() -> dict:
    """Per-particle DRAM bytes per kernel from the committed ncu summary."""
    p = os.path.join(REPO, "profiles", "ncu_traffic_per_particle.json")
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh)
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms during the timed region."""

    def __init__(self, gpu_index: int):
        self.fh = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.fh.flush()
        self.fh.seek(0)
        sm, smax, reasons = [], [], set()
        for line in self.fh.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                               f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.fh.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def _reduce(x: float, op) -> float:
    import torch
    import torch.distributed as dist
    # NCCL reduces device tensors; the gloo backend (CPU runs) host tensors
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def dist_max(x: float, world: int) -> float:
    """The slowest replica's time: the max over ranks."""
    if world == 1:
        return x
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX)


def dist_sum(x: float, world: int) -> float:
    """The particles of all replicas: the sum over ranks."""
    if world == 1:
        return x
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM)


def replica_value(n_active: float, steps: int, ms: float, world: int) -> float:
    """Whole-job particle-updates/s of independent replicas: every rank's
    active particles times the steps, over the slowest rank's time."""
    return dist_sum(float(n_active), world) * steps / (dist_max(ms, world) / 1e3)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------------
# reference solver on the host cores

def run_reference(scene, steps: int, warmup: int, threads: int) -> dict:
    sys.path.insert(0, os.path.join(REPO, "tests"))
    from checkers import Reference, have_reference
    if not have_reference():
        return {"unavailable": "oracle/_ref/libsphref.so was not built (needs the reference source tree)"}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "input.dat")
        scenes.write_input_dat(scene, path, ntd=threads)
        t0 = time.perf_counter()
        devnull = os.open(os.devnull, os.O_WRONLY)
        saved = os.dup(1)
        os.dup2(devnull, 1)          # the reference prints progress to stdout
        try:
            ref = Reference(path, threads)
            t_init = time.perf_counter() - t0
            err = ref.step(warmup) if warmup else 0
            t1 = time.perf_counter()
            err = err or ref.step(steps)
            t_steps = time.perf_counter() - t1
        finally:
            os.dup2(saved, 1)
            os.close(devnull)
            os.close(saved)
    return {"init_s": t_init, "step_s": t_steps / max(steps, 1), "err": err,
            "value": scene.n_active() * steps / t_steps if t_steps > 0 else None}


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_arm(args, world, rank):
    if rank != 0:
        return 0
    full = scenes.soil_column_3d(dx=args.dx, steps=5000)
    need_gb = full.n * 8.0e3 / 1e9
    try:
        import psutil
        avail_gb = psutil.virtual_memory().available / 1e9
    except Exception:
        avail_gb = float("inf")
    steps = max(1, min(args.steps, 3))
    warm = min(args.warmup, 1)
    threads = host_threads()
    if avail_gb < need_gb * 1.3:
        scene = scenes.soil_column_3d(dx=2 * args.dx, steps=5000)
        sample = (f"{steps} steps of the same scene at dx={2 * args.dx:g} ({scene.n} particles); "
                  f"full size needs ~{need_gb:.0f} GB host RAM, {avail_gb:.0f} GB free")
    else:
        scene = full
        sample = f"{steps} steps (after {warm} warm-up) of the full workload, {scene.n} particles"
    r = run_reference(scene, steps, warm, threads)
    if "unavailable" in r:
        print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}))
        return 0
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": "particle-updates/s",
        "n_gpus": 0, "steps": steps, "warmup": warm, "ms_per_step": r["step_s"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "dx": scene.dr, "particles": scene.n,
                   "active_particles": scene.n_active(), "host_threads": threads,
                   "reference_init_s": round(r["init_s"], 2)},
        "cpu_baseline": {"value": r["value"], "unit": "particle-updates/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": r["value"], "unit": "particle-updates/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------------
# engine arm

STATE_UP = ("xp", "vxp", "axp", "ax", "vx", "ux", "rho", "rhop", "mass", "hl", "pre", "prep", "e",
            "eps", "sig", "adps", "satu", "cop", "porosity", "poro_cop", "cd", "interf", "interfss",
            "type", "matype", "permtype", "etype")


def _rel_l2(a, b, m):
    a, b = a[m], b[m]
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bulk_form(st, args, device, ref_fields, moving):
    """The FP32-bulk form on the same workload: K timed steps after the same
    warm-up, and its state after warm-up + K steps against the FP64 form's."""
    import sphgpu
    eng = sphgpu.Engine(st.params, device=device)
    eng.load_state(st.fields, st.fluid, st.soil)
    eng.set_precision(sphgpu.PREC_FP32_BULK)
    if not args.no_autotune:
        # the FP64 engine's autotuning steps, so that both states are compared
        # after the same number of steps
        eng.autotune(steps=2)
        eng.autotune_reorder(steps=2, every=RESORT_EVERY)
    eng.step(args.warmup)
    eng.synchronize()
    eng.step(args.steps)
    ms = eng.last_step_ms()
    err = {k: _rel_l2(eng.get_field(k), ref_fields[k], moving) for k in ref_fields}
    prof = eng.step_profiled(args.steps)
    eng.close()
    return ms, err, prof


def kl_synthesis(eng, scene, device, R=32, K=400):
    """R realisations of a K-term friction-angle field (normal, mean 30 deg,
    COV 0.1, correlation lengths 0.5 / 0.25 / 0.25 m, depth trend) on the
    workload's particles, on the tensor cores, into device memory."""
    import sphgpu
    import torch
    d = scenes.kl_domain(scene)
    dom = sphgpu.kl_domain(d["nb_min"], d["nb_max"], d["soil_max"], d["water_max"])
    field = sphgpu.kl_field(0, 1, 30.0, 3.0, [0.5, 0.25, 0.25], 2.0)
    xi = np.random.default_rng(20261203).standard_normal((R, K))
    out = torch.empty(R * eng.n, dtype=torch.float32, device=f"cuda:{device}")
    eng.kl_synthesize(dom, field, xi, out.data_ptr(), K)           # warm-up (plan + launch)
    t0 = time.perf_counter()
    ms = eng.kl_synthesize(dom, field, xi, out.data_ptr(), K)
    wall = time.perf_counter() - t0
    flops = 2.0 * eng.n * K * R * 3            # three TF32 products per term
    del out
    return {"realisations": R, "terms": K, "particles": eng.n, "kernel_ms": ms, "call_s": wall,
            "tensor_tflops": flops / (ms / 1e3) / 1e12,
            "fields_per_s": R / wall,
            "what": "tcgen05 kind::tf32 split-operand product, eigenfunction tiles generated in shared memory"}


def slope_heights(count: int = 256, dx: float = 0.05, seed: int = 20261203) -> np.ndarray:
    """Heights H = 5 + 7 u of the batched slopes, u uniform from a Philox
    stream of the given seed, rounded to the particle spacing."""
    u = np.random.Generator(np.random.Philox(seed)).random(count)
    return np.round((5.0 + 7.0 * u) / dx) * dx


def batched_slopes(args, device: int, count: int = 256, dx: float = 0.05, steps_run: int = 20000, K: int = 200):
    """The batched Monte Carlo slope workload: `count` 2-D cohesive-frictional
    slopes (1:1.5 face, 6.25 m crest, H from slope_heights, Drucker-Prager,
    phi = 25 deg, E = 20 MPa, dry) in one batched context, each with its own
    lognormal K-L cohesion field (mean 10 kPa, COV 0.3, correlation lengths
    10 m / 1 m, K terms, its own standard normals).  Times K-L generation for
    all instances, then args.steps steps after args.warmup, in the FP64 and
    FP32-bulk forms; realisations per hour = count x 3600 / (K-L time +
    steps_run x step time)."""
    import sphgpu
    H = slope_heights(count, dx)
    insts, parts, first = [], [], 0
    shared = None
    keep = ("xp", "vxp", "axp", "rho", "rhop", "mass", "hl", "pre", "prep", "e", "sig", "satu", "porosity",
            "cd", "type", "matype", "permtype", "etype")
    cols = {k: [] for k in keep}
    fl, so, doms = [], [], []
    n_active = 0
    for h in H:
        sc = scenes.slope_2d(H=float(h), dx=dx, c=10.0e3, fai=25.0, E=2.0e7)
        st = scenes.initialise(sc)
        p = st.params
        if shared is None:
            shared = dict(p)
        insts.append(sphgpu.Instance(first, sc.n, p["xmin"], p["xmax"], p["ymin"], p["ymax"], p["zmin"], p["zmax"],
                                     p["cxm"], p["cym"], p["czm"], p["ctotal"]))
        first += sc.n
        n_active += sc.n_active()
        for k in keep:
            cols[k].append(st.fields[k])
        fl.append(st.fluid)
        so.append(st.soil)
        d = scenes.kl_domain(sc)
        doms.append(sphgpu.kl_domain(d["nb_min"], d["nb_max"], d["soil_max"], d["water_max"]))
        del st
    fields = {k: np.concatenate(v) for k, v in cols.items()}
    del cols
    fluid, soil = np.concatenate(fl), np.concatenate(so)
    del fl, so
    shared["ntotal"] = first
    xi = np.random.Generator(np.random.Philox(20261204)).standard_normal((count, K))
    field = sphgpu.kl_field(1, 2, 10.0e3, 3.0e3, [10.0, 1.0, 0.0])
    out = {"instances": count, "particles": first, "active_particles": n_active, "dx": dx,
           "heights_m": [float(H.min()), float(H.max())],
           "particles_per_instance": [int(min(q.count for q in insts)), int(max(q.count for q in insts))]}
    for form in ("fp64", "fp32_bulk"):
        eng = sphgpu.Engine(shared, device=device, instances=insts)
        eng.load_state(fields, fluid, soil)
        t0 = time.perf_counter()
        eng.kl_generate_batched(doms, field, xi)
        kl_s = time.perf_counter() - t0
        if form == "fp32_bulk":
            eng.set_precision(sphgpu.PREC_FP32_BULK)
        if not args.no_autotune:
            eng.autotune(steps=2)
        eng.step(args.warmup)
        eng.synchronize()
        eng.step(args.steps)
        ms = eng.last_step_ms() / args.steps
        eng.close()
        runs_hr = count * 3600.0 / (kl_s + steps_run * ms / 1e3)
        out[form] = {"ms_per_step": ms, "value": n_active / (ms / 1e3), "unit": "particle-updates/s",
                     "kl_generate_s": kl_s, "rf_runs_per_hour": runs_hr}
    out["fp32_bulk"]["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["fp32_bulk"]["ms_per_step"]
    out["what"] = (f"{count} slopes in one batched context (one graph per step over all instances), "
                   f"runs/hr for {steps_run} steps each with K-L generation")
    return out


def batched_slopes_cpu(threads: int, dx: float = 0.05, steps_run: int = 20000):
    """The reference on one slope of the median height, on the host cores:
    realisations per hour when each runs alone for steps_run steps."""
    H = float(np.median(slope_heights()))
    sc = scenes.slope_2d(H=H, dx=dx, c=10.0e3, fai=25.0, E=2.0e7)
    r = run_reference(sc, 3, 1, threads)
    if "unavailable" in r:
        return None
    return {"value": sc.n_active() / r["step_s"], "unit": "particle-updates/s", "ms_per_step": r["step_s"] * 1e3,
            "rf_runs_per_hour": 3600.0 / (steps_run * r["step_s"]), "cores": threads, "kind": "reference",
            "sample": f"3 steps (after 1 warm-up) of one slope, H = {H:g} m ({sc.n} particles); "
                      f"its K-L generation not included"}


MCC = dict(ramda=0.2, kapa=0.04, zmf=1.2, eps0=0.9, poi=0.3, sme0=50.0e3, ann=1.0, ocr=1.5, e=0.0, fs=1.0)


def dam_break_scene(dx: float = 0.005):
    """The 2-D dam break: a 0.4 m x 0.8 m water column in a 1.6 m x 1.0 m tank,
    12,800 water particles at dx = 5 mm, 3 wall layers."""
    return scenes.dam_break_2d(dx=dx, steps=2000)


def footing_scene(dx: float = 0.04):
    """The 3-D soil-structure case: a rigid strip footing 2 m wide, 0.28 m tall
    and 5 m long (43,750 structure particles at dx = 40 mm) pushed down at
    0.01 m/s into a 10 x 5 x 5 m subloading Cam-clay bed (lambda 0.2, kappa
    0.04, M 1.2, OCR 1.5, e0 0.9; 3.9 M soil particles), penalty contact.  The
    footing starts two spacings above the soil."""
    sc = scenes.footing(ndim=3, dx=dx, bed=(10.0, 5.0, 5.0), width=2.0, height=0.28, gap=2.0, v=0.01, ss_type=3,
                        myu=0.3, zeta=0.1, steps=5000, matype=1)
    return scenes.set_soil_model(sc, 1, **MCC)


def geostatic_soil(st, K0: float = 0.3 / 0.7) -> None:
    """A K0 geostatic stress in the soil (vertical stress rho g depth below
    the soil's top, horizontal K0 times it), so that a Cam-clay bed starts
    from a stress state rather than from zero stiffness."""
    t, xp = st.fields["type"], st.fields["xp"]
    soil = t == 2
    if not soil.any():
        return
    dens = np.asarray(st.soil["dens"])
    top = xp[soil, 1].max() + 0.5 * st.params["dr"]
    sig = np.array(st.fields["sig"], dtype=np.float64).reshape(-1, 6).copy()
    sv = -dens * 9.81 * (top - xp[:, 1])
    sig[soil, 1] = sv[soil]
    sig[soil, 0] = K0 * sv[soil]
    sig[soil, 2] = K0 * sv[soil]
    st.fields["sig"] = sig


def config_leg(args, device, make, cpu_make, threads, prepare=None):
    """One more named workload: K steps after the warm-up in the FP64 and
    FP32-bulk forms (the bulk form's state compared with the FP64 form's after
    the same steps), and the reference on the host cores on a sample of it."""
    import sphgpu
    sc = make()
    st = scenes.initialise(sc)
    if prepare is not None:
        prepare(st)
    n_active = sc.n_active()
    out = {"particles": sc.n, "active_particles": n_active}
    moving = (st.fields["type"] >= 1) & (st.fields["type"] <= 4)
    ref = None
    for form in ("fp64", "fp32_bulk"):
        eng = sphgpu.Engine(st.params, device=device)
        eng.load_state(st.fields, st.fluid, st.soil)
        if form == "fp32_bulk":
            eng.set_precision(sphgpu.PREC_FP32_BULK)
        eng.step(args.warmup)
        eng.synchronize()
        eng.step(args.steps)
        ms = eng.last_step_ms() / args.steps
        out[form] = {"ms_per_step": ms, "value": n_active / (ms / 1e3), "unit": "particle-updates/s"}
        fields = {k: eng.get_field(k) for k in ("sig", "ux", "vx", "rho", "xp")}
        if ref is None:
            ref = fields
        else:
            out[form]["rel_l2_vs_fp64"] = {k: _rel_l2(fields[k], ref[k], moving) for k in ref}
        eng.close()
    out["fp32_bulk"]["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["fp32_bulk"]["ms_per_step"]
    if cpu_make is not None and threads:
        small = cpu_make()
        r = run_reference(small, 2, 1, threads)
        if "unavailable" not in r:
            out["cpu_baseline"] = {"value": r["value"], "unit": "particle-updates/s", "cores": threads,
                                   "kind": "reference",
                                   "sample": f"2 steps (after 1 warm-up) of {small.name} ({small.n} particles)"}
    return out


def rain_slope_leg(args, device, threads: int, steps_run: int = 20000, K: int = 400):
    """The 3-D rainfall slope (three phases: Drucker-Prager soil with
    co-located pore air, rain rows over the crest falling as water, Darcy
    drag; 8.65 M particles at dx = 50 mm) with correlated K-L friction and
    cohesion fields (K terms, correlation 0.5, depth trend): one realisation's
    field generation and K steps in the FP64 and FP32-bulk forms; realisations
    per hour for steps_run steps each.  The reference on the host cores runs
    the same scene at dx = 100 mm."""
    import sphgpu
    sc = scenes.rain_slope_3d(dx=0.05, steps=steps_run)
    st = scenes.initialise(sc)
    n_active = sc.n_active()
    d = scenes.kl_domain(sc)
    dom = sphgpu.kl_domain(d["nb_min"], d["nb_max"], d["soil_max"], d["water_max"])
    fai = sphgpu.kl_field(0, 1, 25.0, 2.5, [10.0, 10.0, 1.0], 0.5)
    coh = sphgpu.kl_field(1, 2, 10.0e3, 3.0e3, [10.0, 10.0, 1.0], 500.0)
    u2 = np.random.Generator(np.random.Philox(20261205)).standard_normal((K, 2))
    out = {"particles": sc.n, "active_particles": n_active, "rain_particles": int((sc.ptype == 7).sum()),
           "kl_terms": K}
    for form in ("fp64", "fp32_bulk"):
        eng = sphgpu.Engine(st.params, device=device)
        eng.load_state(st.fields, st.fluid, st.soil, st.rain)
        t0 = time.perf_counter()
        eng.kl_generate_corr(dom, fai, coh, 0.5, u2, K)
        kl_s = time.perf_counter() - t0
        if form == "fp32_bulk":
            eng.set_precision(sphgpu.PREC_FP32_BULK)
        eng.step(args.warmup)
        eng.synchronize()
        eng.step(args.steps)
        ms = eng.last_step_ms() / args.steps
        eng.close()
        out[form] = {"ms_per_step": ms, "value": n_active / (ms / 1e3), "unit": "particle-updates/s",
                     "kl_generate_s": kl_s, "rf_runs_per_hour": 3600.0 / (kl_s + steps_run * ms / 1e3)}
    out["fp32_bulk"]["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["fp32_bulk"]["ms_per_step"]
    if threads:
        small = scenes.rain_slope_3d(dx=0.1, steps=steps_run)
        r = run_reference(small, 2, 1, threads)
        if "unavailable" not in r:
            out["cpu_baseline"] = {"value": r["value"], "unit": "particle-updates/s", "cores": threads,
                                   "kind": "reference", "ms_per_step": r["step_s"] * 1e3,
                                   "sample": f"2 steps (after 1 warm-up) of {small.name} ({small.n} particles); "
                                             f"its K-L generation not included"}
    return out


def rf_cholesky(device, threads: int):
    """The correlation-matrix random field (flspv 3) on the 5 m slope: one
    lognormal cohesion field over about 2,400 cells and one over about
    13,000 (the reference refuses 15,000), timed per call on the GPU; the
    reference's own routine on the 2,400-cell case on the host cores."""
    import sphgpu
    sc = scenes.slope_2d(H=5.0, dx=0.1)
    st = scenes.initialise(sc)
    d = scenes.kl_domain(sc)
    dom = sphgpu.kl_domain(d["nb_min"], d["nb_max"], d["soil_max"], d["water_max"])
    ext = 1.2 * (np.array(d["nb_max"]) - np.array(d["nb_min"]))
    out = {}
    eng = sphgpu.Engine(st.params, device=device)
    eng.load_state(st.fields, st.fluid, st.soil)
    field = sphgpu.kl_field(1, 2, 10.0e3, 3.0e3, [6.0, 1.5, 0.0], 100.0)
    small = None
    for target in (2500, 14000):
        ndx = 1.03 * float(np.sqrt(ext[0] * ext[1] / target) / sc.dr)
        fl = sphgpu.rf_flags(ndx, 1)
        nc = eng.rf_cells(dom, fl)
        z = np.random.default_rng(7).standard_normal((1, nc))
        eng.rf_generate(dom, [field], fl, z)               # warm-up
        t0 = time.perf_counter()
        eng.rf_generate(dom, [field], fl, z)
        out[f"cells_{nc}"] = {"cells": nc, "gpu_s": time.perf_counter() - t0,
                              "factor_flop": nc ** 3 / 3.0}
        if small is None:
            small = (ndx, nc, z)
    eng.close()
    if threads:
        sys.path.insert(0, os.path.join(REPO, "tests"))
        from checkers import have_reference, reference_lib, rf_reference
        if have_reference():
            import ctypes
            ndx, nc, z = small
            lib = reference_lib()
            f = {"no": 1, "type": 2, "mean": 10.0e3, "sd": 3.0e3, "rl": [6.0, 1.5, 0.0], "coe_depth": 100.0,
                 "cell_ndx": ndx, "flag_auto": 1}
            lib.ref_rf_threads(ctypes.c_int(threads))
            try:
                t0 = time.perf_counter()
                rf_reference(2, sc.xp, sc.ptype, sc.dr, f, d, z[0])
                out["cpu_baseline"] = {"cells": nc, "s": time.perf_counter() - t0, "cores": threads,
                                       "kind": "reference"}
            finally:
                lib.ref_rf_threads(ctypes.c_int(1))
    return out


def engine_arm(args, world, rank, local):
    import sphgpu
    scene = scenes.soil_column_3d(dx=args.dx, steps=5000)
    st = scenes.initialise(scene)
    n_active = scene.n_active()
    device = local if world > 1 else args.device
    eng = sphgpu.Engine(st.params, device=device)
    eng.load_state(st.fields, st.fluid, st.soil)
    tune = None
    if not args.no_autotune:
        # the project's autotuner: threads per block of each neighbour pass,
        # timed over steps of the run (4 candidates x 2 steps)
        table = eng.autotune(steps=2)
        tune = {"passes": list(sphgpu.Engine.TUNE_PASSES), "threads_per_block": [int(v) for v in eng.launch()],
                "ms_per_step_by_candidate": {str(b): [round(float(x), 4) for x in table[a]]
                                             for a, b in enumerate((32, 64, 96, 128))},
                # whether to hold the state re-sorted (the caller's order here is
                # a spatial lattice already)
                "reorder": eng.autotune_reorder(steps=2, every=RESORT_EVERY)}
    eng.step(args.warmup)
    barrier(world)
    eng.synchronize()
    clocks = ClockSampler(local if world > 1 else args.device)
    time.sleep(0.3)
    eng.step(args.steps)                              # timed: CUDA events on the engine stream
    ms = eng.last_step_ms()
    launches = eng.last_step_launches()
    clk = clocks.stop()
    ms_max = dist_max(ms, world)
    total_active = dist_sum(float(n_active), world)
    value = total_active * args.steps / (ms_max / 1e3)

    moving = (st.fields["type"] >= 1) & (st.fields["type"] <= 4)
    ref_fields = {k: eng.get_field(k) for k in ("sig", "ux", "vx", "rho", "xp")}
    # stage durations with an event between stages, over the same number of steps
    prof = eng.step_profiled(args.steps)
    stage_ms = {k: v / args.steps for k, v in prof.items()}
    peaks, peak_kind = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    passes = pass_roofline(stage_ms, scene.n, hbm)
    # the roofline line is the pass that takes the most device time
    dominant = max((k for k in passes if passes[k]["ms"] > 0), key=lambda k: passes[k]["ms"])
    dom = passes[dominant]
    avg_ms = dom["ms"]
    alg = dom["bytes_per_particle"] * scene.n
    achieved = dom["achieved_gbs"]
    # the pass's kernels as ncu names them (the momentum stage launches two
    # loop kernels and a tail kernel under the stage name k_accel_b)
    ncu_names = {"k_accel_b": ("k_accel_b", "k_accel_b_drag", "k_accel_b_tail")}
    pass_kernels = [q for k in dom["kernels"] if stage_ms.get(k, 0.0) > 0.01 for q in ncu_names.get(k, (k,))]
    per_kernel = ncu_traffic()
    traffic = (sum(per_kernel[k] for k in pass_kernels)
               if pass_kernels and all(k in per_kernel for k in pass_kernels) else None)
    step_ms = ms_max / args.steps
    step_gbs = STEP_BYTES_3D * scene.n / (step_ms / 1e3) / 1e9

    # end to end through the C ABI from host buffers, as a caller holding the
    # reference's own arrays uses it: its Particle records (sphgpu_upload /
    # download_particles) and its material records (sphgpu_set_materials)
    recs = sphgpu.particle_records({k: st.fields[k] for k in STATE_UP}, scene.n)
    out_recs = np.zeros_like(recs)
    fluid, soil = np.ascontiguousarray(st.fluid), np.ascontiguousarray(st.soil)
    eng2 = sphgpu.Engine(st.params, device=local if world > 1 else args.device)
    barrier(world)
    t0 = time.perf_counter()
    eng2.upload_particles(recs)
    eng2.set_materials(fluid, soil)
    eng2.step(args.steps)
    eng2.download_particles(out_recs)
    t_e2e = time.perf_counter() - t0
    t_e2e = dist_max(t_e2e, world)
    h2d = recs.nbytes + fluid.nbytes + soil.nbytes
    # the download moves the device-owned members only (all but x), ints in
    # 8-byte slots
    d2h = scene.n * sum(8 * nc if k not in sphgpu.INT_FIELDS else 8 for k, nc in sphgpu.FIELDS.items() if k != "x")
    e2e_value = total_active * args.steps / t_e2e
    eng2.close()

    shuffled = None
    if not args.no_shuffled:
        # the same workload with the particles in a random order (a caller's
        # Particle array need not be spatial): the neighbour gathers then hit
        # scattered records
        perm = np.random.Generator(np.random.Philox(20261206)).permutation(scene.n)
        fields_p = {k: np.asarray(v)[perm] for k, v in st.fields.items()}
        eng3 = sphgpu.Engine(st.params, device=device)
        eng3.load_state(fields_p, np.asarray(st.fluid)[perm], np.asarray(st.soil)[perm])
        del fields_p
        eng3.step(args.warmup)
        eng3.synchronize()
        eng3.step(args.steps)
        sh_ms = eng3.last_step_ms() / args.steps
        sh_prof = eng3.step_profiled(args.steps)
        # the engine re-sorting its state (sphgpu_set_reorder) every 20
        # steps: the re-sorts that fall in the timed steps are timed with them;
        # beside it, what the reorder autotuner chooses for this order
        sh_tune = eng3.autotune_reorder(steps=2, every=RESORT_EVERY)
        eng3.set_reorder(RESORT_EVERY)
        eng3.step(args.warmup)
        eng3.synchronize()
        eng3.step(args.steps)
        rs_ms = eng3.last_step_ms() / args.steps
        rs_prof = eng3.step_profiled(args.steps)
        eng3.close()
        spatial_ms = ms_max / args.steps
        shuffled = {"ms_per_step": sh_ms, "value": n_active / (sh_ms / 1e3), "unit": "particle-updates/s",
                    "slowdown_vs_spatial_order": sh_ms / spatial_ms,
                    "stage_ms_per_step": {k: v / args.steps for k, v in sh_prof.items() if v > 0.01},
                    "autotune_reorder": sh_tune,
                    "resorted": {"every_steps": RESORT_EVERY, "ms_per_step": rs_ms,
                                 "value": n_active / (rs_ms / 1e3), "slowdown_vs_spatial_order": rs_ms / spatial_ms,
                                 "resort_ms_per_step": rs_prof.get("reorder", 0.0) / args.steps,
                                 "stage_ms_per_step": {k: v / args.steps for k, v in rs_prof.items() if v > 0.01}},
                    "what": "the same particles in a random order (Philox seed 20261206), held in that order, "
                            "and re-sorted by the engine"}
    bulk_ms, bulk_err, bulk_prof = bulk_form(st, args, device, ref_fields, moving)
    bulk_ms = dist_max(bulk_ms, world)
    kl = kl_synthesis(eng, scene, device) if not args.no_kl else None
    eng.close()
    batched = batched_slopes(args, device) if not args.no_batched else None
    rf = None
    if rank == 0 and not args.no_configs:
        rf = rf_cholesky(device, host_threads() if (world == 1 and not args.no_cpu_baseline) else 0)
    others = None
    if not args.no_configs:
        thr = host_threads() if (rank == 0 and world == 1 and not args.no_cpu_baseline) else 0
        others = {
            "dam_break_2d_dx5mm": config_leg(args, device, dam_break_scene, dam_break_scene, thr),
            "footing_3d_camclay_dx40mm": config_leg(args, device, footing_scene, lambda: footing_scene(0.08), thr,
                                                    prepare=geostatic_soil),
            "rain_slope_3d_dx50mm": rain_slope_leg(args, device, thr),
        }

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        small = scenes.soil_column_3d(dx=2 * args.dx, steps=5000)
        thr = host_threads()
        r = run_reference(small, 2, 1, thr)
        if "unavailable" not in r:
            cpu = {"value": r["value"], "unit": "particle-updates/s", "cores": thr, "kind": "reference",
                   "sample": f"2 steps (after 1 warm-up) of the same scene at dx={2 * args.dx:g} "
                             f"({small.n} particles, {small.n_active()} active)"}
        if batched is not None:
            batched["cpu_baseline"] = batched_slopes_cpu(thr)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "dx": args.dx, "particles_per_gpu": scene.n,
                       "active_particles_per_gpu": n_active, "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (state ~%.1f GB per GPU)" % (scene.n * 1.0e3 / 1e9),
                       "timing": "CUDA events on the engine stream around K graph launches"},
            "gpu_launches": int(launches),
            "autotune": tune,
            "clocks": clk,
            "roofline": {"bound": "hbm", "pass": dominant, "kernels": pass_kernels, "achieved": achieved,
                         "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg, "avg_launch_ms": avg_ms,
                         "traffic": (traffic * scene.n) if traffic else None,
                         "traffic_over_algorithmic": (traffic * scene.n / alg) if traffic else None,
                         "step": {"algorithmic_bytes": STEP_BYTES_3D * scene.n, "ms": step_ms,
                                  "achieved": step_gbs, "frac": step_gbs / hbm}},
            "roofline_fp64": fp64_roofline(device, scene.n, step_ms),
            "passes": passes,
            "stage_ms_per_step": stage_ms,
            "forms": {
                "fp64": {"value": value, "ms_per_step": ms_max / args.steps,
                         "error": "bit-identical to the FP64 oracle (tests/test_gpu_parity.py)"},
                "fp32_bulk": {"value": total_active * args.steps / (bulk_ms / 1e3),
                              "ms_per_step": bulk_ms / args.steps,
                              "speedup_vs_fp64": ms_max / bulk_ms,
                              "rel_l2_vs_fp64_after_warmup_plus_steps": bulk_err,
                              "stage_ms_per_step": {k: v / args.steps for k, v in bulk_prof.items() if v > 0.01}},
            },
            "kl_synthesis": kl,
            "batched_slopes": batched,
            "configs": others,
            "shuffled_order": shuffled,
            "rf_cholesky": rf,
            "e2e": {"value": e2e_value, "unit": "particle-updates/s",
                    "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                    "what": "Particle-record upload, material upload, K steps and Particle-record download "
                            "through the C ABI"},
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--dx", type=float, default=0.005)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-kl", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-configs", action="store_true")
    ap.add_argument("--no-shuffled", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        # host-only arm: rank 0 runs it, the other ranks exit without work
        world = int(os.environ.get("WORLD_SIZE", "1"))
        return reference_arm(args, world, int(os.environ.get("RANK", "0")))
    world, rank, local = dist_setup()
    try:
        rc = engine_arm(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
