"""Synthetic scenes for the SPH engine, in the reference solver's own terms.

A scene is the content of the reference's ``input.dat`` (flag, problem,
material and particle blocks read by ``clFIni_Fun::initial_pro``,
``initial_mat`` and ``input_par``, CPP_2-initialf.cpp:22-1018) held as numpy
arrays and plain dicts.  From it this module

* writes the ``input.dat`` text the reference parses (``write_input_dat``),
  so the reference solver can be run on exactly the same case, and
* computes the initial particle state that ``setting_vis_cons`` /
  ``setting_par`` / ``celllist_ini1`` produce (``initialise``,
  CPP_2-initialf.cpp:1021-1381, CPP_3-NNPS.cpp:96-121), so the GPU engine can
  be started without the reference present.

The generators build the workloads the engine is measured on: a 2-D water dam
break in a walled tank, and a 3-D saturated soil column (Drucker-Prager soil
with co-located pore water) collapsing in a walled box.  Lattice sites sit at
cell centres ``(i + 1/2) dx``; nothing is random.
"""
from __future__ import annotations

import copy
import os
import math
from dataclasses import dataclass, field

import numpy as np

# Para_Fluid / Para_Soil / Para_Structure member order (Class_ParticleProperty.h)
FLUID_FIELDS = ("vis", "vpu", "dens", "paa0", "porosity", "fai", "c",
                "bhtype", "press_type", "acc_type", "pre_coe", "strain_min")
SOIL_FIELDS = ("e", "poi", "eps0", "dens", "damp1", "damp2", "cop", "ramda", "kapa", "zmf",
               "ann", "bnn", "beta", "sitas", "sitar", "epsr", "epss", "sd", "sw", "kse",
               "c1", "c2", "c3", "fai", "c", "ocr", "sme0", "mzm", "azm", "r0",
               "bl", "bz", "zet", "vpu", "porosity", "fs", "etao", "g0", "ds", "damp_coe")
STRUCT_FIELDS = ("dens", "eps0", "e", "poi", "vpu", "porosity", "cop")


def fluid_default() -> dict:
    """Para_Fluid::Para_Fluid (Class_ParticleProperty.cpp)."""
    d = {k: 0.0 for k in FLUID_FIELDS}
    d.update(bhtype=0, press_type=0, acc_type=0, strain_min=1.0)
    return d


def soil_default() -> dict:
    """Para_Soil::Para_Soil (Class_ParticleProperty.cpp): fs = ds = 1."""
    d = {k: 0.0 for k in SOIL_FIELDS}
    d.update(fs=1.0, ds=1.0)
    return d


@dataclass
class Scene:
    """One reference input deck."""
    name: str
    ndim: int
    dr: float
    dt: float
    loop: int
    xp: np.ndarray            # (n, 3) float64, z = 0 in 2-D
    vxp: np.ndarray           # (n, 3)
    ptype: np.ndarray         # (n,) int32  Particle::type
    matype: np.ndarray        # (n,) int32
    permtype: np.ndarray      # (n,) int32
    etype: np.ndarray         # (n,) int32
    flags: dict = field(default_factory=dict)     # block FL
    problem: dict = field(default_factory=dict)   # blocks PR XP AT GF IP BP
    water: list = field(default_factory=list)     # 3 Para_Fluid dicts (block WP)
    air: dict | None = None                       # block AP
    model_flags: tuple = (0,) * 10                # block MS: em sb dp um am bui pl ve focc ep
    soils: dict = field(default_factory=dict)     # {index: Para_Soil dict}, index = layer*10 + model
    structure: dict | None = None                 # block SM
    rain: dict | None = None                      # block RP (flr = 1)
    vibration: dict | None = None                 # block VL + vibra.dat (flv >= 1): ttime nsteps sttime edtime loads

    @property
    def n(self) -> int:
        return int(self.xp.shape[0])

    def n_active(self) -> int:
        """Particles of types 1-4 (water, soil, air, structure)."""
        t = self.ptype
        return int(np.count_nonzero((t >= 1) & (t <= 4)))


# --------------------------------------------------------------------------
# lattice helpers

def _grid(nx, ny, nz, dx, origin):
    """Cell-centre lattice, x fastest, z slowest.  (nx, ny, nz) >= 1."""
    ix = (np.arange(nx, dtype=np.float64) + 0.5) * dx + origin[0]
    iy = (np.arange(ny, dtype=np.float64) + 0.5) * dx + origin[1]
    iz = (np.arange(nz, dtype=np.float64) + 0.5) * dx + origin[2]
    Z, Y, X = np.meshgrid(iz, iy, ix, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def _grid2(nx, ny, dx, origin):
    ix = (np.arange(nx, dtype=np.float64) + 0.5) * dx + origin[0]
    iy = (np.arange(ny, dtype=np.float64) + 0.5) * dx + origin[1]
    Y, X = np.meshgrid(iy, ix, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)


def _assemble(parts):
    xp = np.concatenate([p[0] for p in parts]).astype(np.float64)
    n = xp.shape[0]
    ptype = np.concatenate([np.full(p[0].shape[0], p[1], np.int32) for p in parts])
    matype = np.concatenate([np.full(p[0].shape[0], p[2], np.int32) for p in parts])
    return xp, np.zeros((n, 3)), ptype, matype, np.zeros(n, np.int32), np.ones(n, np.int32)


# --------------------------------------------------------------------------
# scenes

def dam_break_2d(dx: float = 0.005, water=(0.4, 0.8), tank=(1.6, 1.0), layers: int = 3,
                 steps: int = 2000, c0_factor: float = 10.0, alpha: float = 0.1,
                 eps_xsph: float = 0.5, cfl: float = 0.2) -> Scene:
    """2-D weakly compressible dam break: a water column (type 1) against the
    left wall of a tank of 3 wall layers (type 0, matype 0).

    Tait-like EOS with B = rho0 c0^2 / 7 is expressed through the reference's
    press_type 0 (prep = rhop g dr pre_coe, CPP_2-initialf.cpp:1301-1302) with
    pre_coe = c0^2 / (7 g dr).  The reference ties h to the particle spacing
    (hl = dr), so h = dx here.  fls = 1 with a dummy elastic soil material of
    void ratio 1e8 keeps the fluid porosity at 1 - 1e-8: with fls = 0 every
    fluid porosity is exactly 1 and the porosity term of the continuity
    equation is 0/0 at step 1 (CPP_6-density.cpp:153-156)."""
    g = 9.81
    H = water[1]
    c0 = c0_factor * math.sqrt(2.0 * g * H)
    dt = cfl * dx / c0
    nwx, nwy = int(round(water[0] / dx)), int(round(water[1] / dx))
    ntx, nty = int(round(tank[0] / dx)), int(round(tank[1] / dx))
    parts = [(_grid2(nwx, nwy, dx, (0.0, 0.0)), 1, 0)]
    floor = _grid2(ntx + 2 * layers, layers, dx, (-layers * dx, -layers * dx))
    left = _grid2(layers, nty, dx, (-layers * dx, 0.0))
    right = _grid2(layers, nty, dx, (ntx * dx, 0.0))
    parts += [(floor, 0, 0), (left, 0, 0), (right, 0, 0)]
    xp, vxp, ptype, matype, permtype, etype = _assemble(parts)
    w = fluid_default()
    w.update(dens=1000.0, vis=1.0e-3, vpu=c0, press_type=0, acc_type=0, bhtype=0,
             pre_coe=c0 * c0 / (7.0 * g * dx), strain_min=1.0e-3)
    wmin = copy.deepcopy(w)
    dummy = soil_default()
    dummy.update(kapa=0.05, poi=0.3, dens=2000.0, cop=1.0e-4, eps0=1.0e8, e=1.0e7, ds=1.0e-3)
    return Scene(
        name=f"dam_break_2d_dx{dx:g}", ndim=2, dr=dx, dt=dt, loop=steps,
        xp=xp, vxp=vxp, ptype=ptype, matype=matype, permtype=permtype, etype=etype,
        flags=dict(fla=0, fls=1, flr=0, fli=0, flv=0, fleob=0, flts=0, flspv=0, flknl=1,
                   ntd=1, flbndy=1),
        problem=dict(threshold_min=0.1, threshold_max=0.12, fop=max(steps, 1), inip=0,
                     step_regu=100000000, dttype=1,
                     xsph=(eps_xsph, 0.0, 0.0), art_vis=((alpha, 0.0), (0.0, 0.0), (0.0, 0.0)),
                     art_stre_coe=0.0, g=(0.0, -g, 0.0),
                     interc=0.0, permtype=0, pers=0.0, perl=0.0, perm=0.0,
                     ss=(0, 0.0, 0.0, 0), if_cal=0, if_move=0, coe_bndy=0.3),
        water=[w, copy.deepcopy(wmin), copy.deepcopy(wmin)],
        model_flags=(1, 0, 0, 0, 0, 0, 0, 0, 0, 0),
        soils={0: dummy},
    )


def soil_column_3d(dx: float = 0.005, block=(1.0, 0.5, 0.5), box=(2.0, 0.5, 0.6),
                   layers: int = 3, steps: int = 5000, with_water: bool = True) -> Scene:
    """3-D saturated soil column collapse: a Drucker-Prager soil block
    (type 2, matype 2: E = 10 MPa, nu = 0.3, phi = 30 deg, c = 0,
    rho_s = 2650, e0 = 0.6667 so porosity 0.4) overlapped site for site by
    pore water (type 1), standing against the back wall of a box with a
    3-layer floor, back wall and two side walls (type 0).  Darcy drag
    (fli = 1, permeability 1e-4 m/s), gravity -z, and the reference's
    variable time step (dttype = 2: dt = 0.25 dr / 600,
    CPP_12-2-dt.cpp:13-20)."""
    g = 9.81
    nbx, nby, nbz = (int(round(b / dx)) for b in block)
    nox, noy, noz = (int(round(b / dx)) for b in box)
    L = layers
    soil = _grid(nbx, nby, nbz, dx, (0.0, 0.0, 0.0))
    parts = [(soil, 2, 2)]
    if with_water:
        parts.append((soil.copy(), 1, 0))
    floor = _grid(nox + L, noy + 2 * L, L, dx, (-L * dx, -L * dx, -L * dx))
    back = _grid(L, noy + 2 * L, noz, dx, (-L * dx, -L * dx, 0.0))
    side0 = _grid(nox, L, noz, dx, (0.0, -L * dx, 0.0))
    side1 = _grid(nox, L, noz, dx, (0.0, noy * dx, 0.0))
    parts += [(floor, 0, 0), (back, 0, 0), (side0, 0, 0), (side1, 0, 0)]
    xp, vxp, ptype, matype, permtype, etype = _assemble(parts)
    dt_var = 0.25 * dx / 600.0
    w = fluid_default()
    w.update(dens=1000.0, vis=1.0e-3, vpu=30.0, press_type=0, acc_type=0, bhtype=0,
             pre_coe=30.0 * 30.0 / (7.0 * g * dx), strain_min=1.0e-3)
    dp = soil_default()
    dp.update(kapa=0.05, poi=0.3, dens=2650.0, c=0.0, fai=30.0, fs=1.0,
              damp1=0.0, damp2=0.0, cop=1.0e-4, eps0=0.6667, e=1.0e7, ds=1.0e-3)
    return Scene(
        name=f"soil_column_3d_dx{dx:g}", ndim=3, dr=dx,
        dt=dt_var * steps,            # dttype 2: the input dt is the total time
        loop=steps,
        xp=xp, vxp=vxp, ptype=ptype, matype=matype, permtype=permtype, etype=etype,
        flags=dict(fla=0, fls=1, flr=0, fli=1, flv=0, fleob=0, flts=0, flspv=0, flknl=1,
                   ntd=1, flbndy=1),
        problem=dict(threshold_min=0.1, threshold_max=0.12, fop=max(steps, 1), inip=0,
                     step_regu=100000000, dttype=2,
                     xsph=(0.5, 0.1, 0.0), art_vis=((0.1, 0.0), (0.1, 0.0), (0.0, 0.0)),
                     art_stre_coe=0.0, g=(0.0, 0.0, -g),
                     interc=1.0, permtype=0, pers=1.0e-4, perl=1.0e-4, perm=1.0e-4,
                     ss=(0, 0.0, 0.0, 0), if_cal=0, if_move=0, coe_bndy=0.3),
        water=[w, copy.deepcopy(w), copy.deepcopy(w)],
        model_flags=(0, 0, 1, 0, 0, 0, 0, 0, 0, 0),
        soils={2: dp},
    )


def slope_2d(H: float = 5.0, dx: float = 0.05, crest: float = 6.25, gradient: float = 1.5,
             runout: float | None = None, layers: int = 3, steps: int = 20000, c: float = 10.0e3,
             fai: float = 25.0, E: float = 2.0e7, art_stre_coe: float = 0.0, matype: int = 2) -> Scene:
    """2-D cohesive-frictional slope: a soil body (type 2, Drucker-Prager,
    rho = 2000, E = 20 MPa, nu = 0.3, dry) of height H with a crest of
    `crest` metres behind a 1:`gradient` face, on a 3-layer floor between a
    back wall and a far wall (type 0).  Soil area = crest H + gradient H^2 / 2
    (20,000 particles at H = 5, dx = 0.05)."""
    g = 9.81
    if runout is None:
        runout = max(1.0, 0.5 * H)
    L = crest + gradient * H + runout
    nx, ny = int(round(L / dx)), int(round((H + 2 * dx) / dx))
    grid = _grid2(nx, ny, dx, (0.0, 0.0))
    x, y = grid[:, 0], grid[:, 1]
    inside = (y < H) & ((x < crest) | (y < H - (x - crest) / gradient))
    soil = grid[inside]
    wall_h = H + 4 * dx
    nwy = int(round(wall_h / dx))
    parts = [(soil, 2, matype)]
    parts.append((_grid2(nx + 2 * layers, layers, dx, (-layers * dx, -layers * dx)), 0, 0))
    parts.append((_grid2(layers, nwy, dx, (-layers * dx, 0.0)), 0, 0))
    parts.append((_grid2(layers, nwy, dx, (nx * dx, 0.0)), 0, 0))
    xp, vxp, ptype, mt, permtype, etype = _assemble(parts)
    dp = soil_default()
    dp.update(kapa=0.05, poi=0.3, dens=2000.0, c=c, fai=fai, fs=1.0, beta=0.0,
              damp1=0.0, damp2=0.0, cop=1.0e-4, eps0=0.0, e=E, ds=1.0e-3)
    w = fluid_default()
    w.update(dens=1000.0, vis=1.0e-3, vpu=30.0, press_type=0, acc_type=0, bhtype=0,
             pre_coe=30.0 * 30.0 / (7.0 * g * dx), strain_min=1.0e-3)
    mflags = [0] * 10
    mflags[matype % 10] = 1
    return Scene(
        name=f"slope_2d_H{H:g}_dx{dx:g}", ndim=2, dr=dx, dt=0.25 * dx / 600.0 * steps, loop=steps,
        xp=xp, vxp=vxp, ptype=ptype, matype=mt, permtype=permtype, etype=etype,
        flags=dict(fla=0, fls=1, flr=0, fli=0, flv=0, fleob=0, flts=0, flspv=0, flknl=1,
                   ntd=1, flbndy=1),
        problem=dict(threshold_min=0.1, threshold_max=0.12, fop=max(steps, 1), inip=0,
                     step_regu=100000000, dttype=2,
                     xsph=(0.5, 0.1, 0.0), art_vis=((0.1, 0.0), (0.1, 0.0), (0.0, 0.0)),
                     art_stre_coe=art_stre_coe, g=(0.0, -g, 0.0),
                     interc=0.0, permtype=0, pers=0.0, perl=0.0, perm=0.0,
                     ss=(0, 0.0, 0.0, 0), if_cal=0, if_move=0, coe_bndy=0.3),
        water=[w, copy.deepcopy(w), copy.deepcopy(w)],
        model_flags=tuple(mflags),
        soils={matype: dp},
    )


def footing(ndim: int = 2, dx: float = 0.04, bed=(2.0, 1.0, 1.0), width: float = 0.4, height: float = 0.12,
            gap: float = 0.8, v: float = 0.5, ss_type: int = 3, myu: float = 0.3, zeta: float = 0.0,
            layers: int = 3, steps: int = 10000, matype: int = 2) -> Scene:
    """A rigid strip footing pushed into a soil bed: the soil (type 2,
    Drucker-Prager by default) fills bed[0] x bed[1] (x bed[2] in 3-D) on a
    3-layer floor between side walls (type 0); the footing (type 4, etype 5,
    E = 30 GPa) is `width` wide (and bed[2] long in 3-D), `height` tall, centred
    over the bed, its lowest layer `gap` spacings above the top soil layer; it
    moves down at v m/s (if_move 3) and meets the soil through the
    soil-structure contact of type ss_type (1 rigid, 2 deformable, 3 penalty)
    with friction coefficient myu and damping zeta."""
    g = 9.81
    L, D = bed[0], bed[1]
    nx, ny = int(round(L / dx)), int(round(D / dx))
    nf, nh = int(round(width / dx)), int(round(height / dx))
    x0f = (nx - nf) // 2 * dx
    yf = (ny - 0.5 + gap) * dx          # the footing's lowest layer, gap spacings above the soil's top layer
    wall_h = D + height + 4 * dx
    nwy = int(round(wall_h / dx))
    if ndim == 2:
        soil = _grid2(nx, ny, dx, (0.0, 0.0))
        foot = _grid2(nf, nh, dx, (x0f, 0.0))
        foot[:, 1] += yf - foot[:, 1].min()
        parts = [(soil, 2, matype), (foot, 4, 0)]
        parts.append((_grid2(nx + 2 * layers, layers, dx, (-layers * dx, -layers * dx)), 0, 0))
        parts.append((_grid2(layers, nwy, dx, (-layers * dx, 0.0)), 0, 0))
        parts.append((_grid2(layers, nwy, dx, (nx * dx, 0.0)), 0, 0))
        gvec, mv = (0.0, -g, 0.0), (0.0, -v, 0.0)
    else:
        nz = int(round(bed[2] / dx))
        soil = _grid(nx, ny, nz, dx, (0.0, 0.0, 0.0))
        foot = _grid(nf, nh, nz, dx, (x0f, 0.0, 0.0))
        foot[:, 1] += yf - foot[:, 1].min()
        parts = [(soil, 2, matype), (foot, 4, 0)]
        parts.append((_grid(nx + 2 * layers, layers, nz + 2 * layers, dx, (-layers * dx, -layers * dx, -layers * dx)), 0, 0))
        parts.append((_grid(layers, nwy, nz, dx, (-layers * dx, 0.0, 0.0)), 0, 0))
        parts.append((_grid(layers, nwy, nz, dx, (nx * dx, 0.0, 0.0)), 0, 0))
        parts.append((_grid(nx, nwy, layers, dx, (0.0, 0.0, -layers * dx)), 0, 0))
        parts.append((_grid(nx, nwy, layers, dx, (0.0, 0.0, nz * dx)), 0, 0))
        gvec, mv = (0.0, -g, 0.0), (0.0, -v, 0.0)
    xp, vxp, ptype, mt, permtype, etype = _assemble(parts)
    etype[ptype == 4] = 5
    dp = soil_default()
    dp.update(kapa=0.05, poi=0.3, dens=2000.0, c=5.0e3, fai=30.0, fs=1.0, beta=0.0,
              damp1=0.0, damp2=0.0, cop=1.0e-4, eps0=0.0, e=2.0e7, ds=1.0e-3)
    w = fluid_default()
    w.update(dens=1000.0, vis=1.0e-3, vpu=30.0, press_type=0, acc_type=0, bhtype=0,
             pre_coe=30.0 * 30.0 / (7.0 * g * dx), strain_min=1.0e-3)
    mflags = [0] * 10
    mflags[matype % 10] = 1
    return Scene(
        name=f"footing_{ndim}d_dx{dx:g}_ss{ss_type}", ndim=ndim, dr=dx, dt=0.25 * dx / 600.0 * steps, loop=steps,
        xp=xp, vxp=vxp, ptype=ptype, matype=mt, permtype=permtype, etype=etype,
        flags=dict(fla=0, fls=1, flr=0, fli=0, flv=0, fleob=0, flts=0, flspv=0, flknl=1,
                   ntd=1, flbndy=1),
        problem=dict(threshold_min=0.1, threshold_max=0.12, fop=max(steps, 1), inip=0,
                     step_regu=100000000, dttype=2,
                     xsph=(0.5, 0.1, 0.0), art_vis=((0.1, 0.0), (0.1, 0.0), (0.0, 0.0)),
                     art_stre_coe=0.0, g=gvec,
                     interc=0.0, permtype=0, pers=0.0, perl=0.0, perm=0.0,
                     ss=(ss_type, myu, zeta, 0), if_cal=0, if_move=3, coe_bndy=0.3, move_vx=mv),
        water=[w, copy.deepcopy(w), copy.deepcopy(w)],
        model_flags=tuple(mflags),
        soils={matype: dp},
        structure=dict(dens=2500.0, eps0=0.0, cop=0.0, e=3.0e10, poi=0.2),
    )


def shaking_box(ndim: int = 2, flv: int = 1, dx: float = 0.05, box=(2.0, 1.0, 0.4), layers: int = 3,
                steps: int = 40, ff_columns: int = 2, damp=(0.5, 0.02), amplitude: float | None = None,
                window=(3, 30)) -> Scene:
    """A soil block on a shaking base (vibration, flv 1 or 2): Drucker-Prager
    soil (type 2, matype 2, E = 20 MPa, rho = 2000) of box[0] x box[1]
    (x box[2] in 3-D) with free-field columns of `ff_columns` particles at
    both x ends (matype 52, the same material; permtype 1 on the left, 2 on
    the right: the wave direction ff_stress reads), on a `layers`-layer floor
    between side walls.  The floor takes the vibration load: matype 3
    (flv 1, acceleration) or 4 (flv 2, velocity), matype 5 under the
    free-field columns; the side walls are matype 5 (permtype 1 / 2).  Soil
    damping damp1, damp2 (soil_damping_vibration).  The load table: 20
    entries per period of 40 steps, a sine in x with a smaller cosine in y
    (amplitude 2 m/s^2 or 0.05 m/s), one entry of 1500 (the reference's
    cut-off), applied between steps window[0] and window[1] (sttime and
    edtime as multiples of dt)."""
    g = 9.81
    L = layers
    nx, ny = int(round(box[0] / dx)), int(round(box[1] / dx))
    parts = []
    if ndim == 2:
        soil = _grid2(nx, ny, dx, (0.0, 0.0))
        xs = soil[:, 0]
        ffl = xs < ff_columns * dx
        ffr = xs > (nx - ff_columns) * dx
        core = ~(ffl | ffr)
        parts += [(soil[core], 2, 2), (soil[ffl], 2, 52), (soil[ffr], 2, 52)]
        floor = _grid2(nx + 2 * L, L, dx, (-L * dx, -L * dx))
        fx = floor[:, 0]
        under_ff = (fx < ff_columns * dx) | (fx > (nx - ff_columns) * dx)
        parts += [(floor[~under_ff], 0, 3 if flv == 1 else 4), (floor[under_ff], 0, 5)]
        nwy = ny + 2
        parts += [(_grid2(L, nwy, dx, (-L * dx, 0.0)), 0, 5), (_grid2(L, nwy, dx, (nx * dx, 0.0)), 0, 5)]
        grav = (0.0, -g, 0.0)
    else:
        nz = int(round(box[2] / dx))
        soil = _grid(nx, nz, ny, dx, (0.0, 0.0, 0.0))       # y across, z up
        xs = soil[:, 0]
        ffl = xs < ff_columns * dx
        ffr = xs > (nx - ff_columns) * dx
        core = ~(ffl | ffr)
        parts += [(soil[core], 2, 2), (soil[ffl], 2, 52), (soil[ffr], 2, 52)]
        floor = _grid(nx + 2 * L, nz + 2 * L, L, dx, (-L * dx, -L * dx, -L * dx))
        fx = floor[:, 0]
        under_ff = (fx < ff_columns * dx) | (fx > (nx - ff_columns) * dx)
        parts += [(floor[~under_ff], 0, 3 if flv == 1 else 4), (floor[under_ff], 0, 5)]
        nwz = ny + 2
        parts += [(_grid(L, nz + 2 * L, nwz, dx, (-L * dx, -L * dx, 0.0)), 0, 5),
                  (_grid(L, nz + 2 * L, nwz, dx, (nx * dx, -L * dx, 0.0)), 0, 5),
                  (_grid(nx, L, nwz, dx, (0.0, -L * dx, 0.0)), 0, 0),
                  (_grid(nx, L, nwz, dx, (0.0, nz * dx, 0.0)), 0, 0)]
        grav = (0.0, 0.0, -g)
    xp, vxp, ptype, mt, permtype, etype = _assemble(parts)
    # wave directions: left free-field soil and left wall 1, right 2
    left = xp[:, 0] < 0.5 * nx * dx
    sel = (mt == 52) | (mt == 5)
    permtype[sel & left] = 1
    permtype[sel & ~left] = 2
    dt = 0.25 * dx / 600.0
    dp = soil_default()
    dp.update(kapa=0.05, poi=0.3, dens=2000.0, c=5.0e3, fai=30.0, fs=1.0, beta=0.0,
              damp1=damp[0], damp2=damp[1], cop=1.0e-4, eps0=0.0, e=2.0e7, ds=1.0e-3)
    w = fluid_default()
    w.update(dens=1000.0, vis=1.0e-3, vpu=30.0, press_type=0, acc_type=0, bhtype=0,
             pre_coe=30.0 * 30.0 / (7.0 * g * dx), strain_min=1.0e-3)
    nsteps = 20
    amp = amplitude if amplitude is not None else (2.0 if flv == 1 else 0.05)
    ph = 2.0 * np.pi * np.arange(nsteps) / nsteps
    loads = np.stack([amp * np.sin(ph), 0.3 * amp * np.cos(ph), 0.1 * amp * np.sin(2 * ph)], axis=1)
    loads[7, 0] = 1500.0
    vib = dict(ttime=40 * dt, nsteps=nsteps, sttime=window[0] * dt, edtime=window[1] * dt, loads=loads)
    return Scene(
        name=f"shaking_box_{ndim}d_flv{flv}_dx{dx:g}", ndim=ndim, dr=dx, dt=dt, loop=steps,
        xp=xp, vxp=vxp, ptype=ptype, matype=mt, permtype=permtype, etype=etype,
        flags=dict(fla=0, fls=1, flr=0, fli=0, flv=flv, fleob=0, flts=0, flspv=0, flknl=1,
                   ntd=1, flbndy=1),
        problem=dict(threshold_min=0.1, threshold_max=0.12, fop=max(steps, 1), inip=0,
                     step_regu=100000000, dttype=1,
                     xsph=(0.5, 0.1, 0.0), art_vis=((0.1, 0.0), (0.1, 0.0), (0.0, 0.0)),
                     art_stre_coe=0.0, g=grav,
                     interc=0.0, permtype=0, pers=0.0, perl=0.0, perm=0.0,
                     ss=(0, 0.0, 0.0, 0), if_cal=0, if_move=0, coe_bndy=0.3),
        water=[w, copy.deepcopy(w), copy.deepcopy(w)],
        model_flags=(0, 0, 1, 0, 0, 0, 0, 0, 0, 0),
        soils={2: dp},
        vibration=vib,
    )


def rain_slope_3d(dx: float = 0.05, H: float = 5.0, crest: float = 6.25, gradient: float = 1.5,
                  width: float = 10.0, length: float = 20.0, rows: int = 3, steps: int = 20000,
                  layers: int = 3) -> Scene:
    """A 3-D rainfall slope with three phases (fla 1): the 1:`gradient` slope
    of height H behind a `crest`-metre crest, extruded `width` metres across
    (y; z up), in a `length`-metre box with a `layers`-layer floor, a back
    wall and two side walls (type 0).  Drucker-Prager soil (type 2, phi 25
    deg, c 10 kPa, E 20 MPa, rho 2000, porosity 0.4) holds co-located pore
    air (type 3); `rows` rows of rain (type 7) over the crest fall as water
    (rainfall type 1, lp = steps / (rows + 1)) and drain through the soil by
    Darcy drag (fli 1, permeability 1e-4 m/s)."""
    g = 9.81
    nx, nw = int(round(length / dx)), int(round(width / dx))
    nz = int(round((H + 2 * dx) / dx))
    grid = _grid(nx, nw, nz, dx, (0.0, 0.0, 0.0))
    x, z = grid[:, 0], grid[:, 2]
    inside = (z < H) & ((x < crest) | (z < H - (x - crest) / gradient))
    soil = grid[inside]
    L = layers
    wall_h = H + 6 * dx
    nwz = int(round(wall_h / dx))
    parts = [(soil, 2, 2), (soil.copy(), 3, 0)]
    parts.append((_grid(nx + L, nw + 2 * L, L, dx, (-L * dx, -L * dx, -L * dx)), 0, 0))
    parts.append((_grid(L, nw + 2 * L, nwz, dx, (-L * dx, -L * dx, 0.0)), 0, 0))
    parts.append((_grid(nx, L, nwz, dx, (0.0, -L * dx, 0.0)), 0, 0))
    parts.append((_grid(nx, L, nwz, dx, (0.0, nw * dx, 0.0)), 0, 0))
    xp, vxp, ptype, mt, permtype, etype = _assemble(parts)
    dp = soil_default()
    dp.update(kapa=0.05, poi=0.3, dens=2000.0, c=10.0e3, fai=25.0, fs=1.0, beta=0.0,
              damp1=0.0, damp2=0.0, cop=1.0e-4, eps0=0.6667, e=2.0e7, ds=1.0e-3)
    w = fluid_default()
    w.update(dens=1000.0, vis=1.0e-3, vpu=30.0, press_type=0, acc_type=0, bhtype=0,
             pre_coe=30.0 * 30.0 / (7.0 * g * dx), strain_min=1.0e-3)
    air = dict(dens=1.293, paa0=100.0, vis=1.8e-5, vpu=30.0, press_type=0, acc_type=0, pre_coe=0.0)
    sc = Scene(
        name=f"rain_slope_3d_dx{dx:g}", ndim=3, dr=dx, dt=0.25 * dx / 600.0 * steps, loop=steps,
        xp=xp, vxp=vxp, ptype=ptype, matype=mt, permtype=permtype, etype=etype,
        flags=dict(fla=1, fls=1, flr=0, fli=1, flv=0, fleob=0, flts=0, flspv=0, flknl=1,
                   ntd=1, flbndy=1),
        problem=dict(threshold_min=0.1, threshold_max=0.12, fop=max(steps, 1), inip=0,
                     step_regu=100000000, dttype=2,
                     xsph=(0.5, 0.1, 0.0), art_vis=((0.1, 0.0), (0.1, 0.0), (0.0, 0.0)),
                     art_stre_coe=0.0, g=(0.0, 0.0, -g),
                     interc=1.0, permtype=0, pers=1.0e-4, perl=1.0e-4, perm=1.0e-4,
                     ss=(0, 0.0, 0.0, 0), if_cal=0, if_move=0, coe_bndy=0.3),
        water=[w, copy.deepcopy(w), copy.deepcopy(w)],
        air=air,
        model_flags=(0, 0, 1, 0, 0, 0, 0, 0, 0, 0),
        soils={2: dp},
    )
    return add_rain(sc, 0.0, crest, rows, H + 2 * dx)


def add_rain(scene: Scene, x0: float, x1: float, rows: int, top: float, press_factor: float = 1.0,
             drop_velocity: float = -1.0) -> Scene:
    """Rain particles (type 7, etype 1: water waiting to fall) appended to
    the scene in `rows` rows of one spacing's pitch above height `top` (y in
    2-D, z in 3-D), each row spanning [x0, x1) at the spacing (and the
    scene's z or y extent in 3-D), the lowest row first since the reference
    releases them in array order (rainpro, CPP_15-1-rain.cpp:43-85); rainfall
    type 1 with nhor = the row's particle count (input block RP)."""
    dx = scene.dr
    nx = int(round((x1 - x0) / dx))
    blocks = []
    for r in range(rows):
        h = top + (r + 0.5) * dx
        if scene.ndim == 2:
            row = _grid2(nx, 1, dx, (x0, 0.0))
            row[:, 1] = h
        else:
            lo, hi = scene.xp[:, 1].min(), scene.xp[:, 1].max()
            ny = max(int(round((hi - lo) / dx)), 1)
            row = _grid(nx, ny, 1, dx, (x0, lo, 0.0))
            row[:, 2] = h
        blocks.append(row)
    rain = np.concatenate(blocks)
    m = rain.shape[0]
    scene.xp = np.concatenate([scene.xp, rain])
    scene.vxp = np.concatenate([scene.vxp, np.zeros((m, 3))])
    scene.ptype = np.concatenate([scene.ptype, np.full(m, 7, np.int32)])
    scene.matype = np.concatenate([scene.matype, np.zeros(m, np.int32)])
    scene.permtype = np.concatenate([scene.permtype, np.zeros(m, np.int32)])
    scene.etype = np.concatenate([scene.etype, np.ones(m, np.int32)])
    scene.flags["flr"] = 1
    scene.rain = dict(rtype=1, nrain=m, nhor=m // rows, press_factor=press_factor, drop_velocity=drop_velocity)
    return scene


def uplift(scene: Scene, axis: int, above: float, v: float = 0.5) -> Scene:
    """Give the soil particles (type 2) above coordinate `above` along `axis`
    an initial velocity v along that axis, which stretches the soil body and
    puts its upper part in tension (used with art_stre_coe > 0 so that the
    tensile branch of the artificial stress acts)."""
    up = (scene.ptype == 2) & (scene.xp[:, axis] > above)
    scene.vxp[up, axis] = v
    return scene


# Para_Soil members each soil model's input block sets (CPP_2-initialf.cpp:
# 490-805); the others keep Para_Soil's defaults
_BASE = ("damp1", "damp2", "cop", "eps0", "e", "ds")
MODEL_FIELDS = {
    0: ("kapa", "poi", "dens") + _BASE,
    1: ("poi", "dens", "eps0", "zmf", "sme0", "fs", "ramda", "kapa", "damp1", "damp2", "cop", "ann", "ocr", "e", "ds"),
    2: ("kapa", "poi", "dens", "c", "fai", "fs") + _BASE,
    3: ("poi", "dens", "eps0", "zmf", "sme0", "fs", "ramda", "kapa", "damp1", "damp2", "cop",
        "ann", "bnn", "beta", "epss", "epsr", "sitas", "sitar", "sd", "sw", "kse", "c1", "c2", "c3",
        "e", "ds"),
    4: ("poi", "dens", "eps0", "zmf", "sme0", "fs", "ramda", "kapa", "damp1", "damp2", "cop",
        "mzm", "azm", "r0", "bl", "bz", "zet", "e", "ds"),
    5: ("kapa", "poi", "dens", "c", "fai", "beta", "fs") + _BASE,
    6: ("kapa", "poi", "dens") + _BASE,
    7: ("kapa", "poi", "dens", "c") + _BASE,
    8: ("dens", "c", "eps0", "cop", "sme0", "g0", "poi", "zmf", "ramda", "etao", "zet", "ann", "bnn",
        "damp1", "damp2", "ds"),
    9: ("kapa", "poi", "dens", "c", "fai", "fs") + _BASE,
}

# the input blocks of models 3, 4 and 8, line by line (CPP_2-initialf.cpp:
# 573-639, 719-740); model 8's reader then sets e = 5e6
_BLOCKS = {
    3: ("UM unsaturated cam-clay", (("poi", "dens", "eps0", "zmf", "sme0", "fs"),
                                    ("ramda", "kapa", "damp1", "damp2", "cop"),
                                    ("ann", "bnn", "beta", "epss", "epsr", "sitas", "sitar"),
                                    ("sd", "sw", "kse", "c1", "c2", "c3"), ("e", "ds"))),
    4: ("AM anisotropic cam-clay", (("poi", "dens", "eps0", "zmf", "sme0", "fs"),
                                    ("ramda", "kapa", "damp1", "damp2", "cop"),
                                    ("mzm", "azm", "r0", "bl", "bz", "zet"), ("e", "ds"))),
    8: ("FC fractional order cam-clay", (("dens", "c", "eps0", "cop", "sme0"),
                                         ("g0", "poi", "zmf", "ramda", "etao"),
                                         ("zet", "ann", "bnn", "damp1", "damp2"), ("ds",))),
}


def set_soil_model(scene: Scene, matype: int, **record) -> Scene:
    """Switch every soil particle (type 2) to constitutive model `matype`
    (0 elastic, 1 subloading Cam-clay, 2 Drucker-Prager, 3 unsaturated
    Cam-clay, 4 anisotropic Cam-clay, 5 Bui DP, 6 elastic, 7 viscous-elastic,
    8 fractional-order Cam-clay, 9 Mohr-Coulomb; one layer).  The record holds the
    members that model's input block reads, from `record`, else from the
    previous soil record; the others keep Para_Soil's defaults."""
    old = next(iter(scene.soils.values())) if scene.soils else soil_default()
    rec = soil_default()
    for k in MODEL_FIELDS[matype % 10]:      # what the model's input block sets
        rec[k] = record.get(k, old.get(k, rec[k]))
    unknown = set(record) - set(MODEL_FIELDS[matype % 10])
    if unknown:
        raise ValueError(f"model {matype} does not read {sorted(unknown)}")
    scene.matype[scene.ptype == 2] = matype
    scene.soils = {matype: rec}
    flags = [0] * 10
    flags[matype % 10] = 1
    scene.model_flags = tuple(flags)
    return scene


def keep(scene: Scene, mask: np.ndarray) -> Scene:
    """The scene with only the particles where `mask` is true, in their order."""
    m = np.asarray(mask, bool)
    for name in ("xp", "vxp", "ptype", "matype", "permtype", "etype"):
        setattr(scene, name, getattr(scene, name)[m].copy())
    return scene


def scaled_loop(scene: Scene) -> int:
    """Steps the reference will run: for dttype 2 the loop count is
    int(tt / dt) + 1 with tt the input dt (CPP_12-2-dt.cpp:13-20)."""
    if scene.problem["dttype"] == 2:
        dtv = 0.25 * scene.dr / 600.0
        return int(scene.dt / dtv) + 1
    return scene.loop


# --------------------------------------------------------------------------
# input.dat writer (the format initial_pro / initial_mat / input_par scan)

def _f(v) -> str:
    return repr(float(v))


def write_input_dat(scene: Scene, path: str, ntd: int = 1) -> None:
    """Write ``scene`` as a reference input deck.  Block markers are two
    characters or more ('A data', 'E end'): the reference's scanner
    (``%c%*[^\\n]%*c``) mis-reads one-character lines."""
    P, F = scene.problem, scene.flags
    L = []
    add = L.append
    add("FL flags")
    add("A data")
    add(" ".join(str(F[k]) for k in ("fla", "fls", "flr", "fli", "flv", "fleob", "flts", "flspv", "flknl")))
    add(f"{ntd} {F['flbndy']}")
    add("E end")
    add("PR problem")
    add("A data")
    add(f"{scene.ndim} {_f(P['threshold_min'])} {_f(P['threshold_max'])}")
    add(f"{P['fop']} {P['inip']} {scene.loop} {scene.n} {P['step_regu']}")
    add(f"{P['dttype']} {_f(scene.dr)} {_f(scene.dt)}")
    add("E end")
    add("XP xsph")
    add("A data")
    add(" ".join(_f(v) for v in P["xsph"]))
    add("E end")
    add("AT artificial viscosity")
    add("A data")
    av = P["art_vis"]
    add(f"{_f(av[0][0])} {_f(av[0][1])}")
    add(f"{_f(av[1][0])} {_f(av[1][1])} {_f(P['art_stre_coe'])}")
    add(f"{_f(av[2][0])} {_f(av[2][1])}")
    add("E end")
    add("GF gravity")
    add("A data")
    add(" ".join(_f(v) for v in P["g"]))
    add("E end")
    add("IP interaction")
    add("A data")
    add(_f(P["interc"]))
    add(f"{P['permtype']} {_f(P['pers'])} {_f(P['perl'])} {_f(P['perm'])}")
    ss = P["ss"]
    add(f"{ss[0]} {_f(ss[1])} {_f(ss[2])} {ss[3]}")
    add("E end")
    add("BP boundary")
    add("A data")
    add(f"{P['if_cal']} {P['if_move']} {_f(P['coe_bndy'])}")
    if P["if_move"] >= 1:
        add(" ".join(_f(v) for v in P.get("move_vx", (0.0, 0.0, 0.0))))
    add("E end")
    if F["flv"] >= 1 and scene.vibration is not None:
        vb = scene.vibration
        add("VL vibration")
        add("A data")
        add(f"{_f(vb['ttime'])} {int(vb['nsteps'])}")
        add(f"{_f(vb['sttime'])} {_f(vb['edtime'])}")
        add("E end")
        # the loads, one row of three per step, in vibra.dat beside the deck
        # (initial_vib, CPP_2-initialf.cpp:292-320)
        with open(os.path.join(os.path.dirname(os.path.abspath(path)), "vibra.dat"), "w") as fv:
            for row in np.asarray(vb["loads"], dtype=np.float64).reshape(-1, 3):
                fv.write(" ".join(_f(v) for v in row) + "\n")
    if F["flr"] == 1 and scene.rain is not None:
        rn = scene.rain
        add("RP rain")
        add("A data")
        add(f"{rn['rtype']} {rn['nrain']} {rn['nhor']} {_f(rn['press_factor'])} {_f(rn['drop_velocity'])}")
        add("E end")
    add("WP water")
    add("A data")
    w0 = scene.water[0]
    add(" ".join([_f(w0["dens"]), _f(w0["vis"]), _f(w0["fai"]), _f(w0["c"]), _f(w0["vpu"]),
                  str(w0["press_type"]), str(w0["acc_type"]), str(w0["bhtype"]),
                  _f(w0["pre_coe"]), _f(w0["strain_min"])]))
    for w in scene.water[1:3]:
        add(" ".join(_f(w[k]) for k in ("dens", "vis", "fai", "c", "vpu")))
    add("E end")
    if scene.air is not None:
        a = scene.air
        add("AP air")
        add("A data")
        add(" ".join([_f(a["dens"]), _f(a["paa0"]), _f(a["vis"]), _f(a["vpu"]),
                      str(a["press_type"]), str(a["acc_type"]), _f(a["pre_coe"])]))
        add("E end")
    add("MS soil models")
    add("A data")
    add(" ".join(str(v) for v in scene.model_flags))
    if F["flts"] >= 1:
        add(" ".join(_f(v) for v in P.get("ts", (0.0, 0.0))))     # alphats, damp_coe
    add("E end")
    mf = scene.model_flags
    for flag, (title, lines) in _BLOCKS.items():
        if mf[flag] >= 1:
            add(title)
            add("A data")
            for layer in range(mf[flag]):
                s = scene.soils[layer * 10 + flag]
                for keys in lines:
                    add(" ".join(_f(s[k]) for k in keys))
            add("E end")
    if mf[0] >= 1:
        add("EM elastic")
        add("A data")
        for layer in range(mf[0]):
            s = scene.soils[layer * 10 + 0]
            add(" ".join(_f(s[k]) for k in ("kapa", "poi", "dens")))
            add(" ".join(_f(s[k]) for k in ("damp1", "damp2", "cop", "eps0")))
            add(" ".join(_f(s[k]) for k in ("e", "ds")))
        add("E end")
    if mf[1] >= 1:
        add("SB subloading cam-clay")
        add("A data")
        for layer in range(mf[1]):
            s = scene.soils[layer * 10 + 1]
            add(" ".join(_f(s[k]) for k in ("poi", "dens", "eps0", "zmf", "sme0", "fs")))
            add(" ".join(_f(s[k]) for k in ("ramda", "kapa", "damp1", "damp2", "cop")))
            add(" ".join(_f(s[k]) for k in ("ann", "ocr")))
            add(" ".join(_f(s[k]) for k in ("e", "ds")))
        add("E end")
    if mf[2] >= 1:
        add("DP drucker prager")
        add("A data")
        for layer in range(mf[2]):
            s = scene.soils[layer * 10 + 2]
            add(" ".join(_f(s[k]) for k in ("kapa", "poi", "dens", "c", "fai", "fs")))
            add(" ".join(_f(s[k]) for k in ("damp1", "damp2", "cop", "eps0")))
            add(" ".join(_f(s[k]) for k in ("e", "ds")))
        add("E end")
    if mf[5] >= 1:
        add("BU bui drucker prager")
        add("A data")
        for layer in range(mf[5]):
            s = scene.soils[layer * 10 + 5]
            add(" ".join(_f(s[k]) for k in ("kapa", "poi", "dens", "c", "fai", "beta", "fs")))
            add(" ".join(_f(s[k]) for k in ("damp1", "damp2", "cop", "eps0")))
            add(" ".join(_f(s[k]) for k in ("e", "ds")))
        add("E end")
    # PP (elastic record read for index 6), VE (viscous-elastic, c = shear
    # modulus) and EP (Mohr-Coulomb), CPP_2-initialf.cpp:666-805
    for flag, code, title, first in ((6, "PP", "plastic", ("kapa", "poi", "dens")),
                                     (7, "VE", "viscous elastic", ("kapa", "poi", "dens", "c")),
                                     (9, "EP", "elastic perfectly plastic", ("kapa", "poi", "dens", "c", "fai", "fs"))):
        if mf[flag] >= 1:
            add(f"{code} {title}")
            add("A data")
            for layer in range(mf[flag]):
                s = scene.soils[layer * 10 + flag]
                add(" ".join(_f(s[k]) for k in first))
                add(" ".join(_f(s[k]) for k in ("damp1", "damp2", "cop", "eps0")))
                add(" ".join(_f(s[k]) for k in ("e", "ds")))
            add("E end")
    if scene.structure is not None:
        st = scene.structure
        add("SM structure")
        add("A data")
        add(" ".join(_f(st[k]) for k in ("dens", "eps0", "cop")))
        add(" ".join(_f(st[k]) for k in ("e", "poi")))
        add("E end")
    add("PA particles")
    add("A data")
    xp, vxp = scene.xp, scene.vxp
    rows = []
    if scene.ndim == 2:
        for i in range(scene.n):
            rows.append(f"{_f(xp[i, 0])} {_f(xp[i, 1])} {_f(vxp[i, 0])} {_f(vxp[i, 1])} "
                        f"{scene.ptype[i]} {scene.matype[i]} {scene.permtype[i]} {scene.etype[i]}")
    else:
        for i in range(scene.n):
            rows.append(f"{_f(xp[i, 0])} {_f(xp[i, 1])} {_f(xp[i, 2])} {_f(vxp[i, 0])} {_f(vxp[i, 1])} "
                        f"{_f(vxp[i, 2])} {scene.ptype[i]} {scene.matype[i]} {scene.permtype[i]} {scene.etype[i]}")
    L.extend(rows)
    add("E end")
    with open(path, "w") as fh:
        fh.write("\n".join(L) + "\n")


# --------------------------------------------------------------------------
# initial state: initial_mat tail, setting_vis_cons, setting_par, input_par's
# domain box and celllist_ini1

def material_tables(scene: Scene):
    """The 30 Para_Soil slots, 3 water and 1 air Para_Fluid records after
    initial_mat (CPP_2-initialf.cpp:797-839)."""
    soils = [soil_default() for _ in range(30)]
    for idx, s in scene.soils.items():
        soils[idx] = dict(s)
    damp_coe = scene.problem.get("ts", (0.0, 0.0))[1] if scene.flags["flts"] >= 1 else 0.0
    for s in soils:
        s["vpu"] = 600.0
        s["damp_coe"] = damp_coe
    for layer in range(scene.model_flags[8]):
        soils[layer * 10 + 8]["e"] = 5.0e6
    water = [dict(fluid_default(), **w) for w in scene.water]
    for k in (1, 2):
        for key in ("press_type", "bhtype", "pre_coe", "strain_min"):
            water[k][key] = water[0][key]
    air = dict(fluid_default(), **(scene.air or {}))
    if scene.flags["fls"] == 0:
        por = 1.0
        for w in water:
            w["porosity"] = 1.0
        air["porosity"] = 1.0
    else:
        for s in soils:
            s["porosity"] = s["eps0"] / (1 + s["eps0"])
        por = 0.0
        for s in soils:
            por = max(por, s["porosity"])
        for w in water:
            w["porosity"] = por
        air["porosity"] = por
    for w in water:
        if w["dens"] <= 0.0:
            w["dens"] = 1000.0
    if air["dens"] <= 0.0:
        air["dens"] = 1.293
    st = dict({k: 0.0 for k in STRUCT_FIELDS}, **(scene.structure or {}))
    st["vpu"] = 600.0
    st["porosity"] = st["eps0"] / (1 + st["eps0"])
    return soils, water, air, st


def moisturesuct(satu: float, dsatu: float, soil) -> float:
    """Suction on the wetting (dsatu > 0) or drying curve,
    CPP_7-2-constitutive.cpp:323-338, with pi = 3.141592653."""
    temp = math.tan(3.141592653 * (soil["sitas"] - satu) / (soil["sitas"] - soil["sitar"]) / 2.0)
    if dsatu > 0.0:
        return math.log(1 + math.exp(soil["c2"] * soil["sw"]) * temp) / soil["c2"]
    return math.log(1 + math.exp(soil["c1"] * soil["sd"]) * temp) / soil["c1"]


@dataclass
class InitialState:
    params: dict          # sphgpu_params members
    fields: dict          # Particle member name -> array (n,) or (n, ncomp)
    fluid: np.ndarray     # (n, 12) records as sphgpu_fluid (structured dtype)
    soil: np.ndarray      # (n,) structured sphgpu_soil
    rain: dict | None = None   # sphgpu_rain members (flr = 1)
    vibration: dict | None = None   # Para_Vibra: ttime nsteps sttime edtime loads (flv >= 1)


FLUID_DTYPE = np.dtype([(k, np.int32 if k in ("bhtype", "press_type", "acc_type") else np.float64)
                        for k in FLUID_FIELDS], align=True)
SOIL_DTYPE = np.dtype([(k, np.float64) for k in SOIL_FIELDS], align=True)


def initialise(scene: Scene) -> InitialState:
    """Initial particle state as the reference's initialisation leaves it
    (vectorised; every expression keeps the reference's operation order)."""
    n, dim, dr = scene.n, scene.ndim, scene.dr
    soils, water, air, st = material_tables(scene)
    P = scene.problem
    gx, gy, gz = P["g"]
    t, mt, et = scene.ptype, scene.matype, scene.etype
    # setting_vis_cons (CPP_2-initialf.cpp:1021-1058)
    fdef = fluid_default()
    fl = np.zeros(n, FLUID_DTYPE)
    for k in FLUID_FIELDS:
        fl[k] = fdef[k]
    water_tab = np.zeros(3, FLUID_DTYPE)
    for q in range(3):
        water_tab[q] = tuple(water[q][k] for k in FLUID_FIELDS)
    is_w = (t == 1) | ((t == 7) & (et == 1))
    fl[is_w] = water_tab[np.clip(mt[is_w], 0, 2)]
    fl[t == 3] = tuple(air[k] for k in FLUID_FIELDS)
    sdef = soil_default()
    so = np.zeros(n, SOIL_DTYPE)
    for k in SOIL_FIELDS:
        so[k] = sdef[k]
    soil_tab = np.zeros(30, SOIL_DTYPE)
    for q in range(30):
        soil_tab[q] = tuple(soils[q][k] for k in SOIL_FIELDS)
    is_s = (t == 2) | ((t == 7) & (et == 2))
    idx = np.where(mt < 30, mt, np.where(mt >= 50, mt % 10, -1))
    sel = is_s & (idx >= 0)
    so[sel] = soil_tab[idx[sel]]

    f = {name: np.zeros((n, nc)) for name, nc in
         (("x", 3), ("vx", 3), ("ax", 3), ("axp", 3), ("ux", 3), ("strep", 3), ("interf", 3),
          ("interfss", 3), ("eps", 6), ("sig", 6), ("adps", 6))}
    f["tssig"] = np.zeros((n, 6))
    for name in ("rho", "rhop", "mass", "hl", "pre", "prep", "e", "satu", "dsatu", "suct", "cop", "porosity",
                 "cd", "poro_cop", "prew", "prea", "vsig", "veps", "divq", "divr", "meps", "tsqc"):
        f[name] = np.zeros(n)
    f["xp"] = scene.xp.copy()
    f["vxp"] = scene.vxp.copy()
    f["type"], f["matype"] = t.copy(), mt.copy()
    f["permtype"], f["etype"] = scene.permtype.copy(), et.copy()
    sitas = max(s_["sitas"] for s_ in soils)
    g_axp = np.array([gx, gy, gz])
    # setting_par first loop (:1088-1282)
    wall = t == 0
    f["rhop"][wall] = 1500.0
    f["satu"][wall] = sitas
    f["hl"][wall] = dr
    f["axp"][wall & (mt == 5)] = g_axp
    f["rhop"][is_w] = fl["porosity"][is_w] * fl["dens"][is_w]
    f["satu"][is_w] = sitas
    f["hl"][is_w] = dr
    f["axp"][is_w] = g_axp
    f["porosity"][is_w] = fl["porosity"][is_w]
    por = so["porosity"]
    f["rhop"][is_s] = (1 - por[is_s]) * so["dens"][is_s]
    m10 = mt % 10
    f["satu"][is_s] = 1.0
    um = is_s & np.isin(mt, (3, 13, 23, 53))
    f["satu"][um] = so["sitar"][um]
    f["e"][is_s] = so["eps0"][is_s]
    f["porosity"][is_s] = por[is_s]
    f["hl"][is_s] = dr
    f["axp"][is_s] = g_axp
    s7 = (t == 7) & (et == 2)
    f["cop"][s7] = so["cop"][s7]
    air_ = t == 3
    f["rhop"][air_] = fl["porosity"][air_] * fl["dens"][air_]
    f["hl"][air_] = dr
    f["axp"][air_] = g_axp
    stc = t == 4
    f["rhop"][stc] = (1 - st["porosity"]) * st["dens"]
    f["satu"][stc] = 1.0
    f["e"][stc] = st["eps0"]
    f["hl"][stc] = dr
    f["axp"][stc] = g_axp
    has_mass = (t == 0) | (t == 1) | (t == 2) | (t == 3) | (t == 4) | is_w | is_s
    h = f["hl"]
    if dim == 2:
        mass = f["rhop"] * h * h
    else:
        mass = f["rhop"] * h * h * h
    f["mass"][has_mass] = mass[has_mass]
    with np.errstate(divide="ignore", invalid="ignore"):
        cd_s = so["damp_coe"] * np.sqrt(so["e"] / f["rhop"] / h / h)
        cd_t = so["damp_coe"] * np.sqrt(st["e"] / f["rhop"] / h / h)
    f["cd"][is_s] = cd_s[is_s]
    f["cd"][stc] = cd_t[stc]
    f["rho"][:] = f["rhop"]
    z = scene.xp[:, dim - 1]
    hmaxw = max(-100000.0, float(z[t == 1].max())) if np.any(t == 1) else -100000.0
    hminw = min(100000.0, float(z[t == 1].min())) if np.any(t == 1) else 100000.0
    hmaxs = max(-100000.0, float(z[t == 2].max())) if np.any(t == 2) else -100000.0
    hmins = min(100000.0, float(z[t == 2].min())) if np.any(t == 2) else 100000.0
    g = gy if dim == 2 else gz
    # setting_par second loop (:1291-1369)
    f["prep"][wall] = 1500.0 * (-g) * abs(hmaxw - hminw) * 0.5
    f["pre"][wall] = f["prep"][wall]
    w1 = t == 1
    pc = fl["pre_coe"]
    pt0 = w1 & (fl["press_type"] == 0)
    f["prep"][pt0] = f["rhop"][pt0] * (-g) * dr * pc[pt0]
    pt1 = w1 & (fl["press_type"] != 0)
    f["prep"][pt1] = f["rhop"][pt1] * (-g) * np.abs(z[pt1] - hmaxw - pc[pt1] * dr)
    f["pre"][w1] = f["prep"][w1]
    w7 = (t == 7) & (et == 1)
    f["prep"][w7] = f["rhop"][w7] * (-g) * dr * pc[w7]
    f["pre"][w7] = f["prep"][w7]
    big = is_s & (np.abs(so["sme0"]) > 1.0e-3)
    for k in range(3):
        f["sig"][big, k] = -so["sme0"][big]
    geo = (t == 2) & ~big
    v = f["rho"][geo] * g * (hmaxs - hmins) * 0.5
    for k in range(3):
        f["sig"][geo, k] = v
    a0 = air_ & (fl["press_type"] == 0)
    f["prep"][a0] = fl["paa0"][a0]
    a1 = air_ & (fl["press_type"] != 0)
    f["prep"][a1] = fl["dens"][a1] * (-g) * np.abs(z[a1] - hmaxw - fl["pre_coe"][a1] * dr)
    f["pre"][air_] = f["prep"][air_]
    # suction of unsaturated Cam-clay soil, moisturesuct(satu, -1e-4) with the
    # C library's tan / exp / log (:1345-1346, 1356-1357)
    for i in np.nonzero(is_s & np.isin(mt, (3, 13, 23)))[0]:
        f["suct"][i] = moisturesuct(f["satu"][i], -0.0001, so[i])
    f.pop("roue", None)
    # input_par domain box (:917-1002) and celllist_ini1 (CPP_3-NNPS.cpp:96-121)
    bmax = np.maximum(scene.xp.max(axis=0), -10000.0)
    bmin = np.minimum(scene.xp.min(axis=0), 10000.0)
    for j in range(dim):
        bmax[j] = bmax[j] + 2.0 * dr
        bmin[j] = bmin[j] - 2.0 * dr
    cdr = 2.0 * dr
    cxm = int((bmax[0] - bmin[0]) / cdr + 3.0)
    cym = int((bmax[1] - bmin[1]) / cdr + 3.0)
    czm = int((bmax[2] - bmin[2]) / cdr + 3.0) if dim == 3 else 1
    dttype = P["dttype"]
    dt, loop = scene.dt, scene.loop
    if dttype == 2:
        tt = dt
        dt = 0.25 * dr / 600.0
        loop = int(tt / dt) + 1
    params = dict(
        ndim=dim, ntotal=n, fla=scene.flags["fla"], fls=scene.flags["fls"], flr=scene.flags["flr"],
        fli=scene.flags["fli"], flv=scene.flags["flv"], fleob=scene.flags["fleob"],
        flts=scene.flags["flts"], flspv=scene.flags["flspv"], flknl=scene.flags["flknl"],
        flbndy=scene.flags["flbndy"], inip=P["inip"], step_regu=P["step_regu"], loop=loop,
        fop=P["fop"], dr=dr, dt=dt, xsph=tuple(P["xsph"]), art_vis=tuple(map(tuple, P["art_vis"])),
        art_stre_coe=P["art_stre_coe"], gx=gx, gy=gy, gz=gz,
        threshold_min=P["threshold_min"], threshold_max=P["threshold_max"],
        interc=P["interc"], permtype=P["permtype"], pers=P["pers"], perl=P["perl"], perm=P["perm"],
        ss_type=P["ss"][0], ss_myu=P["ss"][1], ss_zeta=P["ss"][2], ss_acc_type=P["ss"][3],
        coe_bndy=P["coe_bndy"], if_cal=P["if_cal"], if_move=P["if_move"],
        move_vx=tuple(P.get("move_vx", (0.0, 0.0, 0.0))),
        xmin=bmin[0], xmax=bmax[0], ymin=bmin[1], ymax=bmax[1], zmin=bmin[2], zmax=bmax[2],
        cxm=cxm, cym=cym, czm=czm, ctotal=cxm * cym * czm,
        flagum=scene.model_flags[3],
        alphats=P.get("ts", (0.0, 0.0))[0] if scene.flags["flts"] >= 1 else 0.0,
        water_acc_type=water[0]["acc_type"], air_acc_type=air["acc_type"],
        structure=st,
    )
    rain = None
    if scene.flags.get("flr", 0) == 1 and scene.rain is not None:
        # input_par counts the waiting rain particles (CPP_2-initialf.cpp:979-1017)
        rain = dict(scene.rain, nrain=int(np.count_nonzero((t == 7) & (et == 1))))
        if rain["nhor"] == 0:
            rain["nhor"] = 35
    vib = scene.vibration if scene.flags.get("flv", 0) >= 1 else None
    return InitialState(params=params, fields=f, fluid=fl, soil=so, rain=rain, vibration=vib)


def kl_domain(scene: Scene) -> dict:
    """The values the K-L generators take from Cell_Con (input_par,
    CPP_2-initialf.cpp:933-1010; SpatialVariables_Generate_2D/3D,
    CPP_17-1_K-L_expansion_non.cpp:66-90, 160-186): the half extents `a` and
    centre `x_trans` of the non-boundary particles' box widened by 20% per
    side, and soil_max / water_max along y (2-D) or z (3-D).  input_par forms
    those maxima as fmax(running min, x), so they hold the coordinate of the
    last soil / water particle in particle order, not the maximum."""
    nd = scene.ndim
    t = scene.ptype
    nb = (t != 0) & (t != 7)
    lo, hi = np.full(3, 10000.0), np.full(3, -10000.0)
    if nb.any():
        lo = np.minimum(lo, scene.xp[nb].min(axis=0))
        hi = np.maximum(hi, scene.xp[nb].max(axis=0))
    axis = 1 if nd == 2 else 2
    soil = np.flatnonzero(t == 2)
    water = np.flatnonzero(t == 1)
    soil_max = float(scene.xp[soil[-1], axis]) if len(soil) else -100000.0
    water_max = float(scene.xp[water[-1], axis]) if len(water) else -100000.0
    a, xt = np.zeros(3), np.zeros(3)
    for d in range(nd):
        xmin = lo[d] - 0.2 * (hi[d] - lo[d])
        xmax = hi[d] + 0.2 * (hi[d] - lo[d])
        xt[d] = (xmax + xmin) / 2.0
        a[d] = (xmax - xmin) / 2.0
    return {"a": a, "x_trans": xt, "soil_max": soil_max, "water_max": water_max,
            "nb_min": lo, "nb_max": hi}
