"""Generate the golden fixtures of tests/golden/ by running the reference solver.

    python tests/golden/make_golden.py [case ...]     (default: every case)

Needs oracle/_ref/libsphref.so, i.e. the reference solver compiled from its own
sources (make -C oracle ref REF=<reference source tree>).  For each
case the reference parses the input deck written by scenes.write_input_dat,
initialises itself, and runs one thread (its deterministic, sequential order).
Saved per case (.npz): the input deck parameters the reference parsed, the
initial state, the neighbour lists of step 1 (counts, indices, kernel values),
and the state after STEPS steps.  The fixtures let the CPU tests pin the
oracle against the reference where the reference itself is not available.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(REPO, "multiphase-sph-solver_b200"), os.path.join(REPO, "tests")]

import scenes  # noqa: E402
import sphgpu  # noqa: E402
from checkers import STATE_FIELDS, Reference, kl_reference  # noqa: E402

def _kgc_regu():
    """The soil column with the Yang-Liu kernel, kernel gradient correction
    (flknl 4) and strain/stress regularisation every 2 steps."""
    sc = scenes.soil_column_3d(dx=0.1, steps=200)
    sc.flags["flknl"] = 4
    sc.problem["step_regu"] = 2
    return sc


def _slope_art_stress():
    """A 2-D cohesive slope with artificial stress (art_stre_coe 0.5); the upper
    half of the soil starts moving up at 0.5 m/s (scenes.uplift), which puts
    its top in tension so that the tensile branch of the artificial stress
    acts."""
    return scenes.uplift(scenes.slope_2d(H=1.0, dx=0.05, art_stre_coe=0.5), 1, 0.5)


def _column_art_stress():
    """The soil column (cohesion 20 kPa) with artificial stress; soil above
    z = 0.25 starts moving up at 0.5 m/s."""
    sc = scenes.soil_column_3d(dx=0.1, steps=200)
    sc.soils[2]["c"] = 20.0e3
    sc.problem["art_stre_coe"] = 0.5
    return scenes.uplift(sc, 2, 0.25)


def _column_drag(fli, eps0, vw):
    """The soil column with the Tsuji/Shi (fli 2) or Peng (fli 3) soil-water
    drag; void ratio eps0 (5.0 gives porosity 0.83, the dilute branch of
    fli 2), and the pore water starting at x-velocities 0, vw, 2 vw, 3 vw in
    turn so that every Reynolds-number branch is reached."""
    def make():
        sc = scenes.soil_column_3d(dx=0.1, steps=200)
        sc.flags["fli"] = fli
        sc.soils[2]["eps0"] = eps0
        w = np.flatnonzero(sc.ptype == 1)
        sc.vxp[w, 0] = vw * (np.arange(len(w)) % 4)
        return sc
    return make


MCC = dict(ramda=0.2, kapa=0.04, zmf=1.2, eps0=0.9, poi=0.3, sme0=50.0e3, ann=1.0, ocr=1.5, e=0.0, fs=1.0)


def _column_model(matype, **record):
    """The soil column with its soil switched to another constitutive model:
    subloading Cam-clay (1; lambda 0.2, kappa 0.04, M 1.2, e0 0.9, p0 50 kPa,
    E from kappa and p), anisotropic Cam-clay (4), viscous-elastic (7),
    fractional-order Cam-clay (8) or Mohr-Coulomb (9)."""
    return lambda: scenes.set_soil_model(scenes.soil_column_3d(dx=0.1, steps=200), matype, **record)


def _tm_boundary(factory, flbndy=2):
    """A scene with another wall treatment: flbndy 2 (velocity_set_domain +
    tm_boundary_2d / tm_boundary_3d), 3 / 4 (no_slip_tran / free_slip_tran)
    or 13 / 14 (velocity_set_domain + no_slip_tran / free_slip_tran),
    coe_bndy 0.3."""
    def make():
        sc = factory()
        sc.flags["flbndy"] = flbndy
        return sc
    return make


def _free_solid(factory, shift):
    """flbndy 5: boundary_effect_free_struct and boundary_free_solid (friction
    0.3, zeta 0.5).  With `shift` the water starts 0.45 spacings from the left
    wall so that the wall contact acts.  (In 3-D the reference's contact also
    runs over wall particles and yields NaN accelerations on degenerate
    triangles, which reach moving particles in the second step.)"""
    def make():
        sc = factory()
        sc.flags["flbndy"] = 5
        sc.problem["ss"] = (0, 0.3, 0.5, 0)
        if shift:
            w = sc.ptype == 1
            sc.xp[w, 0] -= 0.55 * sc.dr
        return sc
    return make


def _footing(ndim, dx, ss_type, coupled=False):
    """A strip footing (type 4, pushed down at 0.5 m/s, if_move 3) 0.4 spacings
    above a Drucker-Prager soil bed, with soil-structure contact ss_type
    (1 rigid, 2 deformable, 3 penalty), friction 0.3, zeta 0.1; `coupled`
    adds coupled_Water_Soil_Structure (acc_type 2)."""
    def make():
        sc = scenes.footing(ndim=ndim, dx=dx, bed=(1.2, 0.6, 0.5), width=0.4, height=0.2, gap=0.4,
                            ss_type=ss_type, zeta=0.1, v=0.5)
        if coupled:
            sc.problem["ss"] = (ss_type, 0.3, 0.1, 2)
        return sc
    return make


# unsaturated Cam-clay (3): saturation between 0.95 and 1 with the pore
# water below z = 0.15 only, so that the saturation pass leaves the upper
# soil at the residual saturation; beta = 2 keeps pow() of the hardening term
# real when roue turns negative
UMCC = dict(poi=0.3, dens=2650.0, eps0=0.9, zmf=1.2, sme0=50.0e3, fs=1.0, ramda=0.2, kapa=0.04, damp1=0.0,
            damp2=0.0, cop=1.0e-4, ann=1.0, bnn=0.5, beta=2.0, epss=0.9, epsr=0.905, sitas=1.0, sitar=0.95,
            sd=20.0, sw=10.0, kse=0.0, c1=0.05, c2=0.1, c3=0.0, e=0.0, ds=1.0e-3)
# anisotropic Cam-clay (4): its model body is empty in the reference
AMCC = dict(poi=0.3, dens=2650.0, eps0=0.9, zmf=1.2, sme0=50.0e3, fs=1.0, ramda=0.2, kapa=0.04, damp1=0.0,
            damp2=0.0, cop=1.0e-4, mzm=1.0, azm=0.5, r0=0.8, bl=0.95, bz=1.0, zet=0.1, e=1.0e7, ds=1.0e-3)
# fractional-order Cam-clay (8): a sand-like parameter set (G0 125, M 1.25,
# lambda 0.019, e_Gamma 0.934, xi 0.7, alpha 1.2, beta 1, h1 1.8, h2 1.1)
FOCC = dict(dens=2650.0, c=0.75, eps0=0.8, cop=1.0e-4, sme0=50.0e3, g0=125.0, poi=0.25, zmf=1.25, ramda=0.019,
            etao=0.934, zet=0.7, ann=1.2, bnn=1.0, damp1=1.8, damp2=1.1, ds=1.0e-3)


def _column_unsat():
    """The soil column with unsaturated Cam-clay soil and the saturation pass
    (flagum 1); pore water only below z = 0.15."""
    sc = scenes.set_soil_model(scenes.soil_column_3d(dx=0.1, steps=200), 3, **UMCC)
    return scenes.keep(sc, ~((sc.ptype == 1) & (sc.xp[:, 2] > 0.15)))


def _column_tssmp():
    """The Drucker-Prager soil column inside the TSSMP stress transformation
    (flts 1, alpha 0.5, damping coefficient 0.05).  Over more steps, or at
    finer spacing, the reference's TSSMP around Drucker-Prager diverges (NaN
    stresses after about 15 steps at dx = 0.05); around Cam-clay, the pairing
    the transformation is meant for, it stays bounded."""
    sc = scenes.soil_column_3d(dx=0.1, steps=200)
    sc.flags["flts"] = 1
    sc.problem["ts"] = (0.5, 0.05)
    return sc


# pore air (type 3, input block AP): density 1.293, initial pressure 100 Pa,
# sound speed 30 m/s; the reference's air equation of state makes the
# pressure -0.403 paa0 whatever the density (CPP_7-1-eos_CR.cpp:34)
AIR = dict(dens=1.293, paa0=100.0, vis=1.8e-5, vpu=30.0, press_type=0, acc_type=0, pre_coe=0.0)


def _three_phase(acc_type=0, unsat=True):
    """The soil column with three phases (fla 1): pore water below z = 0.15 and
    pore air (type 3) above it, both co-located with the soil; unsaturated
    Cam-clay soil with the saturation pass (saturation 0.95-1, so that the
    soil-air drag of interact1, weighted by (1 - satu)^2, is not zero) or
    Drucker-Prager soil; acc_type 1 selects the minor momentum forms of both
    fluids (fluid_acceleration_minorwater / _minorair)."""
    def make():
        sc = scenes.soil_column_3d(dx=0.1, steps=200)
        if unsat:
            sc = scenes.set_soil_model(sc, 3, **UMCC)
        up = (sc.ptype == 1) & (sc.xp[:, 2] > 0.15)
        sc.ptype[up] = 3
        sc.flags["fla"] = 1
        sc.air = dict(AIR, acc_type=acc_type)
        sc.water[0]["acc_type"] = acc_type
        return sc
    return make


def _dam_break_variant(acc_type=0, bhtype=0, moving=False, dx=0.04):
    """The dam break with the minor water momentum form (acc_type 1), a
    Bingham water (bhtype 1: friction angle 20 deg, yield stress 50 Pa,
    strain_min 1e-3), or a moving right wall (if_move 1: the wall's particles
    get matype 2 and move at -0.2 m/s along x from the first step,
    veocity_update / update, CPP_11-xsph.cpp:61-84, CPP_12-1-update.cpp:38-47)."""
    def make():
        sc = scenes.dam_break_2d(dx=dx, steps=200)
        sc.water[0]["acc_type"] = acc_type
        if bhtype:
            sc.water[0].update(bhtype=1, fai=20.0, c=50.0, strain_min=1.0e-3)
        if moving:
            right = (sc.ptype == 0) & (sc.xp[:, 0] > 1.6)
            sc.matype[right] = 2
            sc.problem["if_move"] = 1
            sc.problem["move_vx"] = (-0.2, 0.0, 0.0)
        return sc
    return make


def _column_moving_wall():
    """The soil column whose far side wall (y > 0.5) moves towards the soil at
    0.1 m/s (if_move 1, matype 2 wall particles)."""
    sc = scenes.soil_column_3d(dx=0.1, steps=200)
    wall = (sc.ptype == 0) & (sc.xp[:, 1] > 0.5)
    sc.matype[wall] = 2
    sc.problem["if_move"] = 1
    sc.problem["move_vx"] = (0.0, -0.1, 0.0)
    return sc


def _geostatic(factory, inip, camclay=False, step_regu=100000000):
    """A geostatic stage of `inip` steps (Para_Pro::inip): elastic stresses
    while l < inip (CPP_7-2-constitutive.cpp:104-115), the damping of
    soil_damping_geostress while l <= inip (CPP_9-4-derivation_stress.cpp:
    850-897), strains reset at l == inip (CPP_7-1-strain.cpp:35-39) and
    displacements restarted by update (CPP_12-1-update.cpp:19-28).  With
    `camclay` the soil is subloading Cam-clay inside the TSSMP transformation
    (flts 1), whose input line also carries the damping coefficient 0.05 that
    gives the damping a nonzero cd."""
    def make():
        sc = factory()
        if camclay:
            sc = scenes.set_soil_model(sc, 1, **MCC)
            sc.flags["flts"] = 1
            sc.problem["ts"] = (0.5, 0.05)
        sc.problem["inip"] = inip
        sc.problem["step_regu"] = step_regu
        return sc
    return make


def _rain(partidel=True):
    """The dam break (dx = 0.04, 40 steps) with three rows of ten rain
    particles above the tank (rainfall type 1, falling at 1 m/s, pressure
    factor 1): lp = 40 / (30 / 10 + 1) = 10, so rows fall at steps 10, 20 and
    30 (rainpro, CPP_15-1-rain.cpp:43-85).  With `partidel` one water particle
    stands alone 0.4 m left of the tank moving left at 9 spacings per step:
    after its first update it lies 7 spacings beyond the domain's left end and
    partidel (CPP_15-2-partidel.cpp:19-58) takes it out; the reference's
    parttocell folds coordinates below the grid's minimum back (the fabs of
    CPP_3-NNPS.cpp:213), so it stays in the grid."""
    def make():
        sc = scenes.dam_break_2d(dx=0.04, steps=40)
        if partidel:
            dt = sc.dt
            sc.xp = np.concatenate([sc.xp, [[-0.5, 0.5, 0.0]]])
            sc.vxp = np.concatenate([sc.vxp, [[-9.0 * sc.dr / dt, 0.0, 0.0]]])
            sc.ptype = np.concatenate([sc.ptype, np.array([1], np.int32)])
            sc.matype = np.concatenate([sc.matype, np.array([0], np.int32)])
            sc.permtype = np.concatenate([sc.permtype, np.array([0], np.int32)])
            sc.etype = np.concatenate([sc.etype, np.array([1], np.int32)])
        return scenes.add_rain(sc, 0.6, 1.0, 3, 0.9)
    return make


CASES = {
    # name: (scene factory, steps)
    "dam_break_2d_dx0.04": (lambda: scenes.dam_break_2d(dx=0.04, steps=200), 25),
    "soil_column_3d_dx0.1": (lambda: scenes.soil_column_3d(dx=0.1, steps=200), 15),
    "soil_column_3d_dx0.1_kgc_regu": (_kgc_regu, 9),
    "slope_2d_H1_dx0.05_art_stress": (_slope_art_stress, 30),
    "soil_column_3d_dx0.1_art_stress": (_column_art_stress, 12),
    "soil_column_3d_dx0.1_drag_tsuji_dilute": (_column_drag(2, 5.0, 1.0), 10),
    "soil_column_3d_dx0.1_drag_peng": (_column_drag(3, 0.6667, 0.05), 10),
    "soil_column_3d_dx0.1_camclay": (_column_model(1, **MCC), 20),
    "soil_column_3d_dx0.1_mohr_coulomb": (_column_model(9, c=0.0, fai=30.0, e=1.0e7), 20),
    "soil_column_3d_dx0.1_visco_elastic": (_column_model(7, c=1.0e5, e=1.0e7), 20),
    "dam_break_2d_dx0.04_tm_boundary": (_tm_boundary(lambda: scenes.dam_break_2d(dx=0.04, steps=200)), 25),
    "soil_column_3d_dx0.1_tm_boundary": (_tm_boundary(lambda: scenes.soil_column_3d(dx=0.1, steps=200)), 15),
    "dam_break_2d_dx0.04_no_slip": (_tm_boundary(lambda: scenes.dam_break_2d(dx=0.04, steps=200), 3), 25),
    "dam_break_2d_dx0.04_free_slip_vsd": (_tm_boundary(lambda: scenes.dam_break_2d(dx=0.04, steps=200), 14), 25),
    "soil_column_3d_dx0.1_free_slip": (_tm_boundary(lambda: scenes.soil_column_3d(dx=0.1, steps=200), 4), 15),
    "soil_column_3d_dx0.1_no_slip_vsd": (_tm_boundary(lambda: scenes.soil_column_3d(dx=0.1, steps=200), 13), 15),
    "dam_break_2d_dx0.04_free_solid": (_free_solid(lambda: scenes.dam_break_2d(dx=0.04, steps=200), True), 15),
    "soil_column_3d_dx0.1_free_solid": (_free_solid(lambda: scenes.soil_column_3d(dx=0.1, steps=200), False), 3),
    "footing_2d_rigid": (_footing(2, 0.04, 1), 12),
    "footing_2d_deformable": (_footing(2, 0.04, 2), 12),
    "footing_2d_penalty": (_footing(2, 0.04, 3), 12),
    "footing_3d_deformable": (_footing(3, 0.1, 2), 12),
    "footing_3d_penalty": (_footing(3, 0.1, 3), 12),
    "footing_2d_penalty_coupled": (_footing(2, 0.04, 3, True), 12),
    "footing_3d_deformable_coupled": (_footing(3, 0.1, 2, True), 12),
    "soil_column_3d_dx0.1_unsat": (_column_unsat, 20),
    "soil_column_3d_dx0.1_amcc": (_column_model(4, **AMCC), 20),
    "soil_column_3d_dx0.1_focc": (_column_model(8, **FOCC), 20),
    "soil_column_3d_dx0.1_tssmp": (_column_tssmp, 20),
    "three_phase_column_3d_dx0.1_unsat": (_three_phase(0, True), 15),
    "three_phase_column_3d_dx0.1_minor": (_three_phase(1, False), 15),
    "dam_break_2d_dx0.04_minor": (_dam_break_variant(acc_type=1), 25),
    "dam_break_2d_dx0.04_bingham": (_dam_break_variant(bhtype=1), 25),
    "dam_break_2d_dx0.04_moving_wall": (_dam_break_variant(moving=True), 25),
    "soil_column_3d_dx0.1_moving_wall": (_column_moving_wall, 15),
    "soil_column_3d_dx0.1_geostatic": (_geostatic(lambda: scenes.soil_column_3d(dx=0.1, steps=200), 6), 12),
    "soil_column_3d_dx0.1_geostatic_camclay": (
        _geostatic(lambda: scenes.soil_column_3d(dx=0.1, steps=200), 6, camclay=True, step_regu=4), 12),
    "slope_2d_H1_dx0.05_geostatic": (_geostatic(lambda: scenes.slope_2d(H=1.0, dx=0.05), 8), 16),
    "dam_break_2d_dx0.04_rain": (_rain(), 35),
    # vibration (flv 1, 2): a shaking base, free-field columns, soil damping
    "shaking_box_2d_flv1": (lambda: scenes.shaking_box(ndim=2, flv=1, dx=0.05), 36),
    "shaking_box_2d_flv2": (lambda: scenes.shaking_box(ndim=2, flv=2, dx=0.05), 36),
    "shaking_box_3d_flv1": (lambda: scenes.shaking_box(ndim=3, flv=1, dx=0.1), 24),
    "shaking_box_3d_flv2": (lambda: scenes.shaking_box(ndim=3, flv=2, dx=0.1), 24),
    # the 3-D rainfall slope, reduced: three phases (soil, pore air, rain
    # falling as water), Darcy drag, rows released every lp = 15 steps
    "rain_slope_3d_dx0.25": (lambda: scenes.rain_slope_3d(dx=0.25, H=2.0, crest=2.0, width=1.5, length=5.0,
                                                          steps=60), 50),
}


# K-L random fields (CPP_17-1_K-L_expansion_non.cpp) through the reference's
# own solve_wi / solve_ramdai / solve_h with injected standard normals:
# name: (scene factory, field, seed of the normals)
KL_CASES = {
    "kl_slope_2d_cohesion_lognormal": (
        lambda: scenes.slope_2d(H=5.0, dx=0.1),
        {"no": 1, "type": 2, "mean": 10.0e3, "sd": 3.0e3, "rl": [10.0, 1.0, 0.0], "coe_depth": 0.0}, 1),
    "kl_slope_2d_friction_normal_depth": (
        lambda: scenes.slope_2d(H=5.0, dx=0.1),
        {"no": 0, "type": 1, "mean": 25.0, "sd": 2.5, "rl": [5.0, 2.0, 0.0], "coe_depth": 0.4}, 2),
    "kl_column_3d_friction_normal_depth": (
        lambda: scenes.soil_column_3d(dx=0.05, steps=100),
        {"no": 0, "type": 1, "mean": 30.0, "sd": 3.0, "rl": [0.5, 0.3, 0.2], "coe_depth": 2.0}, 3),
    "kl_column_3d_fluid_cohesion_lognormal": (
        lambda: scenes.soil_column_3d(dx=0.05, steps=100),
        {"no": 5, "type": 2, "mean": 50.0, "sd": 10.0, "rl": [0.4, 0.4, 0.3], "coe_depth": 0.0}, 4),
}


def _column_no_walls():
    """The soil column's soil and water only (the 3-D generator puts every
    particle into a cell, and the walls reach past the cells)."""
    sc = scenes.soil_column_3d(dx=0.05, steps=100)
    return scenes.keep(sc, sc.ptype != 0)


# correlation-matrix (Cholesky) random fields, nonstationary_random_2D / _3D
# (CPP_17-3-Nonstationary-RF.cpp) through the reference's own routine with
# injected cell normals: name: (scene factory, field, seed of the normals)
RF_CASES = {
    "rf_slope_2d_cohesion_lognormal": (
        lambda: scenes.slope_2d(H=5.0, dx=0.1),
        {"no": 1, "type": 2, "mean": 10.0e3, "sd": 3.0e3, "rl": [10.0, 1.0, 0.0], "cell_ndx": 5.0, "flag_auto": 1},
        11),
    "rf_slope_2d_friction_normal_gauss": (
        lambda: scenes.slope_2d(H=5.0, dx=0.1),
        {"no": 0, "type": 1, "mean": 25.0, "sd": 2.5, "rl": [5.0, 2.0, 0.0], "coe_depth": 0.4, "cell_ndx": 4.0,
         "flag_auto": 2}, 12),
    "rf_slope_2d_cohesion_rotated": (
        lambda: scenes.slope_2d(H=5.0, dx=0.1),
        {"no": 1, "type": 1, "mean": 10.0e3, "sd": 2.0e3, "rl": [6.0, 2.0, 0.0], "cell_ndx": 5.0, "flag_auto": 3,
         "beta": 10.0}, 13),
    "rf_column_3d_friction_rotated": (
        _column_no_walls,
        {"no": 0, "type": 1, "mean": 30.0, "sd": 3.0, "rl": [0.5, 0.3, 0.2], "coe_depth": 2.0, "cell_ndx": 2.0,
         "flag_auto": 3, "beta": 15.0, "beta_1": 30.0}, 14),
    "rf_column_3d_fluid_cohesion_lognormal": (
        _column_no_walls,
        {"no": 5, "type": 2, "mean": 50.0, "sd": 10.0, "rl": [0.4, 0.4, 0.3], "coe_depth": 20.0, "cell_ndx": 2.0,
         "flag_auto": 1}, 15),
}


def make_rf(name: str) -> str:
    from checkers import rf_oracle, rf_reference
    factory, field, seed = RF_CASES[name]
    sc = factory()
    dom = scenes.kl_domain(sc)
    err, _, ncell = rf_oracle(sc.ndim, sc.xp, sc.ptype, sc.dr, field, dom, np.zeros(15000))
    assert err == 0, err
    zeta = np.random.default_rng(seed).standard_normal(ncell)
    err, out = rf_reference(sc.ndim, sc.xp, sc.ptype, sc.dr, field, dom, zeta)
    assert err == 0, err
    spread = _rf_thread_spread(lambda: rf_reference(sc.ndim, sc.xp, sc.ptype, sc.dr, field, dom, zeta)[1], out)
    fn = os.path.join(HERE, name + ".npz")
    np.savez_compressed(fn, ndim=sc.ndim, xp=sc.xp, type=sc.ptype, dr=sc.dr, zeta=zeta, out=out,
                        nb_min=dom["nb_min"], nb_max=dom["nb_max"], soil_max=dom["soil_max"],
                        water_max=dom["water_max"], ref_thread_spread=spread)
    return fn


def _rf_thread_spread(run, out1):
    """The reference's own spread: the largest relative change of the field
    when its OpenMP team has 2 to 8 threads instead of one (its Cholesky
    diagonal is an OpenMP reduction whose order follows the team size,
    CPP_17-3:52-55)."""
    from checkers import reference_lib
    lib = reference_lib()
    ok = np.isfinite(out1)
    scale = np.abs(out1[ok]).max()
    worst = 0.0
    try:
        for t in range(2, 9):
            lib.ref_rf_threads(t)
            o = run()
            worst = max(worst, float(np.abs(o[ok] - out1[ok]).max() / scale))
    finally:
        lib.ref_rf_threads(1)
    return np.array(worst)


# the correlated forms of CPP_17-5-Nonstationary-Correlated-RF.cpp, through the
# reference's own routines with injected normals:
# name: (scene factory, (friction field, cohesion field), coe_frict_cohesion, seed)
_FAI_SOIL = {"no": 0, "type": 2, "mean": 25.0, "sd": 5.0, "rl": [8.0, 1.5, 0.0], "coe_depth": 0.5, "cell_ndx": 5.0,
             "flag_auto": 1}
_C_SOIL = {"no": 1, "type": 2, "mean": 10.0e3, "sd": 3.0e3, "rl": [1.0, 1.0, 0.0], "coe_depth": 200.0}
RF_CORR_CASES = {
    "rfc_slope_2d_soil_lognormal": (lambda: scenes.slope_2d(H=5.0, dx=0.1), (_FAI_SOIL, _C_SOIL), -0.5, 21),
    "rfc_slope_2d_soil_normal_gauss": (
        lambda: scenes.slope_2d(H=5.0, dx=0.1),
        (dict(_FAI_SOIL, type=1, flag_auto=2, rl=[5.0, 2.0, 0.0], cell_ndx=4.0), dict(_C_SOIL, type=1)), -0.3, 22),
    "rfc_column_3d_fluid_normal_rotated": (
        _column_no_walls,
        ({"no": 4, "type": 1, "mean": 5.0, "sd": 1.0, "rl": [0.5, 0.3, 0.2], "coe_depth": 2.0, "cell_ndx": 2.0,
          "flag_auto": 3, "beta": 15.0, "beta_1": 30.0},
         {"no": 5, "type": 1, "mean": 50.0, "sd": 10.0, "rl": [9.0, 9.0, 9.0], "coe_depth": 20.0}), 0.4, 23),
    "rfc_column_3d_soil_lognormal": (
        _column_no_walls,
        (dict(_FAI_SOIL, rl=[0.4, 0.4, 0.3], cell_ndx=2.0), _C_SOIL), -0.6, 24),
}
# random_variable_generate (flspv 5): name: (scene factory, pair, coe, seed)
RV_CASES = {
    "rv_slope_2d_soil_lognormal": (lambda: scenes.slope_2d(H=5.0, dx=0.1), (_FAI_SOIL, _C_SOIL), -0.5, 31),
    "rv_column_3d_fluid_normal": (_column_no_walls, (dict(_FAI_SOIL, no=4, type=1), dict(_C_SOIL, no=5)), 0.3, 32),
}


def make_rf_corr(name: str) -> str:
    from checkers import rf_oracle_corr, rf_reference_corr
    factory, pair, coe, seed = RF_CORR_CASES[name]
    sc = factory()
    dom = scenes.kl_domain(sc)
    err, _, ncell = rf_oracle_corr(sc.ndim, sc.xp, sc.ptype, sc.dr, pair, coe, dom, np.zeros((15000, 2)))
    assert err == 0, err
    u2 = np.random.default_rng(seed).standard_normal((ncell, 2))
    err, out = rf_reference_corr(sc.ndim, sc.xp, sc.ptype, sc.dr, pair, coe, dom, u2)
    assert err == 0, err
    spread = _rf_thread_spread(lambda: rf_reference_corr(sc.ndim, sc.xp, sc.ptype, sc.dr, pair, coe, dom, u2)[1],
                               out)
    fn = os.path.join(HERE, name + ".npz")
    np.savez_compressed(fn, ndim=sc.ndim, xp=sc.xp, type=sc.ptype, dr=sc.dr, u2=u2, out=out,
                        nb_min=dom["nb_min"], nb_max=dom["nb_max"], soil_max=dom["soil_max"],
                        water_max=dom["water_max"], ref_thread_spread=spread)
    return fn


def make_rv(name: str) -> str:
    from checkers import rv_reference
    factory, pair, coe, seed = RV_CASES[name]
    sc = factory()
    u2 = np.random.default_rng(seed).standard_normal(2)
    out = rv_reference(sc.ptype, pair, coe, u2)
    fn = os.path.join(HERE, name + ".npz")
    np.savez_compressed(fn, type=sc.ptype, u2=u2, out=out)
    return fn


def make_kl(name: str) -> str:
    factory, field, seed = KL_CASES[name]
    sc = factory()
    dom = scenes.kl_domain(sc)
    xi = np.random.default_rng(seed).standard_normal(200)
    out, wi, eig, order = kl_reference(sc.ndim, sc.xp, sc.ptype, field, dom, xi)
    fn = os.path.join(HERE, name + ".npz")
    np.savez_compressed(fn, ndim=sc.ndim, xp=sc.xp, type=sc.ptype, xi=xi,
                        field=np.array([field["no"], field["type"]]),
                        field_vals=np.array([field["mean"], field["sd"], field["coe_depth"]] + list(field["rl"])),
                        a=dom["a"], x_trans=dom["x_trans"], soil_max=dom["soil_max"], water_max=dom["water_max"],
                        out=out, wi=wi[:, :sc.ndim], eigval=eig, order=order[:, :sc.ndim])
    return fn


def make(name: str) -> str:
    if name in KL_CASES:
        return make_kl(name)
    if name in RF_CASES:
        return make_rf(name)
    if name in RF_CORR_CASES:
        return make_rf_corr(name)
    if name in RV_CASES:
        return make_rv(name)
    factory, steps = CASES[name]
    sc = factory()
    out = {}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "input.dat")
        scenes.write_input_dat(sc, path)
        ref = Reference(path, 1)
        out["params"] = np.frombuffer(bytes(ref.params), dtype=np.uint8)
        if sc.flags.get("flv", 0) >= 1:
            vb = sc.vibration
            out["vib_par"] = np.array([vb["ttime"], vb["nsteps"], vb["sttime"], vb["edtime"]])
            out["vib_loads"] = np.asarray(vb["loads"], dtype=np.float64)
        if sc.flags.get("flr", 0) == 1:
            rn = ref.rain()
            out["rain"] = np.array([rn["rtype"], rn["nrain"], rn["nhor"], rn["press_factor"], rn["drop_velocity"]])
        fl, so = ref.materials()
        out["fluid"], out["soil"] = fl, so
        for k in STATE_FIELDS:
            out["init_" + k] = ref.get_field(k)
        err, ninflu, influ, wij = ref.nnps(with_wij=True)
        assert err == 0
        out["nnps_ninflu"] = ninflu
        mask = np.arange(100)[None, :] <= ninflu[:, None]
        out["nnps_influ"] = np.where(mask, influ, 0)
        out["nnps_wij"] = np.where(mask[:, :, None], wij, 0.0)
        assert ref.step(steps) == 0
        out["steps"] = np.array(steps)
        if sc.flags.get("flr", 0) == 1:
            out["final_nrain"] = np.array(ref.rain()["nrain"])
        for k in STATE_FIELDS:
            out["final_" + k] = ref.get_field(k)
    fn = os.path.join(HERE, name + ".npz")
    np.savez_compressed(fn, **out)
    return fn


if __name__ == "__main__":
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    os.dup2(devnull, 1)   # the reference prints progress lines
    try:
        files = [make(n) for n in (sys.argv[1:] or list(CASES) + list(KL_CASES) + list(RF_CASES) +
                                         list(RF_CORR_CASES) + list(RV_CASES))]
    finally:
        os.dup2(saved, 1)
    for f in files:
        print(f, os.path.getsize(f))
