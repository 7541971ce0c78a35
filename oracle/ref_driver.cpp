/*
 * ref_driver.cpp -- drives the UNMODIFIED reference solver
 * (wodexinxin2015/MultiPhase-SPH-Solver) through its own public classes, for
 * pinning the oracle restatement and for the CPU baseline.
 * TEST INFRASTRUCTURE ONLY.
 *
 * Built by oracle/Makefile against the reference's own sources (all .cpp
 * files except CPP_0-main.cpp), with output only into oracle/_ref/.  The
 * initialisation sequence and the step body below call the reference's
 * methods in the order SPH_Calculation does (CPP_1-SPHLoops.cpp:238-450 and
 * :523-753); nothing of the reference is re-implemented here.
 */
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>

// The K-L generator's steps (solve_wi, solve_ramdai, solve_h_2D/3D) are
// private members of clFSpatialVariability_Fun; this harness calls them
// directly so that the standard-normal coefficients can be injected in place
// of the generator's time-seeded draw.  The class has no data members, so
// widening access in this translation unit changes nothing else.
#define private public
#include "Class_Functions.h"
#undef private

#include "../include/sphgpu.h"

namespace {

struct RefRun {
    Para_FL fl;
    Para_Pro pro;
    Para_Rain rain;
    Para_Inter inter;
    Para_Boundary bou;
    Para_Vibra vib;
    Para_Soil ffbound;                 // SPH_Calculation's pFFBound: never read from the deck
    clFreeFieldBndy_Fun ffb;
    clFreeFieldBndy_Fun_soil ffs;
    Para_GF gf;
    Para_EC ec;
    Para_SSInter ssi;
    Flag_SpatialVariability fsv;
    Para_Model matter;
    Para_Soil soil[30];
    Para_Fluid water[3];
    Para_Fluid air;
    Para_Structure structure;
    Para_SpatialVariability psv[6];
    Cell_Con cellc;
    double thr_min = 0.1, thr_max = 0.12;
    int k = 0, size_m = 0;

    Particle* par = nullptr;
    Par_Cell* parcell = nullptr;
    StiffMat* stiff = nullptr;
    clRaij* rij = nullptr;
    clInterf_SS** interf_ss = nullptr;
    clPair_SS* pair_ss = nullptr;
    clParti_Pair* partipair = nullptr;
    Para_Fluid* vfluid = nullptr;
    Para_Soil* conspara = nullptr;
    cl_bndy_pair* bndy = nullptr;
    clVar_Boundary* varibndy = nullptr;
    parti_cellid* sorted = nullptr;
    parti_cellid* temp = nullptr;
    double (*vx_temp)[3] = nullptr;
    cell_info* cinfo = nullptr;
    cell_link* clink = nullptr;
    FILE* flog = nullptr;

    clFIni_Fun ini;
    clNNPS_Fun nnps;
    clDensity_Fun dens;
    clStraStre_Fun sts;
    clInterFor_Fun itf;
    clAcce_Fun acc;
    clVel_Fun vel;
    clUpdate_Fun upd;
    clBndy_Fun bnd;
    clSoilStruct_Fun ssinter;
    clRain_Fun rainf;
    int lp = 0;
    double vrain = 0.0, cement_base[3] = {0.0, 0.0, 0.0};
};

int g_last_error = 0;

}  // namespace

extern "C" {

void* ref_create(const char* input_dat_path, int nthreads)
{
    g_last_error = 0;
    FILE* finp = fopen(input_dat_path, "r");
    if (!finp) { g_last_error = 1; return nullptr; }
    RefRun* r = new RefRun();
    r->flog = fopen("/dev/null", "w");
    int err = r->ini.initial_pro(&r->fl, &r->pro, &r->rain, &r->inter, &r->ssi, &r->bou, &r->vib, &r->gf,
                                 &r->ec, &r->thr_min, &r->thr_max, r->flog, finp);
    if (err > 0) { g_last_error = err; fclose(finp); delete r; return nullptr; }
    if (r->pro.dttype == 2) r->upd.timestep(&r->pro);
    if (nthreads > 0) r->fl.ntd = nthreads;
    omp_set_num_threads(r->fl.ntd);
    int n = r->pro.ntotal;
    r->k = (int)log2(n) + 1;
    r->size_m = 1 << r->k;
    r->par = new Particle[n];
    r->rij = new clRaij[n];
    r->parcell = new Par_Cell[n];
    r->stiff = new StiffMat[n];
    r->interf_ss = new clInterf_SS*[n];
    for (int i = 0; i < n; i++) r->interf_ss[i] = new clInterf_SS[r->fl.ntd];
    r->pair_ss = new clPair_SS[n];
    r->partipair = new clParti_Pair[n];
    r->vfluid = new Para_Fluid[n];
    r->conspara = new Para_Soil[n];
    r->bndy = new cl_bndy_pair[n];
    r->varibndy = new clVar_Boundary[n];
    r->sorted = new parti_cellid[r->size_m];
    r->temp = new parti_cellid[r->size_m];
    r->vx_temp = new double[n][3];
    err = r->ini.initial_mat(&r->matter, r->soil, r->water, &r->air, &r->structure, r->fl, &r->fsv, r->psv, r->flog, finp);
    if (err > 0) { g_last_error = err; fclose(finp); return nullptr; }
    r->ini.input_par(r->par, &r->pro, &r->cellc, &r->rain, r->flog, finp);
    fclose(finp);
    // vibra.dat beside the deck, as SPH_Calculation opens it (CPP_1-SPHLoops.cpp:306-340)
    if (r->fl.flv >= 1) {
        std::string dir(input_dat_path);
        const size_t slash = dir.find_last_of('/');
        dir = (slash == std::string::npos) ? std::string(".") : dir.substr(0, slash);
        FILE* fvib = fopen((dir + "/vibra.dat").c_str(), "r");
        if (!fvib) { g_last_error = 1; delete r; return nullptr; }
        err = r->ini.initial_vib(&r->vib, r->flog, fvib);
        fclose(fvib);
        if (err > 0) { g_last_error = err; delete r; return nullptr; }
    }
    r->ini.setting_vis_cons(r->par, r->pro, r->vfluid, r->water, r->air, r->conspara, r->soil, r->structure);
    r->ini.setting_par(r->par, &r->pro, r->vfluid, r->conspara, r->soil, r->gf, r->structure, r->water, &r->rain, r->flog);
    r->nnps.celllist_ini1(&r->cellc, r->pro);
    r->cinfo = new cell_info[r->cellc.ctotal + 4];
    r->clink = new cell_link[r->cellc.ctotal + 4];
    r->nnps.celllist_ini2(r->clink, r->cellc, r->pro.ndim, r->fl.ntd);
    // rainfall set-up as SPH_Calculation does it (CPP_1-SPHLoops.cpp:457-467)
    if (r->fl.flr == 1 && r->rain.rtype <= 7 && r->rain.rtype >= 1) {
        r->rainf.rainini(r->rain, r->pro, &r->lp, &r->vrain);
        r->rainf.center_cement(r->par, r->pro, r->cement_base);
    }
    return r;
}

int ref_get_rain(void* h, sphgpu_rain* o)
{
    RefRun* r = (RefRun*)h;
    o->rtype = r->rain.rtype;
    o->nrain = r->rain.nrain;
    o->nhor = r->rain.nhor;
    o->press_factor = r->rain.press_factor;
    o->drop_velocity = r->rain.drop_velocity;
    return 0;
}

int ref_last_error(void) { return g_last_error; }

void ref_set_threads(void* h, int nthreads)
{
    RefRun* r = (RefRun*)h;
    r->fl.ntd = nthreads;
    omp_set_num_threads(nthreads);
}

int ref_get_params(void* h, sphgpu_params* o)
{
    RefRun* r = (RefRun*)h;
    memset(o, 0, sizeof(*o));
    o->ndim = r->pro.ndim;
    o->ntotal = r->pro.ntotal;
    o->fla = r->fl.fla; o->fls = r->fl.fls; o->flr = r->fl.flr; o->fli = r->fl.fli; o->flv = r->fl.flv;
    o->fleob = r->fl.fleob; o->flts = r->fl.flts; o->flspv = r->fl.flspv; o->flknl = r->fl.flknl;
    o->flbndy = r->fl.flbndy;
    o->inip = r->pro.inip; o->step_regu = r->pro.step_regu; o->loop = r->pro.loop; o->fop = r->pro.fop;
    o->dr = r->pro.dr; o->dt = r->pro.dt;
    for (int a = 0; a < 3; a++) o->xsph[a] = r->pro.xsph[a];
    for (int a = 0; a < 3; a++) for (int b = 0; b < 2; b++) o->art_vis[a][b] = r->pro.art_vis[a][b];
    o->art_stre_coe = r->pro.art_stre_coe;
    o->gx = r->gf.gx; o->gy = r->gf.gy; o->gz = r->gf.gz;
    o->threshold_min = r->thr_min; o->threshold_max = r->thr_max;
    o->interc = r->inter.interc; o->permtype = r->inter.permtype;
    o->pers = r->inter.pers; o->perl = r->inter.perl; o->perm = r->inter.perm;
    o->ss_type = r->ssi.type; o->ss_myu = r->ssi.myu; o->ss_zeta = r->ssi.zeta; o->ss_acc_type = r->ssi.acc_type;
    o->coe_bndy = r->bou.coe_bndy; o->if_cal = r->bou.if_cal; o->if_move = r->bou.if_move;
    for (int a = 0; a < 3; a++) o->move_vx[a] = r->bou.move_vx[a];
    o->xmin = r->cellc.xmin; o->xmax = r->cellc.xmax;
    o->ymin = r->cellc.ymin; o->ymax = r->cellc.ymax;
    o->zmin = r->cellc.zmin; o->zmax = r->cellc.zmax;
    o->cxm = r->cellc.cxm; o->cym = r->cellc.cym; o->czm = r->cellc.czm; o->ctotal = r->cellc.ctotal;
    o->flagum = r->matter.flagum; o->alphats = r->matter.alphats;
    o->water_acc_type = r->water[0].acc_type;
    o->air_acc_type = r->air.acc_type;
    o->structure.dens = r->structure.dens; o->structure.eps0 = r->structure.eps0;
    o->structure.e = r->structure.e; o->structure.poi = r->structure.poi;
    o->structure.vpu = r->structure.vpu; o->structure.porosity = r->structure.porosity;
    o->structure.cop = r->structure.cop;
    return 0;
}

int ref_get_materials(void* h, sphgpu_fluid* fl, sphgpu_soil* so)
{
    RefRun* r = (RefRun*)h;
    for (int i = 0; i < r->pro.ntotal; i++) {
        const Para_Fluid& f = r->vfluid[i];
        sphgpu_fluid o = {f.vis, f.vpu, f.dens, f.paa0, f.porosity, f.fai, f.c,
                          f.bhtype, f.press_type, f.acc_type, f.pre_coe, f.strain_min};
        if (fl) fl[i] = o;
        const Para_Soil& s = r->conspara[i];
        sphgpu_soil q = {s.e, s.poi, s.eps0, s.dens, s.damp1, s.damp2, s.cop, s.ramda, s.kapa, s.zmf,
                         s.ann, s.bnn, s.beta, s.sitas, s.sitar, s.epsr, s.epss, s.sd, s.sw, s.kse,
                         s.c1, s.c2, s.c3, s.fai, s.c, s.ocr, s.sme0, s.mzm, s.azm, s.r0,
                         s.bl, s.bz, s.zet, s.vpu, s.porosity, s.fs, s.etao, s.g0, s.ds, s.damp_coe};
        if (so) so[i] = q;
    }
    return 0;
}

/* copy one Particle member out for all particles (particle-major) */
int ref_get_field(void* h, const char* name, void* out)
{
    RefRun* r = (RefRun*)h;
    int n = r->pro.ntotal;
#define DV(member, nc)                                                                  \
    if (strcmp(name, #member) == 0) {                                                   \
        double* o = (double*)out;                                                       \
        for (int i = 0; i < n; i++) memcpy(o + (size_t)i * nc, &r->par[i].member, 8 * nc); \
        return 0;                                                                       \
    }
#define IV(member)                                                                      \
    if (strcmp(name, #member) == 0) {                                                   \
        int* o = (int*)out;                                                             \
        for (int i = 0; i < n; i++) o[i] = r->par[i].member;                            \
        return 0;                                                                       \
    }
    DV(x, 3) DV(xp, 3) DV(vx, 3) DV(vxp, 3) DV(ax, 3) DV(axp, 3) DV(ux, 3) DV(strep, 3)
    DV(divx, 9) DV(interf, 3) DV(interfss, 3) DV(rho, 1) DV(rhop, 1) DV(mass, 1) DV(hl, 1)
    DV(pre, 1) DV(prep, 1) DV(e, 1) DV(eps, 6) DV(deps, 6) DV(sig, 6) DV(dsig, 6) DV(weps, 9)
    DV(adps, 6) DV(tssig, 6) DV(tsqc, 1) DV(satu, 1) DV(dsatu, 1) DV(suct, 1) DV(cop, 1) DV(vsig, 1) DV(veps, 1)
    DV(divq, 1) DV(divr, 1) DV(meps, 1) DV(prew, 1) DV(prea, 1) DV(porosity, 1) DV(cd, 1)
    DV(poro_cop, 1) DV(beta, 9) DV(beta_ts, 9)
    IV(type) IV(matype) IV(permtype) IV(etype)
#undef DV
#undef IV
    return SPHGPU_E_ARG;
}

/* raw Particle records, for the layout test of the engine's AoS upload */
const void* ref_particles(void* h) { return ((RefRun*)h)->par; }
size_t ref_particle_size(void) { return sizeof(Particle); }

int ref_nnps(void* h, int* ninflu, int* influ, double* wij)
{
    RefRun* r = (RefRun*)h;
    int err = r->nnps.parttocell(r->parcell, r->cinfo, r->cellc, r->sorted, r->temp, r->pro, r->par,
                                 r->pro.ndim, r->fl.ntd, r->size_m, r->k);
    if (err > 0) return err;
    err = r->nnps.partisearching(r->parcell, r->cinfo, r->clink, r->sorted, r->cellc, r->pro, r->par,
                                 r->fl.ntd, r->fl.flknl);
    for (int i = 0; i < r->pro.ntotal; i++) {
        if (ninflu) ninflu[i] = r->parcell[i].ninflu;
        if (influ) memcpy(influ + (size_t)i * 100, r->parcell[i].influ, sizeof(int) * 100);
        if (wij) memcpy(wij + (size_t)i * 400, r->parcell[i].wij, sizeof(double) * 400);
    }
    return err;
}

/* the body of the main loop, CPP_1-SPHLoops.cpp:481-760, for the flag set the
 * engine covers (rain, no excavation or vibration) */
int ref_step(void* h, int nsteps)
{
    RefRun* r = (RefRun*)h;
    Para_Pro& P = r->pro;
    Para_FL& F = r->fl;
    for (int s = 0; s < nsteps; s++) {
        if (!(P.t < P.tt)) return 0;
        P.t = P.t + P.dt;
        // rainfall (CPP_1-SPHLoops.cpp:497-513)
        if (F.flr == 1 && (P.l - P.inip) > 0 && (P.l - P.inip) % r->lp == 0) {
            if (r->rain.rtype == 1) r->rainf.rainpro(r->par, &r->rain, &P, r->vfluid, r->gf, r->vrain);
            else if (r->rain.rtype == 2) r->rainf.waterdel_min(r->par, &r->rain, &P);
            else if (r->rain.rtype == 3) r->rainf.waterdel_max(r->par, &r->rain, &P);
            else if (r->rain.rtype == 4)
                r->rainf.cementpro(r->par, &r->rain, &P, r->vfluid, r->gf, r->vrain, r->cement_base);
        }
        int err = r->nnps.parttocell(r->parcell, r->cinfo, r->cellc, r->sorted, r->temp, P, r->par, P.ndim,
                                     F.ntd, r->size_m, r->k);
        if (err > 0) return err;
        err = r->nnps.partisearching(r->parcell, r->cinfo, r->clink, r->sorted, r->cellc, P, r->par, F.ntd, F.flknl);
        if (err > 0) return err;
        if (F.flknl > 2) r->nnps.kernel_gradient_correction(r->par, r->parcell, P);
        r->dens.density(r->par, r->parcell, r->vfluid, r->bndy, r->varibndy, P, F.flbndy);
        r->sts.strain_noreg(r->par, r->parcell, r->bndy, r->varibndy, P, F.flbndy);
        if (P.l % P.step_regu == 0) r->sts.strain_regu(r->par, r->parcell, P);
        if (r->matter.flagum == 1) r->itf.saturation(r->par, r->parcell, r->conspara, P, F.ntd);
        if (F.fli == 1) r->itf.cal_permeability(r->par, r->inter, r->conspara, P, F.ntd);
        r->sts.eos(r->par, r->parcell, r->vfluid, P, F.ntd);
        r->sts.strain_to_stress(r->par, r->conspara, r->stiff, r->vfluid, r->structure, P, F.ntd, F.flts, r->matter.alphats);
        if (P.l % P.step_regu == 0) r->sts.stress_regu(r->par, r->parcell, P);
        r->sts.free_surface_check(r->par, r->parcell, P, r->thr_max, r->thr_min);
        r->sts.Stress_eigValue(r->par, P, F.ntd);
        if (r->water[0].acc_type == 0) r->acc.fluid_acceleration_water(r->par, r->parcell, r->vfluid, P, r->gf, F.ntd);
        else r->acc.fluid_acceleration_minorwater(r->par, r->parcell, r->vfluid, P, r->gf, F.ntd);
        if (r->air.acc_type == 0) r->acc.fluid_acceleration_air(r->par, r->parcell, r->vfluid, P, r->gf, F.ntd);
        else r->acc.fluid_acceleration_minorair(r->par, r->parcell, r->vfluid, P, r->gf, F.ntd);
        r->acc.soil_acceleration_noreg(r->par, r->parcell, r->conspara, P, r->gf, F.ntd);
        r->acc.structure_acceleration_noreg(r->par, r->parcell, P, r->gf, F.ntd);
        r->acc.artificial_viscosity(r->par, r->parcell, r->conspara, r->vfluid, P, F.ntd);
        if (P.ndim == 2 && P.art_stre_coe > 0.0) r->acc.artificial_stress_2d(r->par, r->parcell, P, r->rij, F.ntd);
        else if (P.ndim == 3 && P.art_stre_coe > 0.0) r->acc.artificial_stress_3d(r->par, r->parcell, P, r->rij, F.ntd);
        if (F.flbndy == 1 || F.flbndy == 2) r->acc.boundary_moving_stress_effect(r->par, r->parcell, P, F.ntd);
        else if (F.flbndy == 3 || F.flbndy == 4 || F.flbndy == 13 || F.flbndy == 14)
            r->acc.boundary_stress_effect_tran(r->par, r->parcell, r->varibndy, P, F.ntd);
        else r->acc.boundary_effect_free_struct(r->par, r->parcell, P, F.ntd);
        if (F.flv != 0) {
            // free-field boundaries (CPP_1-SPHLoops.cpp:621-635) with
            // SPH_Calculation's default-constructed pFFBound (:253)
            r->ffb.free_field_solid(r->par, r->bndy, r->ffbound, r->parcell, P, F.ntd);
            r->ffs.free_field_solid(r->par, r->conspara, r->parcell, P, F.ntd);
        }
        if (r->ssi.type >= 1 && r->ssi.type <= 3 && r->ssi.acc_type == 2)
            r->acc.coupled_Water_Soil_Structure(r->par, r->parcell, r->vfluid, r->conspara, P, r->gf, F.ntd);
        if (F.flv == 1) r->acc.vibration_acceleration(r->par, r->vib, P, F.ntd);
        if (F.fli == 1) r->itf.interact1(r->par, r->parcell, r->inter, r->vfluid, P, r->gf, F.ntd);
        else if (F.fli == 2) r->itf.interact2(r->par, r->parcell, r->inter, r->conspara, r->vfluid, P, r->gf, F.ntd);
        else if (F.fli == 3) r->itf.interact3(r->par, r->parcell, r->inter, r->conspara, r->vfluid, P, r->gf, F.ntd);
        if (r->ssi.type == 1)
            err = r->ssinter.interaction_ss_rigid(r->par, r->parcell, r->pair_ss, r->interf_ss, r->partipair, r->ssi, P, F.ntd);
        else if (r->ssi.type == 2)
            err = r->ssinter.interaction_ss_deformable(r->par, r->parcell, r->pair_ss, r->interf_ss, r->partipair, r->ssi, P,
                                                       F.ntd);
        else if (r->ssi.type == 3)
            err = r->ssinter.interaction_ss_penalty(r->par, r->parcell, r->pair_ss, r->interf_ss, r->partipair, r->ssi, P, F.ntd);
        if (err > 0) return err;
        if (P.l <= P.inip) r->acc.soil_damping_geostress(r->par, r->parcell, P, F.ntd);
        if (F.flv > 0) r->acc.soil_damping_vibration(r->par, r->parcell, r->conspara, r->stiff, P);
        if (F.flbndy == 5) r->bnd.boundary_free_solid(r->par, r->parcell, P, r->ssi, F.ntd);
        r->vel.veocity_update(r->par, P, r->bou, F.flv);
        if (F.flv == 2) r->acc.vibration_velocity(r->par, r->vib, P, F.ntd);
        if (r->bou.if_move != 2) r->vel.xsph(r->par, r->parcell, r->bndy, r->varibndy, P, r->vx_temp, F.flbndy);
        if (F.flbndy == 1) r->bnd.tmboundary(r->par, r->parcell, r->bndy, P);
        else if (F.flbndy == 2) {
            r->bnd.velocity_set_domain(r->par, r->parcell, r->bndy, P, r->bou.coe_bndy);
            if (P.ndim == 2) r->bnd.tm_boundary_2d(r->par, r->parcell, r->bndy, r->varibndy, P, F.ntd);
            else r->bnd.tm_boundary_3d(r->par, r->parcell, r->bndy, r->varibndy, P, F.ntd);
        } else if (F.flbndy == 3) r->bnd.no_slip_tran(r->par, r->parcell, r->varibndy, P, F.ntd);
        else if (F.flbndy == 4) r->bnd.free_slip_tran(r->par, r->parcell, r->varibndy, P, F.ntd);
        else if (F.flbndy == 13) {
            r->bnd.velocity_set_domain(r->par, r->parcell, r->bndy, P, r->bou.coe_bndy);
            r->bnd.no_slip_tran(r->par, r->parcell, r->varibndy, P, F.ntd);
        } else if (F.flbndy == 14) {
            r->bnd.velocity_set_domain(r->par, r->parcell, r->bndy, P, r->bou.coe_bndy);
            r->bnd.free_slip_tran(r->par, r->parcell, r->varibndy, P, F.ntd);
        }
        r->bnd.check_domain(r->par, r->cellc, r->bou, P);
        r->upd.update(r->par, P, r->bou, F.ntd);
        if (F.flr == 1) r->rainf.partidel(r->par, &r->rain, &P, r->cellc, F.ntd);
        P.l++;
    }
    return 0;
}

int ref_get_step(void* h) { return ((RefRun*)h)->pro.l; }

void ref_destroy(void* h)
{
    RefRun* r = (RefRun*)h;
    if (!r) return;
    if (r->flog) fclose(r->flog);
    for (int i = 0; i < r->pro.ntotal; i++) delete[] r->interf_ss[i];
    delete[] r->interf_ss;
    delete[] r->par; delete[] r->rij; delete[] r->parcell; delete[] r->stiff;
    delete[] r->pair_ss; delete[] r->partipair; delete[] r->vfluid; delete[] r->conspara;
    delete[] r->bndy; delete[] r->varibndy; delete[] r->sorted; delete[] r->temp;
    delete[] r->vx_temp; delete[] r->cinfo; delete[] r->clink;
    delete r;
}

}  // extern "C"

/*
 * The reference's K-L random field (CPP_17-1_K-L_expansion_non.cpp) for one
 * field with injected standard-normal coefficients uu[klterm]: solve_wi,
 * solve_ramdai and solve_h_2D / solve_h_3D as SpatialVariables_Generate_2D /
 * _3D call them (CPP_17-1:138-157, 250-269).  n particles with positions xp
 * (n x 3) and types; a[3], x_trans[3], soil_max, water_max as the generator
 * derives them.  Returns the reference's code; out[i] receives the member the
 * field writes (NaN where it writes none), wi (200 x 3), eigval (200) and
 * order (200 x 3) the intermediate results.
 */
extern "C" int ref_kl_field(int ndim, int n, const double* xp, const int* type, int no, int dist_type,
                            double mean_value, double sd_value, double coe_depth, const double* rl,
                            const double* a, const double* x_trans, double soil_max, double water_max,
                            const double* uu, double* out, double* wi_out, double* eigval_out, int* order_out)
{
    const int K = 200;
    Particle* par = new Particle[n];
    Para_Fluid* fl = new Para_Fluid[n];
    Para_Soil* so = new Para_Soil[n];
    const double nan = 0.0 / 0.0;
    for (int i = 0; i < n; i++) {
        for (int d = 0; d < 3; d++) par[i].xp[d] = xp[(size_t)i * 3 + d];
        par[i].type = type[i];
        fl[i].fai = fl[i].c = nan;
        so[i].fai = so[i].c = so[i].cop = so[i].ds = nan;
    }
    Para_Pro pro;
    pro.ndim = ndim;
    pro.ntotal = n;
    Para_SpatialVariability psv;
    psv.no = no;
    psv.type = dist_type;
    psv.mean_value = mean_value;
    psv.sd_value = sd_value;
    psv.coe_depth = coe_depth;
    for (int d = 0; d < 3; d++) { psv.rl_value[d] = rl[d]; psv.a[d] = a[d]; }
    double wi[200][3], eigval[200], xt[3] = {x_trans[0], x_trans[1], x_trans[2]};
    int order_id[200][3];
    double u[200];
    for (int j = 0; j < K; j++) u[j] = uu[j];
    clFSpatialVariability_Fun f;
    f.solve_wi(wi, psv.a, psv.rl_value, ndim);
    int err = f.solve_ramdai(eigval, wi, psv.rl_value, order_id, ndim);
    if (!err) {
        if (ndim == 2)
            err = f.solve_h_2D(par, fl, so, pro, wi, eigval, u, xt, order_id, psv, soil_max, water_max, no);
        else
            err = f.solve_h_3D(par, fl, so, pro, wi, eigval, u, xt, order_id, psv, soil_max, water_max, no);
    }
    for (int i = 0; i < n; i++) {
        double v = nan;
        switch (no) {
        case 0: v = so[i].fai; break;
        case 1: v = so[i].c; break;
        case 2: v = so[i].cop; break;
        case 3: v = so[i].ds; break;
        case 4: v = fl[i].fai; break;
        case 5: v = fl[i].c; break;
        }
        out[i] = v;
    }
    for (int j = 0; j < K; j++) {
        eigval_out[j] = eigval[j];
        for (int d = 0; d < 3; d++) { wi_out[j * 3 + d] = wi[j][d]; order_out[j * 3 + d] = order_id[j][d]; }
    }
    delete[] par;
    delete[] fl;
    delete[] so;
    return err;
}

/*
 * The reference's correlation-matrix random fields (nonstationary_random_2D /
 * _3D, CPP_17-3-Nonstationary-RF.cpp:76-849; nonstationary_correlated_random_
 * 2D / _3D and random_variable_generate, CPP_17-5-Nonstationary-Correlated-
 * RF.cpp:87-863) with the normals injected: both translation units are
 * compiled without inlining for this library (oracle/Makefile), so their
 * calls of the time-seeded generate_SND (CPP_17-3:32-43, which fills n
 * values; CPP_17-5:35-46, which fills n pairs) reach the definition below,
 * which hands out zeta (g_zeta_per values per requested unit).
 */
namespace {
const double* g_zeta = nullptr;
int g_zeta_n = 0;
int g_zeta_per = 1;
int g_rf_threads = 1;
}  // namespace

/* The OpenMP team the random-field routines run with (1 by default: their
 * Cholesky diagonal is an OpenMP reduction whose order follows the team size,
 * CPP_17-3:52-55, so only one thread makes the result reproducible). */
extern "C" void ref_rf_threads(int n) { g_rf_threads = n > 0 ? n : 1; }

void generate_SND(double* kexi, int n)
{
    for (int i = 0; i < n * g_zeta_per; i++) kexi[i] = (g_zeta && i < g_zeta_n) ? g_zeta[i] : 0.0 / 0.0;
}

extern "C" int ref_rf_cholesky(int ndim, int n, const double* xp, const int* type, double dr, int no, int dist_type,
                               double mean_value, double sd_value, double coe_depth, const double* rl,
                               double cell_ndx, int flag_auto, double beta, double beta_1, const double* nb_min,
                               const double* nb_max, double soil_max, double water_max, const double* zeta,
                               int nzeta, double* out)
{
    Particle* par = new Particle[n];
    Para_Fluid* fl = new Para_Fluid[n];
    Para_Soil* so = new Para_Soil[n];
    const double nan = 0.0 / 0.0;
    for (int i = 0; i < n; i++) {
        for (int d = 0; d < 3; d++) par[i].xp[d] = xp[(size_t)i * 3 + d];
        par[i].type = type[i];
        fl[i].fai = fl[i].c = nan;
        so[i].fai = so[i].c = so[i].cop = so[i].ds = nan;
    }
    Para_Pro pro;
    pro.ndim = ndim;
    pro.ntotal = n;
    pro.dr = dr;
    Flag_SpatialVariability fsv;
    fsv.flag_fai = no == 0; fsv.flag_c = no == 1; fsv.flag_cop = no == 2; fsv.flag_ds = no == 3;
    fsv.flag_faiw = no == 4; fsv.flag_cw = no == 5;
    fsv.cell_ndx = cell_ndx;
    fsv.flag_auto = flag_auto;
    fsv.beta = beta;
    fsv.beta_1 = beta_1;
    Para_SpatialVariability psv[6];
    psv[no].no = no;
    psv[no].type = dist_type;
    psv[no].mean_value = mean_value;
    psv[no].sd_value = sd_value;
    psv[no].coe_depth = coe_depth;
    for (int d = 0; d < 3; d++) psv[no].rl_value[d] = rl[d];
    Cell_Con cc;
    cc.xmin_nb = nb_min[0]; cc.ymin_nb = nb_min[1]; cc.zmin_nb = nb_min[2];
    cc.xmax_nb = nb_max[0]; cc.ymax_nb = nb_max[1]; cc.zmax_nb = nb_max[2];
    for (int d = 0; d < 3; d++) { cc.soil_max[d] = soil_max; cc.water_max[d] = water_max; }
    g_zeta = zeta;
    g_zeta_n = nzeta;
    const int threads = omp_get_max_threads();
    omp_set_num_threads(g_rf_threads);
    clFSpatialVariability_Fun f;
    const int err = (ndim == 2) ? f.nonstationary_random_2D(par, fl, so, pro, fsv, psv, cc)
                                : f.nonstationary_random_3D(par, fl, so, pro, fsv, psv, cc);
    omp_set_num_threads(threads);
    g_zeta = nullptr;
    g_zeta_n = 0;
    for (int i = 0; i < n; i++) {
        double v = nan;
        switch (no) {
        case 0: v = so[i].fai; break;
        case 1: v = so[i].c; break;
        case 2: v = so[i].cop; break;
        case 3: v = so[i].ds; break;
        case 4: v = fl[i].fai; break;
        case 5: v = fl[i].c; break;
        }
        out[i] = v;
    }
    delete[] par;
    delete[] fl;
    delete[] so;
    return err;
}

namespace {

struct RFRun {
    Particle* par;
    Para_Fluid* fl;
    Para_Soil* so;
    Para_Pro pro;
    RFRun(int ndim, int n, const double* xp, const int* type, double dr)
    {
        par = new Particle[n];
        fl = new Para_Fluid[n];
        so = new Para_Soil[n];
        const double nan = 0.0 / 0.0;
        for (int i = 0; i < n; i++) {
            for (int d = 0; d < 3; d++) par[i].xp[d] = xp ? xp[(size_t)i * 3 + d] : 0.0;
            par[i].type = type[i];
            fl[i].fai = fl[i].c = nan;
            so[i].fai = so[i].c = so[i].cop = so[i].ds = nan;
        }
        pro.ndim = ndim;
        pro.ntotal = n;
        pro.dr = dr;
    }
    ~RFRun() { delete[] par; delete[] fl; delete[] so; }
    // friction then cohesion of the pair's phase
    void pair_out(int soil, double* out) const
    {
        for (int i = 0; i < pro.ntotal; i++) {
            out[i] = soil ? so[i].fai : fl[i].fai;
            out[(size_t)pro.ntotal + i] = soil ? so[i].c : fl[i].c;
        }
    }
};

void pair_setup(int no0, int dist_type, const double* mean, const double* sd, const double* coe_depth, const double* rl,
                double coe, Flag_SpatialVariability& fsv, Para_SpatialVariability* psv)
{
    const int soil = no0 == 0;
    fsv.flag_fai = soil; fsv.flag_c = soil; fsv.flag_cop = 0; fsv.flag_ds = 0;
    fsv.flag_faiw = !soil; fsv.flag_cw = !soil;
    fsv.coe_frict_cohesion = coe;
    for (int k = 0; k < 2; k++) {
        Para_SpatialVariability& p = psv[no0 + k];
        p.no = no0 + k;
        p.type = dist_type;
        p.mean_value = mean[k];
        p.sd_value = sd[k];
        p.coe_depth = coe_depth[k];
        for (int d = 0; d < 3; d++) p.rl_value[d] = rl[d];
    }
}

}  // namespace

/* flspv 4 with the pair normals u2 (cells x 2): friction and cohesion of the
 * phase of no0 (0 soil, 4 fluid) into out (2 x n) */
extern "C" int ref_rf_cholesky_corr(int ndim, int n, const double* xp, const int* type, double dr, int no0,
                                    int dist_type, const double* mean, const double* sd, const double* coe_depth,
                                    const double* rl, double cell_ndx, int flag_auto, double beta, double beta_1,
                                    double coe, const double* nb_min, const double* nb_max, double soil_max,
                                    double water_max, const double* u2, int nu, double* out)
{
    RFRun r(ndim, n, xp, type, dr);
    Flag_SpatialVariability fsv;
    Para_SpatialVariability psv[6];
    pair_setup(no0, dist_type, mean, sd, coe_depth, rl, coe, fsv, psv);
    fsv.cell_ndx = cell_ndx;
    fsv.flag_auto = flag_auto;
    fsv.beta = beta;
    fsv.beta_1 = beta_1;
    Cell_Con cc;
    cc.xmin_nb = nb_min[0]; cc.ymin_nb = nb_min[1]; cc.zmin_nb = nb_min[2];
    cc.xmax_nb = nb_max[0]; cc.ymax_nb = nb_max[1]; cc.zmax_nb = nb_max[2];
    for (int d = 0; d < 3; d++) { cc.soil_max[d] = soil_max; cc.water_max[d] = water_max; }
    g_zeta = u2;
    g_zeta_n = 2 * nu;
    g_zeta_per = 2;
    const int threads = omp_get_max_threads();
    omp_set_num_threads(g_rf_threads);
    clFSpatialVariability_Fun f;
    const int err = (ndim == 2) ? f.nonstationary_correlated_random_2D(r.par, r.fl, r.so, r.pro, fsv, psv, cc)
                                : f.nonstationary_correlated_random_3D(r.par, r.fl, r.so, r.pro, fsv, psv, cc);
    omp_set_num_threads(threads);
    g_zeta = nullptr;
    g_zeta_n = 0;
    g_zeta_per = 1;
    r.pair_out(no0 == 0, out);
    return err;
}

/* flspv 5 with the two normals u2 */
extern "C" int ref_rv_corr(int n, const int* type, int no0, int dist_type, const double* mean, const double* sd,
                           double coe, const double* u2, double* out)
{
    RFRun r(2, n, nullptr, type, 1.0);
    Flag_SpatialVariability fsv;
    Para_SpatialVariability psv[6];
    const double zero[2] = {0.0, 0.0}, rl[3] = {1.0, 1.0, 1.0};
    pair_setup(no0, dist_type, mean, sd, zero, rl, coe, fsv, psv);
    g_zeta = u2;
    g_zeta_n = 2;
    g_zeta_per = 2;
    clFSpatialVariability_Fun f;
    const int err = f.random_variable_generate(r.par, r.fl, r.so, r.pro, fsv, psv);
    g_zeta = nullptr;
    g_zeta_n = 0;
    g_zeta_per = 1;
    r.pair_out(no0 == 0, out);
    return err;
}
