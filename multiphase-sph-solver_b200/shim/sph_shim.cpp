// sph_shim.cpp -- the reference's step classes, backed by the B200 engine.
//
// A drop-in for the hot-path translation units of MultiPhase-SPH-Solver
// (CPP_3-NNPS, CPP_6-density, CPP_7-1/7-2/7-3, CPP_8-x, CPP_9-3/9-4/9-5,
// CPP_10/10-1, CPP_11, CPP_12-1, CPP_13): it defines the public methods of
// clNNPS_Fun, clDensity_Fun, clStraStre_Fun, clInterFor_Fun, clAcce_Fun (the
// vibration methods of CPP_9-1 included), clVel_Fun, clUpdate_Fun::update,
// clBndy_Fun, clSoilStruct_Fun and the free-field classes of CPP_19
// (clFreeFieldBndy_Fun, clFreeFieldBndy_Fun_soil) with the signatures of the
// reference's own Class_Functions.h (:41-185, :242-253, :278-296), which this
// file includes from the caller's source tree.  SPH_Calculation (CPP_1-SPHLoops.cpp) then links
// against it unchanged and runs its time steps on the GPU through the sphgpu
// C ABI (include/sphgpu.h).
//
// How the calls map onto the engine.  The device holds the particle state;
// the caller's Particle array is its host copy.
//   * parttocell / partisearching run at once (sphgpu_parttocell /
//     sphgpu_partisearching), because the caller acts on their codes 3 and 5;
//     on an error the host copy is brought up to date before the return, for
//     the caller's output_total.
//   * every other method up to update records what its arguments tell about
//     the run (boundary type, kernel flags, drag form, soil-structure contact,
//     thresholds, gravity, moving boundaries, the material records) and
//     returns; update pushes the recorded parameters (sphgpu_update_params)
//     and runs the rest of the step as the engine's fused passes
//     (sphgpu_update).  An error from that work, which update cannot return,
//     is returned by the next parttocell.
//   * host copy: the Particle array is uploaded when a run starts (an array,
//     a particle count or a step counter the device's state does not
//     continue: l = 1, or an l other than the device's) and downloaded after the
//     steps whose state SPH_Calculation writes out (l % fop == 0, l == 1, and
//     the step after which the time runs out, CPP_1-SPHLoops.cpp:761-783).
//     With SPHGPU_SHIM_SYNC=always in the environment it is uploaded before
//     and downloaded after every step instead, for callers whose host code
//     edits or reads particles between steps (rain, excavation).
// celllist_ini1 computes the cell counts on the host as the reference does
// (CPP_3-NNPS.cpp:96-121); celllist_ini2's table is left to the device, which
// forms each cell's stencil itself.  Host arrays the engine keeps on the
// device (Par_Cell, cell_info, cell_link, parti_cellid, cl_bndy_pair,
// clVar_Boundary, clRaij, clPair_SS, clInterf_SS, clParti_Pair, StiffMat,
// vx_temp) are accepted and not touched.
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "Class_Functions.h"
#include "sphgpu.h"

// The material records cross the C ABI as the engine's structs; their
// members must sit where the reference's classes keep them.
#define SHIM_SAME(T, U, m) static_assert(offsetof(T, m) == offsetof(U, m), #T "::" #m " offset")
SHIM_SAME(Para_Fluid, sphgpu_fluid, vis); SHIM_SAME(Para_Fluid, sphgpu_fluid, vpu);
SHIM_SAME(Para_Fluid, sphgpu_fluid, dens); SHIM_SAME(Para_Fluid, sphgpu_fluid, paa0);
SHIM_SAME(Para_Fluid, sphgpu_fluid, porosity); SHIM_SAME(Para_Fluid, sphgpu_fluid, fai);
SHIM_SAME(Para_Fluid, sphgpu_fluid, c); SHIM_SAME(Para_Fluid, sphgpu_fluid, bhtype);
SHIM_SAME(Para_Fluid, sphgpu_fluid, press_type); SHIM_SAME(Para_Fluid, sphgpu_fluid, acc_type);
SHIM_SAME(Para_Fluid, sphgpu_fluid, pre_coe); SHIM_SAME(Para_Fluid, sphgpu_fluid, strain_min);
static_assert(sizeof(Para_Fluid) == sizeof(sphgpu_fluid), "Para_Fluid size");
SHIM_SAME(Para_Soil, sphgpu_soil, e); SHIM_SAME(Para_Soil, sphgpu_soil, poi); SHIM_SAME(Para_Soil, sphgpu_soil, eps0);
SHIM_SAME(Para_Soil, sphgpu_soil, dens); SHIM_SAME(Para_Soil, sphgpu_soil, damp1);
SHIM_SAME(Para_Soil, sphgpu_soil, damp2); SHIM_SAME(Para_Soil, sphgpu_soil, cop);
SHIM_SAME(Para_Soil, sphgpu_soil, ramda); SHIM_SAME(Para_Soil, sphgpu_soil, kapa); SHIM_SAME(Para_Soil, sphgpu_soil, zmf);
SHIM_SAME(Para_Soil, sphgpu_soil, ann); SHIM_SAME(Para_Soil, sphgpu_soil, bnn); SHIM_SAME(Para_Soil, sphgpu_soil, beta);
SHIM_SAME(Para_Soil, sphgpu_soil, sitas); SHIM_SAME(Para_Soil, sphgpu_soil, sitar);
SHIM_SAME(Para_Soil, sphgpu_soil, epsr); SHIM_SAME(Para_Soil, sphgpu_soil, epss); SHIM_SAME(Para_Soil, sphgpu_soil, sd);
SHIM_SAME(Para_Soil, sphgpu_soil, sw); SHIM_SAME(Para_Soil, sphgpu_soil, kse); SHIM_SAME(Para_Soil, sphgpu_soil, c1);
SHIM_SAME(Para_Soil, sphgpu_soil, c2); SHIM_SAME(Para_Soil, sphgpu_soil, c3); SHIM_SAME(Para_Soil, sphgpu_soil, fai);
SHIM_SAME(Para_Soil, sphgpu_soil, c); SHIM_SAME(Para_Soil, sphgpu_soil, ocr); SHIM_SAME(Para_Soil, sphgpu_soil, sme0);
SHIM_SAME(Para_Soil, sphgpu_soil, mzm); SHIM_SAME(Para_Soil, sphgpu_soil, azm); SHIM_SAME(Para_Soil, sphgpu_soil, r0);
SHIM_SAME(Para_Soil, sphgpu_soil, bl); SHIM_SAME(Para_Soil, sphgpu_soil, bz); SHIM_SAME(Para_Soil, sphgpu_soil, zet);
SHIM_SAME(Para_Soil, sphgpu_soil, vpu); SHIM_SAME(Para_Soil, sphgpu_soil, porosity);
SHIM_SAME(Para_Soil, sphgpu_soil, fs); SHIM_SAME(Para_Soil, sphgpu_soil, etao); SHIM_SAME(Para_Soil, sphgpu_soil, g0);
SHIM_SAME(Para_Soil, sphgpu_soil, ds); SHIM_SAME(Para_Soil, sphgpu_soil, damp_coe);
static_assert(sizeof(Para_Soil) == sizeof(sphgpu_soil), "Para_Soil size");
// Particle records cross as whole records (sphgpu_upload/download_particles)
static_assert(sizeof(Particle) >= 1064, "Particle record");
#undef SHIM_SAME

namespace {

struct ShimRun {
    sphgpu_ctx* ctx = nullptr;
    Particle* par = nullptr;          // the host array the device state mirrors
    int n = 0;
    sphgpu_params P;                  // the run as the method arguments describe it
    sphgpu_params pushed;             // the parameters the context last took
    const Para_Fluid* fluid = nullptr;
    const Para_Soil* soil = nullptr;
    bool mats_sent = false;
    int pending = 0;                  // an error of the last update, for the next parttocell
    bool sync_always = false;
    const Para_Vibra* vib = nullptr;  // the vibration table the vibration methods were handed
    bool vib_sent = false;
};

ShimRun g_run;

void shim_fail(const char* what, int code)
{
    std::fprintf(stderr, "sphgpu shim: %s failed: %d (%s)\n", what, code, sphgpu_error_string(code));
}

// SPHGPU_SHIM_TRACE=1: the parameters each push hands the engine, on stderr
void trace_params(const char* when, const sphgpu_params& P)
{
    const char* t = std::getenv("SPHGPU_SHIM_TRACE");
    if (!t || t[0] != '1') return;
    std::fprintf(stderr,
                 "sphgpu shim %s: ndim %d n %d flknl %d flbndy %d fli %d flv %d flts %d flagum %d inip %d "
                 "step_regu %d loop %d fop %d dr %.17g dt %.17g g %.17g %.17g %.17g thr %.17g %.17g "
                 "interc %.17g permtype %d pers %.17g perl %.17g perm %.17g ss %d %.17g %.17g %d coe_bndy %.17g "
                 "if_cal %d if_move %d move %.17g %.17g %.17g alphats %.17g acc %d %d art %.17g xsph %.17g %.17g %.17g "
                 "st %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n",
                 when, P.ndim, P.ntotal, P.flknl, P.flbndy, P.fli, P.flv, P.flts, P.flagum, P.inip, P.step_regu,
                 P.loop, P.fop, P.dr, P.dt, P.gx, P.gy, P.gz, P.threshold_min, P.threshold_max, P.interc,
                 P.permtype, P.pers, P.perl, P.perm, P.ss_type, P.ss_myu, P.ss_zeta, P.ss_acc_type, P.coe_bndy,
                 P.if_cal, P.if_move, P.move_vx[0], P.move_vx[1], P.move_vx[2], P.alphats, P.water_acc_type,
                 P.air_acc_type, P.art_stre_coe, P.xsph[0], P.xsph[1], P.xsph[2], P.structure.dens,
                 P.structure.eps0, P.structure.e, P.structure.poi, P.structure.vpu, P.structure.porosity,
                 P.structure.cop);
}

void take_pro(const Para_Pro& pro)
{
    sphgpu_params& P = g_run.P;
    P.ndim = pro.ndim;
    P.ntotal = pro.ntotal;
    P.inip = pro.inip;
    P.step_regu = pro.step_regu;
    P.loop = pro.loop;
    P.fop = pro.fop;
    P.dr = pro.dr;
    P.dt = pro.dt;
    for (int a = 0; a < 3; a++) P.xsph[a] = pro.xsph[a];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 2; b++) P.art_vis[a][b] = pro.art_vis[a][b];
    P.art_stre_coe = pro.art_stre_coe;
}

void take_gravity(const Para_GF& g)
{
    g_run.P.gx = g.gx;
    g_run.P.gy = g.gy;
    g_run.P.gz = g.gz;
}

void take_inter(const Para_Inter& in)
{
    sphgpu_params& P = g_run.P;
    P.interc = in.interc;
    P.permtype = in.permtype;
    P.pers = in.pers;
    P.perl = in.perl;
    P.perm = in.perm;
}

void take_ss(const Para_SSInter& ss)
{
    sphgpu_params& P = g_run.P;
    P.ss_myu = ss.myu;
    P.ss_zeta = ss.zeta;
    P.ss_acc_type = ss.acc_type;
}

void download()
{
    if (!g_run.ctx) return;
    int rc = sphgpu_download_particles(g_run.ctx, g_run.par, g_run.n, sizeof(Particle));
    if (rc) shim_fail("sphgpu_download_particles", rc);
}

// the context for this Particle array, created (and loaded from the host
// copy) when the array or its particle count is new
int ensure_context(Particle* par, const Cell_Con& cc, const Para_Pro& pro)
{
    take_pro(pro);
    sphgpu_params& P = g_run.P;
    P.xmin = cc.xmin; P.xmax = cc.xmax;
    P.ymin = cc.ymin; P.ymax = cc.ymax;
    P.zmin = cc.zmin; P.zmax = cc.zmax;
    P.cxm = cc.cxm; P.cym = cc.cym; P.czm = cc.czm; P.ctotal = cc.ctotal;
    const char* mode = std::getenv("SPHGPU_SHIM_SYNC");
    g_run.sync_always = mode && std::strcmp(mode, "always") == 0;
    // a new run: another array, another particle count, or a step counter
    // that does not continue the device's (a run that starts again at l = 1
    // may be handed an array at the address the previous run's had)
    if (g_run.ctx && (g_run.par != par || g_run.n != pro.ntotal || pro.l == 1 ||
                      pro.l != sphgpu_get_step(g_run.ctx))) {
        sphgpu_destroy(g_run.ctx);
        g_run.ctx = nullptr;
    }
    if (!g_run.ctx) {
        // a new run: nothing recorded for an earlier array carries over
        const sphgpu_params keep = P;
        P = sphgpu_params{};
        take_pro(pro);
        P.xmin = keep.xmin; P.xmax = keep.xmax; P.ymin = keep.ymin; P.ymax = keep.ymax;
        P.zmin = keep.zmin; P.zmax = keep.zmax;
        P.cxm = keep.cxm; P.cym = keep.cym; P.czm = keep.czm; P.ctotal = keep.ctotal;
        g_run.fluid = nullptr;
        g_run.soil = nullptr;
        g_run.vib = nullptr;
        g_run.vib_sent = false;
        // what the methods of the first step have not told yet: the
        // reference's defaults (velocity-correction walls, the cubic spline,
        // the free-surface thresholds of CPP_1-SPHLoops.cpp:83-84)
        if (P.flbndy == 0) P.flbndy = 1;
        if (P.flknl == 0) P.flknl = 1;
        if (P.threshold_max == 0.0 && P.threshold_min == 0.0) {
            P.threshold_min = 0.1;
            P.threshold_max = 0.12;
        }
        g_run.ctx = sphgpu_create(&P, 0);
        if (!g_run.ctx) return sphgpu_last_create_error();
        g_run.par = par;
        g_run.n = pro.ntotal;
        g_run.pushed = P;
        g_run.mats_sent = false;
        int rc = sphgpu_upload_particles(g_run.ctx, par, pro.ntotal, sizeof(Particle));
        if (rc) return rc;
    } else if (g_run.sync_always) {
        int rc = sphgpu_upload_particles(g_run.ctx, par, pro.ntotal, sizeof(Particle));
        if (rc) return rc;
        g_run.mats_sent = false;
    }
    if (sphgpu_get_step(g_run.ctx) != pro.l) return sphgpu_set_step(g_run.ctx, pro.l);
    return 0;
}

}  // namespace

// The suction of an unsaturated soil at saturation satu on the wetting
// (dsatu > 0) or drying branch of its water-retention curve, a free function
// of the replaced CPP_7-2-constitutive.cpp (:323-338) that the reference's
// initialisation (CPP_2-initialf.cpp:1348, 1359) also calls: the tangent of
// the saturation's position between sitar and sitas, scaled through the
// curve's c and s parameters, with the reference's truncated pi.
double moisturesuct(double satu, double dsatu, const Para_Soil& Soil)
{
    const double pi_ref = 3.141592653;
    const double t = tan(pi_ref * (Soil.sitas - satu) / (Soil.sitas - Soil.sitar) / 2.0);
    if (dsatu > 0.0) return log(1 + exp(Soil.c2 * Soil.sw) * t) / Soil.c2;
    return log(1 + exp(Soil.c1 * Soil.sd) * t) / Soil.c1;
}

// ---------------------------------------------------------------- clNNPS_Fun

void clNNPS_Fun::celllist_ini1(Cell_Con* pCellc, const Para_Pro& pPPro)
{
    // cell edges of 2 dr and three cells of margin per axis
    const double cdr = 2.0 * pPPro.dr;
    pCellc->cxm = (int)((pCellc->xmax - pCellc->xmin) / cdr + 3.0);
    pCellc->cym = (int)((pCellc->ymax - pCellc->ymin) / cdr + 3.0);
    pCellc->czm = (pPPro.ndim == 3) ? (int)((pCellc->zmax - pCellc->zmin) / cdr + 3.0) : 1;
    pCellc->ctotal = pCellc->cxm * pCellc->cym * pCellc->czm;
}

void clNNPS_Fun::celllist_ini2(cell_link*, const Cell_Con&, int, int) {}

int clNNPS_Fun::parttocell(Par_Cell*, cell_info*, const Cell_Con& pCellc, parti_cellid*, parti_cellid*,
                           const Para_Pro& pPPro, Particle* pPar, int, int, int, int)
{
    int rc = g_run.pending;
    g_run.pending = 0;
    if (rc) {
        download();
        return rc;
    }
    // what the presence of a call tells (a drag form, a soil-structure
    // contact, the saturation pass) is learnt afresh every step: a step that
    // makes no such call runs without it
    sphgpu_params& P = g_run.P;
    P.fli = 0;
    P.interc = 0.0; P.permtype = 0; P.pers = 0.0; P.perl = 0.0; P.perm = 0.0;
    P.ss_type = 0; P.ss_myu = 0.0; P.ss_zeta = 0.0; P.ss_acc_type = 0;
    P.flagum = 0;
    rc = ensure_context(pPar, pCellc, pPPro);
    if (rc) return rc;
    rc = sphgpu_parttocell(g_run.ctx);
    if (rc) download();
    return rc;
}

int clNNPS_Fun::partisearching(Par_Cell*, cell_info*, cell_link*, parti_cellid*, const Cell_Con&,
                               const Para_Pro&, Particle*, int, int flknl)
{
    if (!g_run.ctx) return SPHGPU_E_STATE;
    g_run.P.flknl = flknl;
    if (g_run.pushed.flknl != flknl) {
        int rc = sphgpu_update_params(g_run.ctx, &g_run.P);
        if (rc) return rc;
        g_run.pushed = g_run.P;
    }
    int rc = sphgpu_partisearching(g_run.ctx);
    if (rc) download();
    return rc;
}

void clNNPS_Fun::kernel_gradient_correction(Particle*, Par_Cell*, const Para_Pro&) {}

// ------------------------------------------------------------- clDensity_Fun

void clDensity_Fun::density(Particle*, Par_Cell*, Para_Fluid* pVFluid, cl_bndy_pair*, clVar_Boundary*,
                            const Para_Pro&, int bndytype)
{
    g_run.P.flbndy = bndytype;
    g_run.fluid = pVFluid;
}

// ------------------------------------------------------------ clStraStre_Fun

void clStraStre_Fun::strain_noreg(Particle*, Par_Cell*, cl_bndy_pair*, clVar_Boundary*, const Para_Pro&,
                                  int bndytype)
{
    g_run.P.flbndy = bndytype;
}

void clStraStre_Fun::strain_to_stress(Particle*, const Para_Soil* pParti_ConsPara, StiffMat*,
                                      const Para_Fluid* pVFluid, const Para_Structure& pStruct, const Para_Pro&,
                                      int, int flts, double alpha)
{
    sphgpu_params& P = g_run.P;
    P.flts = flts;
    P.alphats = alpha;
    P.structure.dens = pStruct.dens;
    P.structure.eps0 = pStruct.eps0;
    P.structure.e = pStruct.e;
    P.structure.poi = pStruct.poi;
    P.structure.vpu = pStruct.vpu;
    P.structure.porosity = pStruct.porosity;
    P.structure.cop = pStruct.cop;
    g_run.soil = pParti_ConsPara;
    g_run.fluid = pVFluid;
}

void clStraStre_Fun::Stress_eigValue(Particle*, const Para_Pro&, int) {}
void clStraStre_Fun::eos(Particle*, Par_Cell*, Para_Fluid* pVFluid, const Para_Pro&, int) { g_run.fluid = pVFluid; }
void clStraStre_Fun::stress_regu(Particle*, Par_Cell*, const Para_Pro&) {}
void clStraStre_Fun::strain_regu(Particle*, Par_Cell*, const Para_Pro&) {}

void clStraStre_Fun::free_surface_check(Particle*, Par_Cell*, const Para_Pro&, double max, double min)
{
    g_run.P.threshold_max = max;
    g_run.P.threshold_min = min;
}

// ------------------------------------------------------------ clInterFor_Fun

void clInterFor_Fun::saturation(Particle*, Par_Cell*, const Para_Soil* pParti_ConsPara, const Para_Pro&, int)
{
    g_run.P.flagum = 1;
    g_run.soil = pParti_ConsPara;
}

void clInterFor_Fun::cal_permeability(Particle*, const Para_Inter& pPInter, const Para_Soil* pParti_ConsPara,
                                      const Para_Pro&, int)
{
    take_inter(pPInter);
    g_run.soil = pParti_ConsPara;
}

void clInterFor_Fun::interact1(Particle*, Par_Cell*, const Para_Inter& pInter, const Para_Fluid*,
                               const Para_Pro&, Para_GF pgf, int)
{
    g_run.P.fli = 1;
    take_inter(pInter);
    take_gravity(pgf);
}

void clInterFor_Fun::interact2(Particle*, Par_Cell*, const Para_Inter& pInter, const Para_Soil*,
                               const Para_Fluid*, const Para_Pro&, Para_GF pgf, int)
{
    g_run.P.fli = 2;
    take_inter(pInter);
    take_gravity(pgf);
}

void clInterFor_Fun::interact3(Particle*, Par_Cell*, const Para_Inter& pInter, const Para_Soil*,
                               const Para_Fluid*, const Para_Pro&, Para_GF pgf, int)
{
    g_run.P.fli = 3;
    take_inter(pInter);
    take_gravity(pgf);
}

// ---------------------------------------------------------------- clAcce_Fun

void clAcce_Fun::fluid_acceleration_water(Particle*, Par_Cell*, const Para_Fluid*, const Para_Pro&,
                                          const Para_GF& pPGf, int)
{
    g_run.P.water_acc_type = 0;
    take_gravity(pPGf);
}

void clAcce_Fun::fluid_acceleration_air(Particle*, Par_Cell*, const Para_Fluid*, const Para_Pro&,
                                        const Para_GF& pPGf, int)
{
    g_run.P.air_acc_type = 0;
    take_gravity(pPGf);
}

void clAcce_Fun::fluid_acceleration_minorwater(Particle*, Par_Cell*, const Para_Fluid*, const Para_Pro&,
                                               const Para_GF& pPGf, int)
{
    g_run.P.water_acc_type = 1;
    take_gravity(pPGf);
}

void clAcce_Fun::fluid_acceleration_minorair(Particle*, Par_Cell*, const Para_Fluid*, const Para_Pro&,
                                             const Para_GF& pPGf, int)
{
    g_run.P.air_acc_type = 1;
    take_gravity(pPGf);
}

void clAcce_Fun::soil_acceleration_noreg(Particle*, Par_Cell*, const Para_Soil* pParti_ConsPara,
                                         const Para_Pro&, const Para_GF& pPGf, int)
{
    g_run.soil = pParti_ConsPara;
    take_gravity(pPGf);
}

void clAcce_Fun::structure_acceleration_noreg(Particle*, Par_Cell*, const Para_Pro&, const Para_GF& pPGf, int)
{
    take_gravity(pPGf);
}

void clAcce_Fun::boundary_moving_stress_effect(Particle*, Par_Cell*, const Para_Pro&, int) {}
void clAcce_Fun::boundary_effect_free_struct(Particle*, Par_Cell*, const Para_Pro&, int) {}
void clAcce_Fun::artificial_viscosity(Particle*, Par_Cell*, const Para_Soil*, const Para_Fluid*, const Para_Pro&,
                                      int) {}
void clAcce_Fun::artificial_stress_2d(Particle*, Par_Cell*, const Para_Pro&, clRaij*, int) {}
void clAcce_Fun::artificial_stress_3d(Particle*, Par_Cell*, const Para_Pro&, clRaij*, int) {}

void clAcce_Fun::coupled_Water_Soil_Structure(Particle*, Par_Cell*, const Para_Fluid*, const Para_Soil*,
                                              const Para_Pro&, const Para_GF& pPGf, int)
{
    take_gravity(pPGf);
}

void clAcce_Fun::soil_damping_geostress(Particle*, Par_Cell*, const Para_Pro&, int) {}

// vibration (flv 1, 2): the table is handed to the engine with the step's
// parameters; the loads, the damping and the free-field terms run inside the
// step
void clAcce_Fun::vibration_acceleration(Particle*, const Para_Vibra& pPVib, const Para_Pro&, int) { g_run.vib = &pPVib; }
void clAcce_Fun::vibration_velocity(Particle*, const Para_Vibra& pPVib, const Para_Pro&, int) { g_run.vib = &pPVib; }
void clAcce_Fun::soil_damping_vibration(Particle*, Par_Cell*, const Para_Soil* pParti_ConsPara, StiffMat*,
                                        const Para_Pro&)
{
    g_run.soil = pParti_ConsPara;
}

// ------------------------------------------------------ free-field boundaries

void clFreeFieldBndy_Fun::free_field_solid(Particle*, cl_bndy_pair*, const Para_Soil, Par_Cell*, const Para_Pro&,
                                           int)
{
}

void clFreeFieldBndy_Fun_soil::free_field_solid(Particle*, const Para_Soil* pParti_ConsPara, Par_Cell*,
                                                const Para_Pro&, int)
{
    g_run.soil = pParti_ConsPara;
}
void clAcce_Fun::boundary_stress_effect_tran(Particle*, Par_Cell*, clVar_Boundary*, const Para_Pro&, int) {}

// ---------------------------------------------------------- clSoilStruct_Fun

int clSoilStruct_Fun::interaction_ss_rigid(Particle*, Par_Cell*, clPair_SS*, clInterf_SS**, clParti_Pair*,
                                           const Para_SSInter& pSSInter, const Para_Pro&, int)
{
    g_run.P.ss_type = 1;
    take_ss(pSSInter);
    return 0;
}

int clSoilStruct_Fun::interaction_ss_deformable(Particle*, Par_Cell*, clPair_SS*, clInterf_SS**, clParti_Pair*,
                                                const Para_SSInter& pSSInter, const Para_Pro&, int)
{
    g_run.P.ss_type = 2;
    take_ss(pSSInter);
    return 0;
}

int clSoilStruct_Fun::interaction_ss_penalty(Particle*, Par_Cell*, clPair_SS*, clInterf_SS**, clParti_Pair*,
                                             const Para_SSInter& pSSInter, const Para_Pro&, int)
{
    g_run.P.ss_type = 3;
    take_ss(pSSInter);
    return 0;
}

// ----------------------------------------------------------------- clVel_Fun

void clVel_Fun::veocity_update(Particle*, const Para_Pro&, const Para_Boundary& pPBou, int flv)
{
    sphgpu_params& P = g_run.P;
    P.flv = flv;
    P.if_cal = pPBou.if_cal;
    P.if_move = pPBou.if_move;
    P.coe_bndy = pPBou.coe_bndy;
    for (int k = 0; k < 3; k++) P.move_vx[k] = pPBou.move_vx[k];
}

void clVel_Fun::xsph(Particle*, Par_Cell*, cl_bndy_pair*, clVar_Boundary*, const Para_Pro&, double (*)[3],
                     int bndytype)
{
    g_run.P.flbndy = bndytype;
}

// ---------------------------------------------------------------- clBndy_Fun

void clBndy_Fun::tmboundary(Particle*, Par_Cell*, cl_bndy_pair*, const Para_Pro&) {}
void clBndy_Fun::tm_boundary_2d(Particle*, Par_Cell*, cl_bndy_pair*, clVar_Boundary*, const Para_Pro&, int) {}
void clBndy_Fun::tm_boundary_3d(Particle*, Par_Cell*, cl_bndy_pair*, clVar_Boundary*, const Para_Pro&, int) {}
void clBndy_Fun::no_slip_tran(Particle*, Par_Cell*, clVar_Boundary*, const Para_Pro&, int) {}
void clBndy_Fun::free_slip_tran(Particle*, Par_Cell*, clVar_Boundary*, const Para_Pro&, int) {}
void clBndy_Fun::check_domain(Particle*, const Cell_Con&, const Para_Boundary&, const Para_Pro&) {}

void clBndy_Fun::velocity_set_domain(Particle*, Par_Cell*, cl_bndy_pair*, const Para_Pro&, double coe_bndy)
{
    g_run.P.coe_bndy = coe_bndy;
}

void clBndy_Fun::boundary_free_solid(Particle*, Par_Cell*, const Para_Pro&, Para_SSInter pSSInter, int)
{
    take_ss(pSSInter);
}

// -------------------------------------------------------------- clUpdate_Fun

void clUpdate_Fun::update(Particle* pPar, const Para_Pro& pPPro, const Para_Boundary& pPBou, int)
{
    if (!g_run.ctx || pPar != g_run.par) return;
    sphgpu_params& P = g_run.P;
    take_pro(pPPro);
    P.if_move = pPBou.if_move;
    for (int k = 0; k < 3; k++) P.move_vx[k] = pPBou.move_vx[k];
    int rc = 0;
    if (std::memcmp(&P, &g_run.pushed, sizeof(P)) != 0) {
        trace_params("update_params", P);
        rc = sphgpu_update_params(g_run.ctx, &P);
        if (rc) shim_fail("sphgpu_update_params", rc);
        else g_run.pushed = P;
    }
    if (!rc && P.flv >= 1 && g_run.vib && !g_run.vib_sent) {
        const Para_Vibra& v = *g_run.vib;
        const sphgpu_vibration vb = {v.ttime, v.nsteps, v.sttime, v.edtime};
        rc = sphgpu_set_vibration(g_run.ctx, &vb, v.loads ? &v.loads[0][0] : nullptr);
        if (rc) shim_fail("sphgpu_set_vibration", rc);
        else g_run.vib_sent = true;
    }
    if (!rc && !g_run.mats_sent) {
        rc = sphgpu_set_materials(g_run.ctx, reinterpret_cast<const sphgpu_fluid*>(g_run.fluid),
                                  reinterpret_cast<const sphgpu_soil*>(g_run.soil), g_run.n);
        if (rc) shim_fail("sphgpu_set_materials", rc);
        else g_run.mats_sent = true;
    }
    if (!rc) rc = sphgpu_update(g_run.ctx);
    if (rc) {
        g_run.pending = rc;
        return;
    }
    // the host copy, where SPH_Calculation reads it next
    const bool out = pPPro.l % pPPro.fop == 0 || pPPro.l == 1 || !(pPPro.t < pPPro.tt);
    if (out || g_run.sync_always) download();
}
