// sph_device.cuh -- device state and per-pair helpers of the sm_100a SPH step.
//
// Layout in HBM (particle arrays indexed by the reference particle index i,
// i.e. the order of the caller's Particle array):
//   * positions: double xh[4 * N], particle-major records (x, y, z, h) --
//                one 32-byte sector per neighbour gather; xs[4 * N] is the
//                same records in cell-sorted order, streamed by the NNPS scan
//   * scalars:   T a[N]
//   * vectors:   double a[3 * N], component k of particle i at a[k * N + i]
//   * tensors:   double a[6 * N] (Voigt order xx yy zz xy yz zx, as
//                Particle::sig), component k at a[k * N + i]
//   * neighbour lists: int nbr[SPH_NB_CAP * N], slot s of particle i at
//                nbr[s * N + i], so the threads of a warp read consecutive
//                words per slot; the pair's kernel gradient and value
//                (Par_Cell::wij) in the same slot order, nbw[s * N + i], as a
//                32-byte FP64 record or a 16-byte FP32 record (bulk form).
// Component-major storage makes every own-particle load of one component a
// coalesced 8-byte-per-lane access.
//
// Arithmetic follows the reference's operation order; the library is built
// with -fmad=false so no multiply-add is contracted, which keeps the FP64
// results identical to the reference's x86-64 build (no FMA).  Where a
// subexpression that the reference evaluates per pair depends on one particle
// only, it is evaluated once per particle and reused when a bitwise guard
// shows the operands are the same (e.g. equal porosities), which yields the
// same rounded value.
#pragma once
#include <cstdint>

#define SPH_NB_CAP 99          // Par_Cell::influ[100], slots 1..99 (Class_NNPS.h:71)
#define SPH_ERR_CELL 3         // parttocell, CPP_3-NNPS.cpp:247-257
#define SPH_ERR_NEIGH 5        // partisearching, CPP_3-NNPS.cpp:313-319
#define SPHK_NSTAGES 21        // entries of sphk_stage_names (one event bracket each)
#ifndef SPHGPU_CHECK
#define SPHGPU_CHECK 0         // 1: the bounds-checked build (k_check_lists after the search)
#endif
#define SPH_ERR_CHECK 106      // its error code (SPHGPU_E_CHECK)

// One instance of a batched context: its particle range, its own cell grid
// (Cell_Con, celllist_ini1) and where its cells start in the context's cell
// numbering.  The instances share every other parameter.
struct InstGrid {
    double xmin, ymin, zmin, xmax, ymax, zmax;
    int cxm, cym, czm, ctotal;
    int cell_base;             // context cell id of the instance's cell 0
    int first, count;          // particles [first, first + count)
    int first_vbx_wall;        // its first wall (index order) with matype > 2, or first + count
};

// Passes whose threads per block the autotuner picks (one particle per
// thread; every pass is written for any multiple of 32 up to its launch
// bound of 128)
enum TunePass {
    TP_NNPS, TP_RESOLVE, TP_PAIRW, TP_DENSITY, TP_SHEPARD, TP_STRAIN, TP_STRESS, TP_ACCEL_A, TP_ACCEL_B,
    TP_XSPH, TP_COUNT
};

struct DevParams {
    int N, ndim, flknl, flbndy, fli, if_move, flv, inip, step_regu;
    int cxm, cym, czm, ctotal;
    int water_minor, air_minor;
    int first_vbx_wall;        // first wall (pid order) with matype > 2, or N
    double dr, dt;
    double xsph0, xsph1, xsph2;
    double av[3][2];
    double gx, gy, gz;
    double thr_min, thr_max;
    double interc, pers, perl, perm;
    int permtype;
    double coe_bndy;
    double move_vx[3];
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double st_e, st_poi;       // Para_Structure elastic constants
    double g_acc;              // |g|, interact1 (CPP_10-interact1.cpp:28)
    double art_stre_coe;       // artificial stress coefficient (0: off)
    int ss_type;               // soil-structure contact: 0 none, 1 rigid, 2 deformable, 3 penalty
    int ss_coupled;            // 1: coupled_Water_Soil_Structure (ss_type 1-3 with acc_type 2)
    double ss_myu, ss_zeta;
    int bulk;                  // 1: the FP32-bulk form (pair records in FP32)
    int flts;                  // >= 1: TSSMP stress transformation around the soil models
    int flagum;                // 1: the saturation pass (one unsaturated Cam-clay layer)
    double alphats;            // TSSMP alpha
    // adaptive time step (an extension, off unless sphgpu_set_cfl turns it
    // on; the reference's dt is constant, CPP_12-2-dt.cpp:13-20): the step
    // reads its dt from the device word dtv, which the last kernel of the
    // previous step set from the CFL and force limits, capped at dt
    int cfl_on;
    double cfl_c, cfl_f;       // factors of h / (c + |v|) and sqrt(h / |a|)
    double st_vpu;             // Para_Structure::vpu, the structure's sound speed
    int ninst;                 // batched context: number of instances (0: one system)
    int tb[TP_COUNT];          // threads per block of the tuned passes
    // rainfall (flr 1, rtype 1): rainini's lp and vrain, Para_Rain::press_factor
    int flr, rain_lp;
    double rain_vrain, rain_press;
    // vibration (flv 1, 2): Para_Vibra's period, steps per period, start and
    // end time (its loads in DevState::vib_loads); the free-field walls'
    // elastic constants (the reference's pFFBound, a default-constructed
    // Para_Soil: e = poi = 0, CPP_1-SPHLoops.cpp:253)
    double vib_ttime, vib_st, vib_ed;
    int vib_nsteps;
    double ff_e, ff_poi;
};

// Members of the soil record that only the unsaturated Cam-clay model, the
// saturation pass and the fractional-order Cam-clay read, in one block
// s_ext[k * N + i] (allocated when a particle uses them)
enum SoilExt {
    SX_EPSS, SX_EPSR, SX_BNN, SX_BETA, SX_SD, SX_SW, SX_C1, SX_C2,
    SX_G0, SX_ETAO, SX_ZET, SX_DAMP1, SX_DAMP2, SX_C4,   // SX_C4 = pow(c, 4), host libm
    SX_COUNT
};

struct DevState {
    // static per particle
    int *type, *matype, *etype, *permtype;
    double *mass, *cd;
    // fluid material record (pVFluid) used by the step
    double *f_dens, *f_por, *f_vpu, *f_vis, *f_c, *f_smin, *f_tanfai;
    int *f_bhtype;
    // soil material record (pParti_ConsPara) used by the step
    double *s_e, *s_poi, *s_eps0, *s_dens, *s_kapa, *s_por, *s_vpu, *s_cop, *s_sitas, *s_sitar;
    double *s_ds;              // mean grain diameter (interact2/3 drag)
    double *s_c, *s_fs;        // cohesion (viscous-elastic: shear modulus), strength reduction factor
    double *s_ann, *s_zmf, *s_ramda, *s_sme0;   // subloading Cam-clay
    double *s_yalf, *s_ykap, *s_yalf_dil;   // Drucker-Prager constants, host-evaluated
    double *s_ext;             // SoilExt members, SX_COUNT * N (or null)
    // positions (x, y, z, h) records, ping-pong
    double *xh, *xh_next;
    double *xs;                // xh in cell-sorted order (NNPS scan)
    float *xsf;                // xs as FP32 (x - xmin, y - ymin, z - zmin, h) records: the NNPS prefilter
    // dynamic state
    double *vx;                // velocity after the step
    double *vx_next;           // per particle (vx x, y, z before XSPH, mass): one 32-byte record
    double *vxp, *axp, *ax, *ux;
    double *rho, *rhop, *pre, *prep, *porosity, *poro_cop, *e;
    double *rho_c;             // per particle (continuity density, mass): one 16-byte record for Shepard
    double *svr;               // per particle (vxp x, y, z, mass / rho) after Shepard: the strain loop's record
    double *pmr;               // per particle (mass, rho, pre, 0) after Shepard: the pressure gathers' record
    double *dr4;               // per particle (rho, satu, porosity, soil: cop | fluid: f_dens) after the
                               // constitutive pass: the drag loop's record
    double *rrho;              // per particle (mass, porosity, rho, RN(1 / rho)) at the start of the step
                               // (k_pairw): k_density's porosity gathers in one record
    double *nv;                // per particle (vxp x, y, z, mass) as the step starts (k_pairw): the
                               // neighbour fields the density, strain and momentum loops gather, in
                               // one 32-byte record instead of four arrays
    double *sig, *sig_next;    // 6N each, ping-pong
    double *eps, *adps;
    double *tssig, *tsqc;      // TSSMP: the transformed stress and its q (flts >= 1)
    double *satu, *dsatu, *suct, *cop, *prew, *prea;
    double *interf, *interfss, *strep;
    double *vsig, *veps, *divq, *divr, *meps;
    // per-step intermediates
    double *de;                // strain rate, 6N
    double *we;                // spin, off-diagonal entries (0,1)(0,2)(1,0)(1,2)(2,0)(2,1): 6N
    double *color;             // free-surface colour sum
    double *sr;                // per particle, 8 doubles in one 64-byte record: stress / rho^2 as the
                               // momentum pass uses it (6, Voigt order), the pore-pressure term / rho^2
                               // and the mass, so that a neighbour's part of the pass is one record
    double *eps_in;            // strain the constitutive pass starts from: eps, or eps_tmp after strain_regu
    double *eps_tmp, *sig_tmp; // outputs of the regularisation passes, 6N each
    double *rij;               // artificial stress tensor R per soil particle, 9N row-major (art_stre_coe > 0)
    // flbndy 2: cl_bndy_pair::vel_bndy of the moving particles (3N), the
    // walls' clVar_Boundary velocities per phase vb[(p * 3 + k) * N + i],
    // p = water, soil, air, structure (12N), and the velocity tm_boundary
    // reads (after XSPH and velocity_set_domain, before check_domain; 3N)
    double *vel_bndy, *vb, *vx_vb;
    // flbndy 3/4/13/14: the walls' clVar_Boundary stresses per phase,
    // sb[(p * 6 + k) * N + i] (24N)
    double *sb;
    // flbndy 5: boundary_free_solid's force per particle, zeta (f_t + f_n)
    // (3N), and whether the particle touches the walls (N)
    double *fsol;
    int *fsol_on;
    // ss acc_type 2: coupled_Water_Soil_Structure's row sums per particle (3N)
    double *cpl;
    // soil-structure contact (ss_type 1-3): per water/soil particle the
    // structure particles it pushes (ss_id, 3N, -1 = none) with the forces
    // they take from it (ss_con, 18N: per slot q the normal then the
    // tangential force, component k at (q * 6 + c) * N + i, signed as the
    // reference applies them) and its own forces (ss_own, 6N: normal, then
    // tangential); per structure particle the gathered forces (ss_fs, 6N)
    int *ss_id;
    double *ss_con, *ss_own, *ss_fs;
    // the order the state is held in: the particle at i is the caller's
    // particle i2o[i] (its index in the reference's particle array), and
    // o2i is the inverse; identity until the state is re-sorted by cell
    int *i2o, *o2i;
    // NNPS
    int *cell;                 // cell id per particle
    uint32_t *key_in, *key_out;
    int *val_in, *pid_sorted;
    int *cstart, *cend;        // [ctotal + 4]
    int *nnb;                  // neighbour count (may exceed the cap: error 5)
    // the neighbour search by cell-sorted position q: pts[q] = the particle
    // index << 3 | its type code (the type for types 0-4, else 7); the scan's
    // provisional count (-1: the particle takes the direct FP64 search) and
    // provisional list nbrs[s * N + q] of candidates' pts words (~word for a
    // candidate within the FP32 margin of the radius); sortpos[i] = q
    int *nps, *nbrs, *sortpos, *pts;
    // the momentum pass's artificial-viscosity, drag and damping sums, from
    // its loop kernel to its tail kernel: accb[(3 g + k) * N + i] (9N); with
    // vibration (flv != 0) also the free-field sums of the walls (g = 3) and
    // of the soil (g = 4), the vibration damping sum (g = 5) and its
    // normaliser (row 18): 19N
    double* accb;
    // vibration (flv > 0): per soil / structure particle the largest of 0 and
    // the diagonal entries 0-2 of the constitutive matrix of its last stress
    // update (StiffMat::depp0, CPP_7-2-constitutive.cpp:112-292), N; and
    // Para_Vibra::loads, vib_nsteps x 3
    double *stiff, *vib_loads;
    // per particle and particle type t = 0..4, bit s set when list slot s
    // holds a particle of type t: nbm[(2 t + w) * N + i], word w = 0 for
    // slots 0-63, 1 for slots 64-98 (written by the search with the list)
    unsigned long long* nbm;
    int *nbr;                  // [SPH_NB_CAP * N]
    double *nbw;               // pair records (grad W, W) of the neighbour-list slots, [SPH_NB_CAP * N]
                               // records of 32 bytes (FP64), or 16 bytes (FP32, bulk form) in the
                               // first half of the same buffer
    // control words
    int *err;                  // first error code raised (0 = none)
    int *step;                 // Para_Pro::l of the step being run
    const InstGrid *inst;      // batched context: the instance table (ninst)
    int *pinst;                // batched context: each particle's instance
    int *nrain;                // rain particles still waiting (Para_Rain::nrain)
    double *tsim;              // Para_Pro::t, the simulated time after the last completed step
    double *dtv;               // dt of the step being run (cfl_on)
    unsigned long long *dtmin; // running minimum of the per-particle limits (bits of a positive double)
};

struct Dev {
    DevParams p;
    DevState s;
};

struct Pos { double x, y, z, h; };

// The cell grid and domain box of particle i: the context's, or in a batched
// context those of the particle's instance, whose cells are numbered from
// `base` in the context's cell ids.
struct CellGrid {
    int cxm, cym, czm, ctotal, base, w0;
    double xmin, ymin, zmin, xmax, ymax, zmax;
};

__device__ __forceinline__ CellGrid cell_grid(const Dev& d, int i)
{
    if (d.p.ninst == 0)
        return CellGrid{d.p.cxm, d.p.cym, d.p.czm, d.p.ctotal, 0, d.p.first_vbx_wall,
                        d.p.xmin, d.p.ymin, d.p.zmin, d.p.xmax, d.p.ymax, d.p.zmax};
    const InstGrid& g = d.s.inst[d.s.pinst[i]];
    return CellGrid{g.cxm, g.cym, g.czm, g.ctotal, g.cell_base, g.first_vbx_wall,
                    g.xmin, g.ymin, g.zmin, g.xmax, g.ymax, g.zmax};
}

// the step's time increment: the input dt, or with the adaptive step on the
// value the previous step's limit reduction left in dtv
__device__ __forceinline__ double step_dt(const Dev& d) { return d.p.cfl_on ? *d.s.dtv : d.p.dt; }

__device__ __forceinline__ Pos load_pos(const double* xh, int i)
{
    const double2* p = reinterpret_cast<const double2*>(xh) + 2 * (size_t)i;
    double2 a = p[0], b = p[1];
    return Pos{a.x, a.y, b.x, b.y};
}

// the momentum record of particle j (DevState::sr)
struct SR { double s[6], p, m; };
__device__ __forceinline__ SR load_sr(const double* sr, int j)
{
    const double2* q = reinterpret_cast<const double2*>(sr) + 4 * (size_t)j;
    const double2 a = q[0], b = q[1], c = q[2], e = q[3];
    return SR{{a.x, a.y, b.x, b.y, c.x, c.y}, e.x, e.y};
}
__device__ __forceinline__ void store_sr(double* sr, int i, const double s[6], double p, double m)
{
    double2* q = reinterpret_cast<double2*>(sr) + 4 * (size_t)i;
    q[0] = make_double2(s[0], s[1]);
    q[1] = make_double2(s[2], s[3]);
    q[2] = make_double2(s[4], s[5]);
    q[3] = make_double2(p, m);
}

// the neighbour record of particle j: vxp (x, y, z) and mass
struct NV { double vx, vy, vz, m; };
__device__ __forceinline__ NV load_nv(const double* nv, int j)
{
    const double2* p = reinterpret_cast<const double2*>(nv) + 2 * (size_t)j;
    double2 a = p[0], b = p[1];
    return NV{a.x, a.y, b.x, b.y};
}

__device__ __forceinline__ void store_pos(double* xh, int i, const Pos& q)
{
    double2* p = reinterpret_cast<double2*>(xh) + 2 * (size_t)i;
    p[0] = make_double2(q.x, q.y);
    p[1] = make_double2(q.z, q.h);
}

// the normalisation constant a1 of weight() / weight2() for support ra
// (CPP_3-NNPS.cpp:24-29, 58-63), in the pair arithmetic's type R
template <typename R>
__device__ __forceinline__ R kernel_a1(R ra, int ndim, int flknl)
{
    if (flknl == 1 || flknl == 3)
        return (ndim == 2) ? R(0.682092613250980) / ra / ra : R(0.477464829275686) / ra / ra / ra;
    return (ndim == 2) ? R(0.106103295394597) / (ra * ra) : R(0.077010456334788) / (ra * ra * ra);
}

// A pair sum.  In FP64 it is the plain running sum the reference forms; in
// FP32 (the bulk form) it is Kahan-compensated, and the compensation is folded
// back in FP64 when the sum is read.
template <typename R> struct Sum;
template <> struct Sum<double> {
    double s = 0.0;
    __device__ __forceinline__ void add(double x) { s = s + x; }
    __device__ __forceinline__ double v() const { return s; }
};
template <> struct Sum<float> {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add(float x)
    {
        const float y = x - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double v() const { return (double)s - (double)c; }
};

// Particle i's side of every pair: position (FP64: pair differences are
// taken in FP64 and then rounded to R), h and a1 for ra = h_i (the
// reference's ra = (h_i + h_j) / 2 equals h_i exactly when h_j == h_i).
template <typename R>
struct PairI {
    double x[3];
    R h, a1;
};

template <int ND, typename R>
__device__ __forceinline__ PairI<R> pair_i(const Dev& d, int i)
{
    Pos q = load_pos(d.s.xh, i);
    PairI<R> I;
    I.x[0] = q.x; I.x[1] = q.y; I.x[2] = q.z; I.h = (R)q.h;
    I.a1 = kernel_a1<R>(I.h, ND, d.p.flknl);
    return I;
}

// x / y correctly rounded, from yr = RN(1 / y): q = RN(x yr) lies within one
// ulp of x / y, the residual x - q y is then exact as a fused multiply-add,
// and RN(q + r yr) is RN(x / y) (Markstein's correction).  A zero residual
// means q is exact and is returned as it is, which also keeps the sign of a
// zero quotient.  A residual that is not finite comes from an infinite or
// NaN operand or a zero or infinite divisor; those take the IEEE division,
// so that inf / y stays inf.  One multiply and two fused multiply-adds in
// place of an IEEE division wherever the reciprocal is shared.
__device__ __forceinline__ double div_rcp(double x, double y, double yr)
{
    const double q = __dmul_rn(x, yr);
    const double r = __fma_rn(-q, y, x);
    if (r == 0.0) return q;
    if (!isfinite(r)) return x / y;
    return __fma_rn(r, yr, q);
}

// x / rho_j: in FP64 the IEEE quotient from the stored reciprocal of rho_j
// (div_rcp), in the FP32 bulk form a plain division
__device__ __forceinline__ double div_rho(double x, double rj, double rrj) { return div_rcp(x, rj, rrj); }
__device__ __forceinline__ float div_rho(float x, float rj, double) { return x / rj; }

// Kernel value and gradient of pair (i, j) exactly as partisearching stored
// them: weight() / weight2() (CPP_3-NNPS.cpp:17-82) with the same
// differences, summation order and sqrt, recomputed from this step's
// positions.  w[0..2] gradient, w[3] value.  In FP64 the quotients by ra
// (rra = RN(1 / h_i) when h_j = h_i), by ra * dst (one reciprocal for the
// components) and by 6 are taken with div_rcp, which gives the IEEE
// quotients.  In FP32 the gradient's common factor is divided once per pair
// instead of once per component.
template <int ND, typename R>
__device__ __forceinline__ void pair_w_raw(const Dev& d, const PairI<R>& I, R rra, const Pos& pj, R w[4])
{
    constexpr int nd = ND;
    constexpr bool f32 = sizeof(R) == 4;
    const double xj[3] = {pj.x, pj.y, pj.z};
    R dx[3] = {R(0), R(0), R(0)}, dst = R(0);
    for (int k = 0; k < nd; k++) {
        const R t = (R)(I.x[k] - xj[k]);
        dst = dst + t * t;
        dx[k] = t;
    }
    dst = sqrt(dst);
    const R hj = (R)pj.h;
    const bool same_h = (hj == I.h);
    const R ra = same_h ? I.h : (I.h + hj) / 2;
    const R a1 = same_h ? I.a1 : kernel_a1<R>(ra, nd, d.p.flknl);
    R s;
    if (!f32 && same_h) s = (R)div_rcp(dst, ra, rra);
    else s = dst / ra;
    // the gradient's quotients by ra * dst
    const R D = ra * dst;
    // RN(1 / D): the correctly rounded reciprocal, the value of the IEEE
    // quotient 1.0 / D, without the general division's scaling steps
    R rD = R(0);
    if constexpr (sizeof(R) == 8) rD = __drcp_rn(D);
    auto grad = [&](R num) -> R { return f32 ? num / D : (R)div_rcp(num, D, rD); };
    w[0] = w[1] = w[2] = w[3] = R(0);
    if (d.p.flknl == 1 || d.p.flknl == 3) {
        if (s == R(0)) {
            w[3] = a1 * (R(0.66666667) - s * s + R(0.5) * s * s * s);
        }
        if (s > R(0) && s <= R(1)) {
            if (f32) {
                const R g = a1 * (-2 * s + R(1.5) * s * s) / D;
                for (int k = 0; k < nd; k++) w[k] = dx[k] * g;
            } else {
                for (int k = 0; k < nd; k++) w[k] = grad(a1 * dx[k] * (-2 * s + R(1.5) * s * s));
            }
            w[3] = a1 * (R(0.66666667) - s * s + R(0.5) * s * s * s);
        } else if (s > R(1) && s <= R(2)) {
            if (f32) {
                const R g = a1 * R(-0.5) * (R(2.0) - s) * (R(2.0) - s) / D;
                for (int k = 0; k < nd; k++) w[k] = dx[k] * g;
                w[3] = a1 * (R(2.0) - s) * (R(2.0) - s) * (R(2.0) - s) / R(6.0);
            } else {
                for (int k = 0; k < nd; k++) w[k] = grad(a1 * R(-0.5) * dx[k] * (R(2.0) - s) * (R(2.0) - s));
                constexpr double r6 = 1.0 / 6.0;
                w[3] = (R)div_rcp(a1 * (R(2.0) - s) * (R(2.0) - s) * (R(2.0) - s), 6.0, r6);
            }
        }
    } else {
        if (s == R(0)) {
            w[3] = a1 * (R(6.0) - R(6.0) * s + R(1.0) * s * s * s);
        }
        if (s > R(0) && s <= R(1)) {
            if (f32) {
                const R g = a1 * (R(-6.0) + R(3.0) * s * s) / D;
                for (int k = 0; k < nd; k++) w[k] = dx[k] * g;
            } else {
                for (int k = 0; k < nd; k++) w[k] = grad(a1 * dx[k] * (R(-6.0) + R(3.0) * s * s));
            }
            w[3] = a1 * (R(6.0) - R(6.0) * s + R(1.0) * s * s * s);
        } else if (s > R(1) && s <= R(2)) {
            if (f32) {
                const R g = a1 * R(-3.0) * (R(2.0) - s) * (R(2.0) - s) / D;
                for (int k = 0; k < nd; k++) w[k] = dx[k] * g;
            } else {
                for (int k = 0; k < nd; k++) w[k] = grad(a1 * R(-3.0) * dx[k] * (R(2.0) - s) * (R(2.0) - s));
            }
            w[3] = a1 * (R(2.0) - s) * (R(2.0) - s) * (R(2.0) - s);
        }
    }
}

// The virtual velocity component k of wall particle j seen by particle i of
// type ti (CPP_6-density.cpp:89-121, CPP_7-1-strain.cpp:92-124): i's own
// velocity with flbndy 1, the wall's per-phase velocity of tm_boundary with
// flbndy 2/3/4/13/14, zero otherwise.
__device__ __forceinline__ double wall_vel(const Dev& d, int ti, int j, const double vi[3], int k)
{
    const int bt = d.p.flbndy;
    if (bt == 1) return vi[k];
    if ((bt == 2 || bt == 3 || bt == 4 || bt == 13 || bt == 14) && ti >= 1 && ti <= 4)
        return d.s.vb[(size_t)((ti - 1) * 3 + k) * d.p.N + j];
    return 0.0;
}

// The stored pair record of slot s of particle i: kernel gradient w[0..2] and
// value w[3], as partisearching stores Par_Cell::wij (CPP_3-NNPS.cpp:339-345),
// corrected in place by kernel_gradient_correction when flknl is 3 or 4.
__device__ __forceinline__ void load_w_raw(const double* nbw, int N, int s, int i, double w[4])
{
    const double2* p = reinterpret_cast<const double2*>(nbw) + 2 * ((size_t)s * N + i);
    const double2 a = p[0], b = p[1];
    w[0] = a.x; w[1] = a.y; w[2] = b.x; w[3] = b.y;
}
__device__ __forceinline__ void load_w_raw(const double* nbw, int N, int s, int i, float w[4])
{
    const float4 f = reinterpret_cast<const float4*>(nbw)[(size_t)s * N + i];
    w[0] = f.x; w[1] = f.y; w[2] = f.z; w[3] = f.w;
}
__device__ __forceinline__ void load_w(const Dev& d, int s, int i, double w[4]) { load_w_raw(d.s.nbw, d.p.N, s, i, w); }
__device__ __forceinline__ void load_w(const Dev& d, int s, int i, float w[4]) { load_w_raw(d.s.nbw, d.p.N, s, i, w); }
// Slot s's pair record for a pass that needs only the kernel value w[3]:
// with no kernel gradient correction (flknl 1, 2) recomputed from the
// neighbour's position exactly as k_pairw computed it (the same operations on
// the same values, so the same bits; the gradient's arithmetic, unused, is
// dropped by the compiler), else the corrected record k_kgc left in nbw.
template <int ND, typename R>
__device__ __forceinline__ void pair_value(const Dev& d, const PairI<R>& I, R rra, int j, int s, int i, R w[4])
{
    if (d.p.flknl <= 2) pair_w_raw<ND, R>(d, I, rra, load_pos(d.s.xh, j), w);
    else load_w(d, s, i, w);
}

__device__ __forceinline__ void store_w(const Dev& d, int s, int i, const double w[4])
{
    double2* p = reinterpret_cast<double2*>(d.s.nbw) + 2 * ((size_t)s * d.p.N + i);
    p[0] = make_double2(w[0], w[1]);
    p[1] = make_double2(w[2], w[3]);
}
__device__ __forceinline__ void store_w(const Dev& d, int s, int i, const float w[4])
{
    reinterpret_cast<float4*>(d.s.nbw)[(size_t)s * d.p.N + i] = make_float4(w[0], w[1], w[2], w[3]);
}

// x^7 rounded to nearest from a double-double product chain (Dekker's exact
// product via fma; relative error of the chain below 2^-100), so the result
// is the correctly rounded power except when x^7 lies within ~2^-48 ulp of a
// rounding midpoint.  Stands in for the reference's pow(x, 7.0) in the
// equation of state (CPP_7-1-eos_CR.cpp:28,40).
struct dd { double h, l; };
__device__ __forceinline__ dd dd_mul(dd a, dd b)
{
    double p = a.h * b.h;
    double e = fma(a.h, b.h, -p);
    e = e + (a.h * b.l + a.l * b.h);
    double s = p + e;
    double t = e - (s - p);
    return dd{s, t};
}
__device__ __forceinline__ double pow7(double x)
{
    dd x1{x, 0.0};
    dd x2 = dd_mul(x1, x1);
    dd x4 = dd_mul(x2, x2);
    dd x6 = dd_mul(x4, x2);
    dd x7 = dd_mul(x6, x1);
    return x7.h + x7.l;
}
