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
//                words per slot.
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
#define SPHK_NSTAGES 18        // entries of sphk_stage_names (one event bracket each)

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
    // positions (x, y, z, h) records, ping-pong
    double *xh, *xh_next;
    double *xs;                // xh in cell-sorted order (NNPS scan)
    // dynamic state
    double *vx, *vx_next;      // vx: velocity after the step; vx_next: before XSPH
    double *vxp, *axp, *ax, *ux;
    double *rho, *rho_c, *rhop, *pre, *prep, *porosity, *poro_cop, *e;
    double *sig, *sig_next;    // 6N each, ping-pong
    double *eps, *adps;
    double *satu, *cop, *prew, *prea;
    double *interf, *interfss, *strep;
    double *vsig, *veps, *divq, *divr, *meps;
    // per-step intermediates
    double *de;                // strain rate, 6N
    double *we;                // spin, off-diagonal entries (0,1)(0,2)(1,0)(1,2)(2,0)(2,1): 6N
    double *color;             // free-surface colour sum
    double *sr;                // stress / rho^2 as the momentum pass uses it, 6N
    double *pp;                // pore-pressure term / rho^2, N
    double *eps_in;            // strain the constitutive pass starts from: eps, or eps_tmp after strain_regu
    double *eps_tmp, *sig_tmp; // outputs of the regularisation passes, 6N each
    double *lmat;              // inverse CSPM matrix per soil/structure particle, 9N (flknl 3/4)
    double *rij;               // artificial stress tensor R per soil particle, 9N row-major (art_stre_coe > 0)
    // NNPS
    int *cell;                 // cell id per particle
    uint32_t *key_in, *key_out;
    int *val_in, *pid_sorted;
    int *cstart, *cend;        // [ctotal + 4]
    int *nnb;                  // neighbour count (may exceed the cap: error 5)
    int *nbr;                  // [SPH_NB_CAP * N]
    // control words
    int *err;                  // first error code raised (0 = none)
    int *step;                 // Para_Pro::l of the step being run
};

struct Dev {
    DevParams p;
    DevState s;
};

struct Pos { double x, y, z, h; };

__device__ __forceinline__ Pos load_pos(const double* xh, int i)
{
    const double2* p = reinterpret_cast<const double2*>(xh) + 2 * (size_t)i;
    double2 a = p[0], b = p[1];
    return Pos{a.x, a.y, b.x, b.y};
}

__device__ __forceinline__ void store_pos(double* xh, int i, const Pos& q)
{
    double2* p = reinterpret_cast<double2*>(xh) + 2 * (size_t)i;
    p[0] = make_double2(q.x, q.y);
    p[1] = make_double2(q.z, q.h);
}

// the normalisation constant a1 of weight() / weight2() for support ra
// (CPP_3-NNPS.cpp:24-29, 58-63)
__device__ __forceinline__ double kernel_a1(double ra, int ndim, int flknl)
{
    if (flknl == 1 || flknl == 3)
        return (ndim == 2) ? 0.682092613250980 / ra / ra : 0.477464829275686 / ra / ra / ra;
    return (ndim == 2) ? 0.106103295394597 / (ra * ra) : 0.077010456334788 / (ra * ra * ra);
}

// Particle i's side of every pair: position, h and a1 for ra = h_i (the
// reference's ra = (h_i + h_j) / 2 equals h_i exactly when h_j == h_i).
struct PairI {
    double x[3];
    double h, a1;
    bool corr;                 // kernel gradient correction applies (flknl 3/4, soil or structure)
    double L[9];               // its inverse CSPM matrix, row-major
};

template <int ND, int KGC>
__device__ __forceinline__ PairI pair_i(const Dev& d, int i)
{
    Pos q = load_pos(d.s.xh, i);
    PairI I;
    I.x[0] = q.x; I.x[1] = q.y; I.x[2] = q.z; I.h = q.h;
    I.a1 = kernel_a1(q.h, ND, d.p.flknl);
    I.corr = false;
    if (KGC) {
        const int t = d.s.type[i];
        I.corr = (t == 2 || t == 4);
        for (int k = 0; k < 9; k++) I.L[k] = I.corr ? d.s.lmat[(size_t)k * d.p.N + i] : 0.0;
    }
    return I;
}

// Kernel value and gradient of pair (i, j) exactly as partisearching stored
// them: weight() / weight2() (CPP_3-NNPS.cpp:17-82) with the same
// differences, summation order and sqrt, recomputed from this step's
// positions.  w[0..2] gradient, w[3] value.
template <int ND>
__device__ __forceinline__ void pair_w_raw(const Dev& d, const PairI& I, const Pos& pj, double w[4]);

// Kernel value and gradient as the consumers read them: with flknl 3/4 the
// gradient of a soil or structure particle's pairs is corrected in place by
// kernel_gradient_correction (CPP_3-NNPS.cpp:464-493): grad' = L^-1 grad,
// in mat_multiply's order (:85-90).
template <int ND, int KGC>
__device__ __forceinline__ void pair_w(const Dev& d, const PairI& I, const Pos& pj, double w[4])
{
    pair_w_raw<ND>(d, I, pj, w);
    if (KGC && I.corr) {
        const double* a = I.L;
        double c0 = a[0] * w[0] + a[1] * w[1] + a[2] * w[2];
        double c1 = a[3] * w[0] + a[4] * w[1] + a[5] * w[2];
        double c2 = a[6] * w[0] + a[7] * w[1] + a[8] * w[2];
        w[0] = c0; w[1] = c1; w[2] = c2;
    }
}

template <int ND>
__device__ __forceinline__ void pair_w_raw(const Dev& d, const PairI& I, const Pos& pj, double w[4])
{
    constexpr int nd = ND;
    const double xj[3] = {pj.x, pj.y, pj.z};
    double dx[3] = {0.0, 0.0, 0.0}, dst = 0.0;
    for (int k = 0; k < nd; k++) {
        dst = dst + (I.x[k] - xj[k]) * (I.x[k] - xj[k]);
        dx[k] = I.x[k] - xj[k];
    }
    dst = sqrt(dst);
    const double ra = (pj.h == I.h) ? I.h : (I.h + pj.h) / 2;
    const double a1 = (pj.h == I.h) ? I.a1 : kernel_a1(ra, nd, d.p.flknl);
    const double s = dst / ra;
    w[0] = w[1] = w[2] = w[3] = 0.0;
    if (d.p.flknl == 1 || d.p.flknl == 3) {
        if (s == 0.0) {
            w[3] = a1 * (0.66666667 - s * s + 0.5 * s * s * s);
        }
        if (s > 0.0 && s <= 1.0) {
            for (int k = 0; k < nd; k++) w[k] = a1 * dx[k] * (-2 * s + 1.5 * s * s) / (ra * dst);
            w[3] = a1 * (0.66666667 - s * s + 0.5 * s * s * s);
        } else if (s > 1.0 && s <= 2.0) {
            for (int k = 0; k < nd; k++) w[k] = a1 * (-0.5) * dx[k] * (2.0 - s) * (2.0 - s) / (ra * dst);
            w[3] = a1 * (2.0 - s) * (2.0 - s) * (2.0 - s) / 6.0;
        }
    } else {
        if (s == 0.0) {
            w[3] = a1 * (6.0 - 6.0 * s + 1.0 * s * s * s);
        }
        if (s > 0.0 && s <= 1.0) {
            for (int k = 0; k < nd; k++) w[k] = a1 * dx[k] * (-6.0 + 3.0 * s * s) / (ra * dst);
            w[3] = a1 * (6.0 - 6.0 * s + 1.0 * s * s * s);
        } else if (s > 1.0 && s <= 2.0) {
            for (int k = 0; k < nd; k++) w[k] = a1 * (-3.0) * dx[k] * (2.0 - s) * (2.0 - s) / (ra * dst);
            w[3] = a1 * (2.0 - s) * (2.0 - s) * (2.0 - s);
        }
    }
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
