// sph_device.cuh -- device state and per-pair helpers of the sm_100a SPH step.
//
// Layout in HBM (all particle arrays indexed by the reference particle index
// i, i.e. the order of the caller's Particle array):
//   * scalars:   T a[N]
//   * vectors:   double a[3 * N], component k of particle i at a[k * N + i]
//   * tensors:   double a[6 * N] (Voigt order xx yy zz xy yz zx, as
//                Particle::sig), component k at a[k * N + i]
//   * neighbour lists: int nbr[SPH_NB_CAP * N], slot s of particle i at
//                nbr[s * N + i] (reference index of the neighbour), so that
//                the threads of a warp read consecutive words per slot.
// Component-major storage makes every per-particle load of one component a
// coalesced 8-byte-per-lane access.
//
// Arithmetic follows the reference's operation order; the library is built
// with -fmad=false so no multiply-add is contracted, which keeps the FP64
// results identical to the reference's x86-64 build (no FMA).
#pragma once
#include <cstdint>

#define SPH_NB_CAP 99          // Par_Cell::influ[100], slots 1..99 (Class_NNPS.h:71)
#define SPH_ERR_CELL 3         // parttocell, CPP_3-NNPS.cpp:247-257
#define SPH_ERR_NEIGH 5        // partisearching, CPP_3-NNPS.cpp:313-319

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
};

struct DevState {
    // static per particle
    int *type, *matype, *etype, *permtype;
    double *mass, *hl, *cd;
    // fluid material record (pVFluid) used by the step
    double *f_dens, *f_por, *f_vpu, *f_vis, *f_c, *f_smin, *f_tanfai;
    int *f_bhtype;
    // soil material record (pParti_ConsPara) used by the step
    double *s_e, *s_poi, *s_eps0, *s_dens, *s_kapa, *s_por, *s_vpu, *s_cop, *s_sitas, *s_sitar;
    double *s_yalf, *s_ykap, *s_yalf_dil;   // Drucker-Prager constants, host-evaluated
    // dynamic state
    double *xp, *xp_next;      // 3N each, swapped every step
    double *vx, *vx_next;      // 3N each, swapped every step
    double *vxp, *axp, *ax, *ux, *x;
    double *rho, *rho_c, *rhop, *pre, *prep, *porosity, *poro_cop, *e;
    double *sig, *sig_next;    // 6N each, swapped every step
    double *eps, *adps;
    double *satu, *cop, *prew, *prea;
    double *interf, *interfss, *strep;
    double *vsig, *veps, *divq, *divr, *meps;
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

// ---------------------------------------------------------------------------
// per-pair kernel value and gradient: weight() / weight2(),
// CPP_3-NNPS.cpp:17-82.  w[0..2] gradient, w[3] value.
__device__ __forceinline__ void sph_weight(double dst, double ra, const double dx[3], double w[4],
                                           int ndim, int flknl)
{
    double a1, s;
    s = dst / ra;
    a1 = 0.0;
    w[0] = w[1] = w[2] = w[3] = 0.0;
    if (flknl == 1 || flknl == 3) {
        if (ndim == 2) a1 = 0.682092613250980 / ra / ra;
        else a1 = 0.477464829275686 / ra / ra / ra;
        if (s == 0.0) {
            w[3] = a1 * (0.66666667 - s * s + 0.5 * s * s * s);
        }
        if (s > 0.0 && s <= 1.0) {
            for (int k = 0; k < ndim; k++) w[k] = a1 * dx[k] * (-2 * s + 1.5 * s * s) / (ra * dst);
            w[3] = a1 * (0.66666667 - s * s + 0.5 * s * s * s);
        } else if (s > 1.0 && s <= 2.0) {
            for (int k = 0; k < ndim; k++) w[k] = a1 * (-0.5) * dx[k] * (2.0 - s) * (2.0 - s) / (ra * dst);
            w[3] = a1 * (2.0 - s) * (2.0 - s) * (2.0 - s) / 6.0;
        }
    } else {
        if (ndim == 2) a1 = 0.106103295394597 / (ra * ra);
        else a1 = 0.077010456334788 / (ra * ra * ra);
        if (s == 0.0) {
            w[3] = a1 * (6.0 - 6.0 * s + 1.0 * s * s * s);
        }
        if (s > 0.0 && s <= 1.0) {
            for (int k = 0; k < ndim; k++) w[k] = a1 * dx[k] * (-6.0 + 3.0 * s * s) / (ra * dst);
            w[3] = a1 * (6.0 - 6.0 * s + 1.0 * s * s * s);
        } else if (s > 1.0 && s <= 2.0) {
            for (int k = 0; k < ndim; k++) w[k] = a1 * (-3.0) * dx[k] * (2.0 - s) * (2.0 - s) / (ra * dst);
            w[3] = a1 * (2.0 - s) * (2.0 - s) * (2.0 - s);
        }
    }
}

// The kernel values of pair (i, j) exactly as partisearching stored them
// (same differences, same summation order, same sqrt), recomputed from the
// positions of this step instead of being stored per pair.
__device__ __forceinline__ void sph_pair_w(const Dev& d, int i, int j, double w[4])
{
    const int N = d.p.N, nd = d.p.ndim;
    double dx[3] = {0.0, 0.0, 0.0}, dst = 0.0;
    for (int k = 0; k < nd; k++) {
        double xi = d.s.xp[k * N + i], xj = d.s.xp[k * N + j];
        dst = dst + (xi - xj) * (xi - xj);
        dx[k] = xi - xj;
    }
    dst = sqrt(dst);
    double ra = (d.s.hl[i] + d.s.hl[j]) / 2;
    sph_weight(dst, ra, dx, w, nd, d.p.flknl);
}

// x^7 rounded to nearest from a double-double product chain (Dekker's exact
// product via fma; relative error of the chain below 2^-100), so the result
// is the correctly rounded power except when x^7 lies within ~2^-48 ulp of a
// rounding midpoint.  Stands in for the reference's pow(x, 7.0) in the
// equation of state (CPP_7-1-eos_CR.cpp:28,40), whose libm result is the
// correctly rounded value on the same inputs (checked on the CPU in tests).
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
