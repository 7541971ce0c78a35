/*
 * sph_oracle.c -- CPU restatement (checker) of the reference's per-step
 * particle loop.  TEST INFRASTRUCTURE ONLY: see sph_oracle.h.
 *
 * Every function below names the reference function and file:line range it
 * restates.  Arithmetic is written in the reference's operation order so that
 * a build with the same compiler settings (no FMA contraction, no fast-math)
 * reproduces the reference bit for bit; the Jacobi/in-place switch is the one
 * intended difference (sph_oracle.h).
 */
#include "sph_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NB 100               /* Par_Cell::influ[100], wij[100][4] (Class_NNPS.h:71-72) */

struct orc_ctx {
    sphgpu_params P;
    int n, l, mode, pow_mode;
    double t;
    /* Particle members (Class_particle.h:13-103), particle-major */
    double *x, *xp, *vx, *vxp, *ax, *axp, *ux, *strep, *divx, *interf, *interfss;
    double *rho, *rhop, *mass, *hl, *pre, *prep, *e;
    double *eps, *deps, *sig, *dsig, *weps, *adps, *tssig, *tsqc;
    double *satu, *dsatu, *suct, *cop, *vsig, *veps, *divq, *divr, *meps;
    double *prew, *prea, *porosity, *cd, *poro_cop, *beta, *beta_ts;
    int *type, *matype, *permtype, *etype;
    /* cl_bndy_pair::vel_bndy and clVar_Boundary::vx_* (Class_particle.h:172-207),
     * the wall virtual velocities of flbndy 2 */
    double *vel_bndy, *vb_water, *vb_soil, *vb_air, *vb_struct;
    /* clVar_Boundary::sig_* (flbndy 3/4/13/14) */
    double *sb_water, *sb_soil, *sb_air, *sb_struct;
    /* clInterf_SS of the one thread (f_n, f_t) of the soil-structure contact */
    double *ss_fn, *ss_ft;
    /* per-particle material records (pVFluid, pParti_ConsPara) */
    sphgpu_fluid* fl;
    sphgpu_soil* so;
    /* NNPS (Class_NNPS.h) */
    int k, size_m;
    int *pc_cell_id, *ninflu, *influ;   /* Par_Cell */
    double* wij;
    int *srt_cell, *srt_pid, *tmp_cell, *tmp_pid;   /* parti_cellid sorted / temp */
    int *ci_start, *ci_end;             /* cell_info[ctotal + 4] */
    /* scratch */
    double* vx_temp;
    double* snap;                        /* Jacobi snapshots */
    double* rij;                         /* clRaij per particle (9), persistent */
    /* rainfall (flr == 1): Para_Rain and rainini's lp / vrain */
    sphgpu_rain rain;
    int rain_set, lp;
    double vrain;
    /* vibration (flv 1, 2): Para_Vibra, and StiffMat::depp0's largest
     * diagonal entry (the only part soil_damping_vibration reads) */
    double vib_ttime, vib_sttime, vib_edtime;
    int vib_nsteps, vib_set;
    double* vib_loads;
    double* stiff;
};

/* ------------------------------------------------------------------------- */
/* field table                                                               */

typedef struct { const char* name; int ncomp; int is_int; size_t off; } field_desc;

#define FD(nm, nc) { #nm, nc, 0, offsetof(struct orc_ctx, nm) }
#define FI(nm) { #nm, 1, 1, offsetof(struct orc_ctx, nm) }
static const field_desc k_fields[] = {
    FD(x, 3), FD(xp, 3), FD(vx, 3), FD(vxp, 3), FD(ax, 3), FD(axp, 3), FD(ux, 3),
    FD(strep, 3), FD(divx, 9), FD(interf, 3), FD(interfss, 3),
    FD(rho, 1), FD(rhop, 1), FD(mass, 1), FD(hl, 1), FD(pre, 1), FD(prep, 1), FD(e, 1),
    FD(eps, 6), FD(deps, 6), FD(sig, 6), FD(dsig, 6), FD(weps, 9), FD(adps, 6), FD(tssig, 6), FD(tsqc, 1),
    FD(satu, 1), FD(dsatu, 1), FD(suct, 1), FD(cop, 1), FD(vsig, 1), FD(veps, 1),
    FD(divq, 1), FD(divr, 1), FD(meps, 1), FD(prew, 1), FD(prea, 1), FD(porosity, 1),
    FD(cd, 1), FD(poro_cop, 1), FD(beta, 9), FD(beta_ts, 9),
    FI(type), FI(matype), FI(permtype), FI(etype),
    FD(vel_bndy, 3), FD(vb_water, 3), FD(vb_soil, 3), FD(vb_air, 3), FD(vb_struct, 3),
    FD(ss_fn, 3), FD(ss_ft, 3),
    FD(sb_water, 6), FD(sb_soil, 6), FD(sb_air, 6), FD(sb_struct, 6),
};
#define NFIELDS (sizeof(k_fields) / sizeof(k_fields[0]))

static const field_desc* find_field(const char* name)
{
    for (size_t i = 0; i < NFIELDS; i++)
        if (strcmp(k_fields[i].name, name) == 0) return &k_fields[i];
    return NULL;
}

orc_ctx* orc_create(const sphgpu_params* p)
{
    if (!p || p->ntotal <= 0) return NULL;
    orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
    c->P = *p;
    c->n = p->ntotal;
    c->l = 1;   /* Para_Pro::l starts at 1 (Class_Problem.cpp:66) */
    c->mode = ORC_JACOBI;
    int n = c->n;
    for (size_t f = 0; f < NFIELDS; f++) {
        void** slot = (void**)((char*)c + k_fields[f].off);
        *slot = calloc((size_t)n * k_fields[f].ncomp, k_fields[f].is_int ? sizeof(int) : sizeof(double));
    }
    c->fl = (sphgpu_fluid*)calloc(n, sizeof(sphgpu_fluid));
    c->so = (sphgpu_soil*)calloc(n, sizeof(sphgpu_soil));
    c->stiff = (double*)calloc(n, sizeof(double));      /* StiffMat(): depp0 = 0 (Class_particle.cpp:220-228) */
    for (int i = 0; i < n; i++) {
        c->fl[i].strain_min = 1.0;   /* Para_Fluid() (Class_ParticleProperty.cpp) */
        c->so[i].fs = 1.0;            /* Para_Soil()  */
        c->so[i].ds = 1.0;
    }
    /* allocation sizes of SPH_Calculation (CPP_1-SPHLoops.cpp:355-376) */
    c->k = (int)log2((double)n) + 1;
    c->size_m = 1 << c->k;
    c->pc_cell_id = (int*)malloc(sizeof(int) * n);
    for (int i = 0; i < n; i++) c->pc_cell_id[i] = -1;
    c->ninflu = (int*)calloc(n, sizeof(int));
    c->influ = (int*)calloc((size_t)n * NB, sizeof(int));
    c->wij = (double*)calloc((size_t)n * NB * 4, sizeof(double));
    c->srt_cell = (int*)malloc(sizeof(int) * c->size_m);
    c->srt_pid = (int*)malloc(sizeof(int) * c->size_m);
    c->tmp_cell = (int*)malloc(sizeof(int) * c->size_m);
    c->tmp_pid = (int*)malloc(sizeof(int) * c->size_m);
    for (int i = 0; i < c->size_m; i++) {   /* parti_cellid() (Class_NNPS.cpp:48-52) */
        c->srt_cell[i] = 10000000; c->srt_pid[i] = 10000000;
        c->tmp_cell[i] = 10000000; c->tmp_pid[i] = 10000000;
    }
    int nc = p->ctotal + 4;
    c->ci_start = (int*)malloc(sizeof(int) * nc);
    c->ci_end = (int*)malloc(sizeof(int) * nc);
    for (int i = 0; i < nc; i++) { c->ci_start[i] = 2000000; c->ci_end[i] = -2000000; } /* cell_info() */
    c->vx_temp = (double*)calloc((size_t)n * 3, sizeof(double));
    c->snap = (double*)calloc((size_t)n * 6, sizeof(double));
    c->rij = (double*)calloc((size_t)n * 9, sizeof(double));   /* clRaij() zeroes Rij */
    return c;
}

void orc_destroy(orc_ctx* c)
{
    if (!c) return;
    for (size_t f = 0; f < NFIELDS; f++) free(*(void**)((char*)c + k_fields[f].off));
    free(c->fl); free(c->so); free(c->stiff); free(c->vib_loads); free(c->pc_cell_id); free(c->ninflu); free(c->influ); free(c->wij);
    free(c->srt_cell); free(c->srt_pid); free(c->tmp_cell); free(c->tmp_pid);
    free(c->ci_start); free(c->ci_end); free(c->vx_temp); free(c->snap); free(c->rij);
    free(c);
}

int orc_set_field(orc_ctx* c, const char* name, const void* host, size_t count)
{
    const field_desc* f = find_field(name);
    if (!f || !host) return SPHGPU_E_ARG;
    size_t want = (size_t)c->n * f->ncomp;
    if (count != want) return SPHGPU_E_ARG;
    memcpy(*(void**)((char*)c + f->off), host, want * (f->is_int ? sizeof(int) : sizeof(double)));
    return 0;
}

int orc_get_field(orc_ctx* c, const char* name, void* host, size_t count)
{
    const field_desc* f = find_field(name);
    if (!f || !host) return SPHGPU_E_ARG;
    size_t want = (size_t)c->n * f->ncomp;
    if (count != want) return SPHGPU_E_ARG;
    memcpy(host, *(void**)((char*)c + f->off), want * (f->is_int ? sizeof(int) : sizeof(double)));
    return 0;
}

int orc_set_materials(orc_ctx* c, const sphgpu_fluid* fluid, const sphgpu_soil* soil, int n)
{
    if (n != c->n) return SPHGPU_E_ARG;
    if (fluid) memcpy(c->fl, fluid, sizeof(sphgpu_fluid) * n);
    if (soil) memcpy(c->so, soil, sizeof(sphgpu_soil) * n);
    return 0;
}

void orc_set_mode(orc_ctx* c, int mode) { c->mode = mode; }
void orc_set_pow_mode(orc_ctx* c, int pow_mode) { c->pow_mode = pow_mode; }

/* x^7 from Dekker products (fma gives each product's exact error term); the
 * double-double chain carries ~100 bits, so the final sum is the correctly
 * rounded x^7 unless x^7 sits within ~2^-48 ulp of a rounding midpoint. */
typedef struct { double h, l; } orc_dd;
static orc_dd orc_dd_mul(orc_dd a, orc_dd b)
{
    double p = a.h * b.h;
    double e = fma(a.h, b.h, -p);
    e = e + (a.h * b.l + a.l * b.h);
    double s = p + e;
    orc_dd r = {s, e - (s - p)};
    return r;
}
double orc_pow7(double x)
{
    orc_dd x1 = {x, 0.0};
    orc_dd x2 = orc_dd_mul(x1, x1);
    orc_dd x4 = orc_dd_mul(x2, x2);
    orc_dd x6 = orc_dd_mul(x4, x2);
    orc_dd x7 = orc_dd_mul(x6, x1);
    return x7.h + x7.l;
}
static double eos_pow7(const orc_ctx* c, double x)
{
    return c->pow_mode == ORC_POW_CR ? orc_pow7(x) : pow(x, 7.0);
}
int orc_get_step(const orc_ctx* c) { return c->l; }

/* ------------------------------------------------------------------------- */
/* NNPS                                                                       */

/* weight(): cubic B-spline value and gradient, CPP_3-NNPS.cpp:17-48 */
static void weight(double dst, double ra, const double dx[], double* w1ij, int ndim)
{
    double a1, s;
    int k;
    s = dst / ra;
    a1 = 0.0;
    if (ndim == 2) {
        a1 = 0.682092613250980 / ra / ra;
        w1ij[ndim] = 0.0;
    }
    if (ndim == 3) a1 = 0.477464829275686 / ra / ra / ra;
    if (s == 0.0) {
        for (k = 0; k < ndim; k++) w1ij[k] = 0.0;
        w1ij[3] = a1 * (0.66666667 - s * s + 0.5 * s * s * s);
    }
    if (s > 0.0 && s <= 1.0) {
        for (k = 0; k < ndim; k++) w1ij[k] = a1 * dx[k] * (-2 * s + 1.5 * s * s) / (ra * dst);
        w1ij[3] = a1 * (0.66666667 - s * s + 0.5 * s * s * s);
    } else if (s > 1.0 && s <= 2.0) {
        for (k = 0; k < ndim; k++) w1ij[k] = a1 * (-0.5) * dx[k] * (2.0 - s) * (2.0 - s) / (ra * dst);
        w1ij[3] = a1 * (2.0 - s) * (2.0 - s) * (2.0 - s) / 6.0;
    }
}

/* weight2(): Yang & Liu kernel, CPP_3-NNPS.cpp:51-82 */
static void weight2(double dst, double ra, const double dx[], double* w1ij, int ndim)
{
    double a1, s;
    int k;
    s = dst / ra;
    a1 = 0.0;
    if (ndim == 2) {
        a1 = 0.106103295394597 / (ra * ra);
        w1ij[ndim] = 0.0;
    }
    if (ndim == 3) a1 = 0.077010456334788 / (ra * ra * ra);
    if (s == 0.0) {
        for (k = 0; k < ndim; k++) w1ij[k] = 0.0;
        w1ij[3] = a1 * (6.0 - 6.0 * s + 1.0 * s * s * s);
    }
    if (s > 0.0 && s <= 1.0) {
        for (k = 0; k < ndim; k++) w1ij[k] = a1 * dx[k] * (-6.0 + 3.0 * s * s) / (ra * dst);
        w1ij[3] = a1 * (6.0 - 6.0 * s + 1.0 * s * s * s);
    } else if (s > 1.0 && s <= 2.0) {
        for (k = 0; k < ndim; k++) w1ij[k] = a1 * (-3.0) * dx[k] * (2.0 - s) * (2.0 - s) / (ra * dst);
        w1ij[3] = a1 * (2.0 - s) * (2.0 - s) * (2.0 - s);
    }
}

/* cell_link entries, celllist_ini2 (CPP_3-NNPS.cpp:124-171): stencil slot p of
 * cell i, 0 when outside [0, m]. */
static int cell_link(const sphgpu_params* P, int i, int p)
{
    int m = P->ctotal, v;
    if (P->ndim == 2) {
        int ky = p / 3 + 1, kx = p % 3 + 1;
        v = (kx - 2) * P->cym + ky - 2 + i;
    } else {
        int kz = p / 9 + 1, kx = (p / 3) % 3 + 1, ky = p % 3 + 1;
        v = (ky - 2) * P->cxm * P->czm + (kx - 2) * P->czm + kz - 2 + i;
    }
    if (v < 0 || v > m) v = 0;
    return v;
}

/* Merge_CellID: CPP_3-NNPS.cpp:561-594 (right element taken on equal keys) */
static void merge_cells(orc_ctx* c, int start, int mid, int end)
{
    int i, j, k;
    for (i = start; i <= end; i++) { c->tmp_cell[i] = c->srt_cell[i]; c->tmp_pid[i] = c->srt_pid[i]; }
    i = start; j = mid + 1; k = start;
    while (i < mid + 1 && j <= end) {
        if (c->tmp_cell[i] < c->tmp_cell[j]) { c->srt_cell[k] = c->tmp_cell[i]; c->srt_pid[k++] = c->tmp_pid[i++]; }
        else { c->srt_cell[k] = c->tmp_cell[j]; c->srt_pid[k++] = c->tmp_pid[j++]; }
    }
    while (i < mid + 1) { c->srt_cell[k] = c->tmp_cell[i]; c->srt_pid[k++] = c->tmp_pid[i++]; }
    while (j <= end) { c->srt_cell[k] = c->tmp_cell[j]; c->srt_pid[k++] = c->tmp_pid[j++]; }
}

/* Binary_Sort: bottom-up merge passes and the cell_info scan,
 * CPP_3-NNPS.cpp:597-630 */
static void binary_sort(orc_ctx* c)
{
    for (int i_k = 1; i_k <= c->k; i_k++) {
        int interval = 1 << i_k;
        int group_num = c->size_m / interval;
        for (int g = 0; g < group_num; g++) {
            int start = g * interval, end = (g + 1) * interval - 1;
            merge_cells(c, start, (start + end) >> 1, end);
        }
    }
    for (int i = 0; i < c->n; i++) {
        int cid = c->srt_cell[i];
        if (i < c->ci_start[cid]) c->ci_start[cid] = i;
        if (i > c->ci_end[cid]) c->ci_end[cid] = i;
    }
}

/* parttocell: CPP_3-NNPS.cpp:175-263 */
static int parttocell(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    int m = P->ctotal, t = 0;
    double xmin[3] = {P->xmin, P->ymin, P->zmin};
    double dr = 2.0 * P->dr;
    for (int i = 0; i < m; i++) { c->ci_start[i] = 10000000; c->ci_end[i] = -10000000; }
    for (int i = 0; i < c->n; i++) {
        int nx_t[3];
        for (int j = 0; j < P->ndim; j++) {
            double nx = fabs(c->xp[i * 3 + j] - xmin[j]) / dr + 2.0;
            nx_t[j] = (int)(nx);
            if (nx_t[j] < 2) nx_t[j] = 2;
        }
        if (P->ndim == 2) c->srt_cell[i] = P->cym * (nx_t[0] - 1) + nx_t[1];
        else c->srt_cell[i] = P->cxm * P->czm * (nx_t[1] - 1) + P->czm * (nx_t[0] - 1) + nx_t[2];
        c->srt_pid[i] = i;
    }
    /* positions >= ntotal keep the padding records (10000000, 10000000) */
    for (int i = c->n; i < c->size_m; i++) { c->srt_cell[i] = 10000000; c->srt_pid[i] = 10000000; }
    for (int i = 0; i < c->n; i++) {
        if (c->srt_cell[i] > 0 && c->srt_cell[i] <= m) c->pc_cell_id[i] = c->srt_cell[i];
        else t = 3;
    }
    if (t > 0) return t;
    binary_sort(c);
    return t;
}

/* partisearching: CPP_3-NNPS.cpp:265-374 */
static int partisearching(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    int dim = P->ndim, temp = (dim == 2) ? 9 : 27, t = 0;
    for (int i = 0; i < c->n; i++) c->ninflu[i] = 0;
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] == 7) continue;
        int nc = c->pc_cell_id[i];
        for (int nj = 0; nj < temp; nj++) {
            int nl = cell_link(P, nc, nj);
            if (nl <= 0) continue;
            int start = c->ci_start[nl], end = c->ci_end[nl];
            for (int np = start; np <= end; np++) {
                int j = c->srt_pid[np];
                double dst = 0.0, dx[3];
                for (int k = 0; k < dim; k++) {
                    dst = dst + (c->xp[i * 3 + k] - c->xp[j * 3 + k]) * (c->xp[i * 3 + k] - c->xp[j * 3 + k]);
                    dx[k] = c->xp[i * 3 + k] - c->xp[j * 3 + k];
                }
                dst = sqrt(dst);
                double ra = (c->hl[i] + c->hl[j]) / 2;
                if (dst <= 2 * ra && i != j) {
                    c->ninflu[i] += 1;
                    int p = c->ninflu[i];
                    if (p <= 99) {
                        c->influ[i * NB + p] = j;
                        if (P->flknl == 1 || P->flknl == 3) weight(dst, ra, dx, &c->wij[(i * NB + p) * 4], dim);
                        else weight2(dst, ra, dx, &c->wij[(i * NB + p) * 4], dim);
                    } else
                        t = 5;
                }
            }
        }
    }
    return t;
}

#define W(i, nj, k) (c->wij[((size_t)(i) * NB + (nj)) * 4 + (k)])
#define NBR(i, nj) (c->influ[(size_t)(i) * NB + (nj)])

/* ------------------------------------------------------------------------- */
/* density: CPP_6-density.cpp:11-189                                          */
/* the virtual velocity of wall particle j seen by particle i: its own
 * velocity (flbndy 1) or the wall's clVar_Boundary velocity for i's phase
 * (flbndy 2/3/4/13/14), CPP_6-density.cpp:89-121, CPP_7-1-strain.cpp:92-124 */
static void wall_velocity(const orc_ctx* c, int i, int j, double vxj[3])
{
    const int bt = c->P.flbndy, ti = c->type[i];
    vxj[0] = vxj[1] = vxj[2] = 0.0;
    if (bt == 1) {
        for (int k = 0; k < 3; k++) vxj[k] = c->vxp[i * 3 + k];
    } else if (bt == 2 || bt == 3 || bt == 4 || bt == 13 || bt == 14) {
        const double* v = ti == 1 ? c->vb_water : ti == 2 ? c->vb_soil : ti == 3 ? c->vb_air : ti == 4 ? c->vb_struct : 0;
        if (v)
            for (int k = 0; k < 3; k++) vxj[k] = v[j * 3 + k];
    }
}

static void density(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    int n = c->n, ndim = P->ndim, l = c->l;
    double dt = P->dt;
    /* fluid porosity from soil neighbours (:25-54) */
    for (int i = 0; i < n; i++) {
        double up = 0.0, down = 0.0;
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[i] != c->type[j] && c->type[i] == 1 && c->type[j] == 2) {
                up = up + c->mass[j] * c->porosity[j] / c->rho[j] * W(i, nj, 3);
                down = down + c->mass[j] / c->rho[j] * W(i, nj, 3);
            }
        }
        if (c->type[i] == 1 && fabs(down) > 1.0e-7) {
            c->poro_cop[i] = c->porosity[i];
            c->porosity[i] = up / down;
            if (l == 1) c->poro_cop[i] = c->porosity[i];
        } else if (c->type[i] == 1 && fabs(down) <= 1.0e-7) {
            c->poro_cop[i] = c->porosity[i];
        }
    }
    /* continuity (:57-165) */
    for (int i = 0; i < n; i++) {
        double drhot = 0.0, up[3] = {0, 0, 0}, down[3] = {0, 0, 0}, vxj[3];
        int ti = c->type[i];
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), k;
            if (ti == c->type[j] && ti != 7 && ti != 0) {
                if (ti == 2 || ti == 4) {
                    for (k = 0; k < ndim; k++) {
                        up[k] = up[k] + c->mass[j] * (c->vxp[i * 3 + k] - c->vxp[j * 3 + k]) * W(i, nj, k);
                        down[k] = down[k] + c->mass[j] * (c->xp[i * 3 + k] - c->xp[j * 3 + k]) * W(i, nj, k);
                    }
                }
                if (ti == 1 || ti == 3) {
                    for (k = 0; k < ndim; k++)
                        up[k] = up[k] + c->mass[j] * (c->vxp[i * 3 + k] - c->vxp[j * 3 + k]) * W(i, nj, k);
                }
            } else if ((ti == 1 || ti == 2 || ti == 3 || ti == 4) && c->type[j] == 0) {
                wall_velocity(c, i, j, vxj);
                if (ti == 2 || ti == 4) {
                    for (k = 0; k < ndim; k++) {
                        up[k] = up[k] + c->mass[j] * (c->vxp[i * 3 + k] - vxj[k]) * W(i, nj, k);
                        down[k] = down[k] + c->mass[j] * (c->xp[i * 3 + k] - c->xp[j * 3 + k]) * W(i, nj, k);
                    }
                }
                if (ti == 1 || ti == 3) {
                    for (k = 0; k < ndim; k++)
                        up[k] = up[k] + c->mass[j] * (c->vxp[i * 3 + k] - vxj[k]) * W(i, nj, k);
                }
            }
        }
        if (ti != 7) {
            int k;
            if (ti == 2 || ti == 4) {
                for (k = 0; k < ndim; k++) {
                    if (fabs(down[k]) > 1.0e-7) drhot -= up[k] / down[k];
                    else drhot += up[k];
                }
            }
            if (ti == 1 || ti == 3)
                for (k = 0; k < ndim; k++) drhot += up[k];
            if (ti == 1) {
                if (fabs(c->porosity[i]) > 0.0001)
                    c->rho[i] = c->rhop[i] + drhot * dt + c->rhop[i] * (c->porosity[i] - c->poro_cop[i]) / (1.0 - c->poro_cop[i]);
                else
                    c->rho[i] = c->rhop[i] + drhot * dt;
            } else {
                c->rho[i] = c->rhop[i] + drhot * dt;
            }
        }
    }
    /* Shepard filter (:168-188).  Reference: in place; Jacobi: snapshot. */
    const double* rho_src = c->rho;
    if (c->mode == ORC_JACOBI) {
        memcpy(c->snap, c->rho, sizeof(double) * n);
        rho_src = c->snap;
    }
    for (int i = 0; i < n; i++) {
        double up = 0.0, down = 0.0;
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[i] == c->type[j]) {
                up = up + c->mass[j] * W(i, nj, 3);
                down = down + c->mass[j] / rho_src[j] * W(i, nj, 3);
            }
        }
        if (c->type[i] != 7 && fabs(down) > 1.0e-7) c->rho[i] = up / down;
    }
}

/* ------------------------------------------------------------------------- */
/* strain_noreg: CPP_7-1-strain.cpp:20-220                                    */
static void strain_noreg(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    int n = c->n, dim = P->ndim;
    for (int i = 0; i < n; i++) {
        double dvx[3], up[9], vxj[3], down[3];
        int j, k;
        if (c->l == P->inip)
            for (j = 0; j < 6; j++) c->eps[i * 6 + j] = 0.0;
        for (j = 0; j < 6; j++) { c->deps[i * 6 + j] = 0.0; c->dsig[i * 6 + j] = 0.0; }
        for (j = 0; j < 9; j++) { c->weps[i * 9 + j] = 0.0; c->divx[i * 9 + j] = 0.0; up[j] = 0.0; }
        for (j = 0; j < 3; j++) down[j] = 0;
        int ti = c->type[i];
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            for (k = 0; k < 3; k++) dvx[k] = 0.0;
            j = NBR(i, nj);
            int touch = 0;
            if (ti == c->type[j] && ti != 7 && ti != 0) {
                for (k = 0; k < 3; k++) dvx[k] = c->vxp[i * 3 + k] - c->vxp[j * 3 + k];
                touch = 1;
            } else if ((ti == 1 || ti == 2 || ti == 3 || ti == 4) && c->type[j] == 0) {
                wall_velocity(c, i, j, vxj);
                for (k = 0; k < 3; k++) dvx[k] = c->vxp[i * 3 + k] - vxj[k];
                touch = 1;
            }
            if (!touch) continue;
            double mr = c->mass[j];
            double rj = c->rho[j];
            up[0] = up[0] + mr / rj * dvx[0] * W(i, nj, 0);
            up[1] = up[1] + mr / rj * dvx[0] * W(i, nj, 1);
            up[2] = up[2] + mr / rj * dvx[0] * W(i, nj, 2);
            up[3] = up[3] + mr / rj * dvx[1] * W(i, nj, 0);
            up[4] = up[4] + mr / rj * dvx[1] * W(i, nj, 1);
            up[5] = up[5] + mr / rj * dvx[1] * W(i, nj, 2);
            up[6] = up[6] + mr / rj * dvx[2] * W(i, nj, 0);
            up[7] = up[7] + mr / rj * dvx[2] * W(i, nj, 1);
            up[8] = up[8] + mr / rj * dvx[2] * W(i, nj, 2);
            if (ti == 2 || ti == 4) {
                down[0] = down[0] + mr / rj * (c->xp[i * 3 + 0] - c->xp[j * 3 + 0]) * W(i, nj, 0);
                down[1] = down[1] + mr / rj * (c->xp[i * 3 + 1] - c->xp[j * 3 + 1]) * W(i, nj, 1);
                down[2] = down[2] + mr / rj * (c->xp[i * 3 + 2] - c->xp[j * 3 + 2]) * W(i, nj, 2);
            }
        }
        double* dv = &c->divx[i * 9];   /* divx[a][b] = dv[a*3+b] */
        if (ti == 1 || ti == 3) {
            dv[0] = up[0]; dv[3] = up[3]; dv[6] = up[6];
            dv[1] = up[1]; dv[4] = up[4]; dv[7] = up[7];
            dv[2] = up[2]; dv[5] = up[5]; dv[8] = up[8];
        } else {
            if (fabs(down[0]) > 1.0e-7) { dv[0] = up[0] / down[0]; dv[3] = up[3] / down[0]; dv[6] = up[6] / down[0]; }
            if (fabs(down[1]) > 1.0e-7) { dv[1] = up[1] / down[1]; dv[4] = up[4] / down[1]; dv[7] = up[7] / down[1]; }
            if (fabs(down[2]) > 1.0e-7) { dv[2] = up[2] / down[2]; dv[5] = up[5] / down[2]; dv[8] = up[8] / down[2]; }
        }
        double* de = &c->deps[i * 6];
        de[0] = dv[0];
        de[1] = dv[4];
        de[2] = dv[8];
        de[3] = dv[1] + dv[3];
        de[4] = dv[5] + dv[7];
        de[5] = dv[6] + dv[2];
        if (dim == 2) { de[2] = 0.0; de[4] = 0.0; de[5] = 0.0; }
        double* we = &c->weps[i * 9];
        we[0] = 0.0;
        we[1] = 0.5 * (dv[1] - dv[3]);
        we[2] = 0.5 * (dv[2] - dv[6]);
        we[3] = 0.5 * (dv[3] - dv[1]);
        we[4] = 0.0;
        we[5] = 0.5 * (dv[5] - dv[7]);
        we[6] = 0.5 * (dv[6] - dv[2]);
        we[7] = 0.5 * (dv[7] - dv[5]);
        we[8] = 0.0;
        if (dim == 2) { we[2] = 0.0; we[5] = 0.0; we[6] = 0.0; we[7] = 0.0; we[8] = 0.0; }
    }
}

/* Shepard smoothing of eps or sig: strain_regu / stress_regu,
 * CPP_7-2-constitutive.cpp:385-450 (in place in the reference) */
static void regularise(orc_ctx* c, double* f)
{
    int n = c->n;
    const double* src = f;
    if (c->mode == ORC_JACOBI) {
        memcpy(c->snap, f, sizeof(double) * 6 * n);
        src = c->snap;
    }
    for (int i = 0; i < n; i++) {
        double up[6] = {0, 0, 0, 0, 0, 0}, down = 0.0;
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[i] == c->type[j]) {
                for (int q = 0; q < 6; q++) up[q] = up[q] + c->mass[j] / c->rho[j] * W(i, nj, 3) * src[j * 6 + q];
                down = down + c->mass[j] / c->rho[j] * W(i, nj, 3);
            }
        }
        if (fabs(down) > 1.0e-6)
            for (int q = 0; q < 6; q++) f[i * 6 + q] = up[q] / down;
    }
}

/* cal_permeability: CPP_7-2-constitutive.cpp:355-382 (Particle::permeablel /
 * permeabletl: Class_particle.cpp:147-173) */
static void cal_permeability(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] != 2) continue;
        if (P->permtype == 0) c->cop[i] = c->so[i].cop;
        else if (P->permtype == 1) c->cop[i] = P->pers;
        else if (P->permtype == 2) {
            double sitas = c->so[i].sitas, sitar = c->so[i].sitar;
            if (c->satu[i] < sitar) c->cop[i] = P->pers;
            else if (c->satu[i] > sitas) c->cop[i] = P->perl;
            else c->cop[i] = (P->perl - P->pers) * c->satu[i] / (sitas - sitar) + P->pers;
        } else if (P->permtype == 3) {
            if (c->permtype[i] == 1) c->cop[i] = P->pers;
            if (c->permtype[i] == 2) c->cop[i] = P->perm;
            if (c->permtype[i] == 3) c->cop[i] = P->perl;
        }
    }
}

/* eos: CPP_7-1-eos_CR.cpp:12-178 */
static void eos(orc_ctx* c)
{
    int n = c->n;
    for (int i = 0; i < n; i++) {
        if (c->type[i] == 1) {
            c->pre[i] = c->prep[i] * (eos_pow7(c, c->rho[i] / c->fl[i].dens / c->fl[i].porosity) - 1.0);
            c->pre[i] = c->pre[i] + c->prep[i];
        }
        if (c->type[i] == 3) {
            /* the reference's comma expression evaluates to -1.0 (:34) */
            c->pre[i] = 1.403 * c->prep[i] * (-1.0);
            c->pre[i] = c->pre[i] + c->prep[i];
        }
        if (c->type[i] == 0 && c->matype[i] == 1) {
            c->pre[i] = c->prep[i] * (eos_pow7(c, c->rho[i] / c->rhop[i]) - 1.0);
            c->pre[i] = c->pre[i] + c->prep[i];
        }
    }
    /* the gathered pressures and wall stresses are all written after the
     * loop reads them only from other types, so one buffer suffices */
    double* sig_new = c->snap;   /* wall stresses: soil sig is read, wall sig written */
    for (int i = 0; i < n; i++) {
        double u1 = 0, u2 = 0, u3 = 0, u4 = 0, d1 = 0, d2 = 0, d3 = 0, d4 = 0, us[6] = {0, 0, 0, 0, 0, 0}, ds = 0;
        int ti = c->type[i];
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), tj = c->type[j];
            if (ti == tj) continue;
            double m = c->mass[j], w = W(i, nj, 3), r = c->rho[j];
            if (ti == 2 && tj == 1) { u1 = u1 + m * c->pre[j] * w / r; d1 = d1 + m * w / r; }
            if (ti == 2 && tj == 3) { u2 = u2 + m * c->pre[j] * w / r; d2 = d2 + m * w / r; }
            if (ti == 4 && tj == 1) { u3 = u3 + m * c->pre[j] * w / r; d3 = d3 + m * w / r; }
            if (ti == 4 && tj == 3) { u4 = u4 + m * c->pre[j] * w / r; d4 = d4 + m * w / r; }
            if (ti == 0 && tj == 1) { u1 = u1 + m * c->pre[j] * w / r; d1 = d1 + m * w / r; }
            if (ti == 0 && tj == 3) { u2 = u2 + m * c->pre[j] * w / r; d2 = d2 + m * w / r; }
            if (ti == 0 && tj == 2) {
                for (int q = 0; q < 6; q++) us[q] = us[q] + m * c->sig[j * 6 + q] * w / r;
                ds = ds + m * w / r;
            }
        }
        if (ti == 2) {
            c->prew[i] = (d1 != 0.0) ? u1 / d1 : u1;
            c->prea[i] = (d2 != 0.0) ? u2 / d2 : u2;
        } else if (ti == 0) {
            c->prew[i] = (d1 != 0.0) ? u1 / d1 : u1;
            c->prea[i] = (d2 != 0.0) ? u2 / d2 : u2;
            for (int q = 0; q < 6; q++) sig_new[i * 6 + q] = (ds != 0.0) ? us[q] / ds : us[q];
        } else if (ti == 4) {
            c->prew[i] = (d3 != 0.0) ? u3 / d3 : u3;
            c->prea[i] = (d4 != 0.0) ? u4 / d4 : u4;
        }
    }
    for (int i = 0; i < n; i++)
        if (c->type[i] == 0)
            for (int q = 0; q < 6; q++) c->sig[i * 6 + q] = sig_new[i * 6 + q];
}

/* Particle::deq, shearstrain, poro_cal, stress_adjust:
 * Class_particle.cpp:121-143, 175-215 */
static void deq(orc_ctx* c, int i)
{
    double* s = &c->sig[i * 6];
    double* ep = &c->eps[i * 6];
    c->veps[i] = ep[0] + ep[1] + ep[2];
    c->vsig[i] = (s[0] + s[1] + s[2]) / 3;
    c->divq[i] = 0.0;
    double sxx = s[0] - c->vsig[i], syy = s[1] - c->vsig[i], szz = s[2] - c->vsig[i];
    double j2 = 0.5 * (sxx * sxx + syy * syy + szz * szz) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    c->divq[i] = sqrt(3 * fabs(j2));
    if (c->vsig[i] != 0.0) c->divr[i] = fabs(c->divq[i] / c->vsig[i]);
    else c->divr[i] = 0.0;
}

static void shearstrain(orc_ctx* c, int i)
{
    double* ep = &c->eps[i * 6];
    double sxx = ep[0] - c->veps[i] / 3.0, syy = ep[1] - c->veps[i] / 3.0, szz = ep[2] - c->veps[i] / 3.0;
    double j2 = 0.5 * (sxx * sxx + syy * syy + szz * szz) + ep[3] * ep[3] + ep[4] * ep[4] + ep[5] * ep[5];
    c->meps[i] = sqrt(2.0 * fabs(j2));
}

static void poro_cal(orc_ctx* c, int i, double dt)
{
    double* de = &c->deps[i * 6];
    double d = (1 + c->e[i]) * (de[0] + de[1] + de[2]) * dt;
    double et = c->e[i] + d;
    if (et < 0.0) et = 0.0;
    c->porosity[i] = et / (1 + et);
    c->e[i] = et;
}

static void stress_adjust(orc_ctx* c, int i)
{
    if (c->vsig[i] > 0.0) {
        double temp = -c->vsig[i];
        double* s = &c->sig[i * 6];
        s[0] = s[0] + temp; s[1] = s[1] + temp; s[2] = s[2] + temp;
        s[3] = 0.0; s[4] = 0.0; s[5] = 0.0;
    }
}

/* elastic D matrix shared by elastic() / dpmodel1() / dpmodel_bui():
 * CPP_8-1-consfactor.cpp:17-59, 301-334, 468-501 */
static void elastic_d(double dept[6][6], const double* sig, const sphgpu_soil* so, double* dlam_o, double* dmu_o, double* sm_o)
{
    double sigct[6], sm, e0, dlam, dmu, dmu2;
    double poi = so->poi, eps0 = so->eps0, zkapa = so->kapa;
    for (int a = 0; a < 6; a++) {
        sigct[a] = -sig[a];
        for (int b = 0; b < 6; b++) dept[a][b] = 0.0;
    }
    sm = (sigct[0] + sigct[1] + sigct[2]) * 0.3333333333;
    if (sm < 1.0) sm = 1.0;
    if (so->e > 1.0) e0 = so->e;
    else e0 = 3 * (1 - 2 * poi) * (1 + eps0) * fabs(sm) / zkapa;
    dlam = e0 * poi / (1.0 + poi) / (1.0 - 2.0 * poi);
    dmu = e0 * 0.5 / (1.0 + poi);
    dmu2 = dmu * 2.0;
    dept[0][0] = dlam + dmu2; dept[1][1] = dlam + dmu2; dept[2][2] = dlam + dmu2;
    dept[0][1] = dlam; dept[0][2] = dlam; dept[1][0] = dlam;
    dept[1][2] = dlam; dept[2][0] = dlam; dept[2][1] = dlam;
    dept[3][3] = dmu; dept[4][4] = dmu; dept[5][5] = dmu;
    *dlam_o = dlam; *dmu_o = dmu; *sm_o = sm;
}

/* Rank-one plastic correction shared by sub_camclay and elastic_plastic:
 * dept[a][b] -= d * ww[a] * zz[b] (CPP_8-1-consfactor.cpp:228-273, 723-768) */
static void plastic_update(double dept[6][6], double d, const double ww[6], const double zz[6])
{
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) dept[a][b] = dept[a][b] - d * ww[a] * zz[b];
}

/* sub_camclay: subloading Cam-clay, CPP_8-1-consfactor.cpp:129-281 */
static void sub_camclay(double dept[6][6], const double* sig, const double* deps, const sphgpu_soil* so, double* adps)
{
    double dlam, dmu, sm;
    double ann = so->ann, zmf = so->zmf, zramda = so->ramda, zkapa = so->kapa, eps0 = so->eps0;
    elastic_d(dept, sig, so, &dlam, &dmu, &sm);
    double dmu2 = dmu * 2.0;
    double sigct[6];
    for (int a = 0; a < 6; a++) sigct[a] = -sig[a];
    double ymf = 3.0 * (zmf - 1.0) / (zmf + 2.0) / so->fs;
    double hee = (zramda - zkapa) / (1.0 + eps0);
    double dx = sigct[0] - sm, dy = sigct[1] - sm, dz = sigct[2] - sm;
    double dxy = sigct[3], dyz = sigct[4], dzx = sigct[5];
    double sjj = 0.5 * (dx * dx + dy * dy + dz * dz) + dxy * dxy + dyz * dyz + dzx * dzx;
    double tt1 = 1.0 / (ymf * ymf * sm * sm + 3.0 * sjj);
    double tt2 = 2.0 * ymf * ymf * sm * tt1 - 1.0 / sm;
    double f11 = tt2 / 3.0 + dx * tt1 * 3.0;
    double f22 = tt2 / 3.0 + dy * tt1 * 3.0;
    double f33 = tt2 / 3.0 + dz * tt1 * 3.0;
    double f12 = 3.0 * dxy * tt1, f23 = 3.0 * dyz * tt1, f31 = 3.0 * dzx * tt1;
    double roue = (1 + eps0) * log(so->sme0 / sm);
    if (roue < 0.0) roue = 0.0;
    double ttt = ann * roue * roue;
    double hdd = f11 + f22 + f33 + ttt / sm;
    double fkk = f11 + f22 + f33;
    double fij = 2.0 * (f11 * f11 + f22 * f22 + f33 * f33) + f12 * f12 + f23 * f23 + f31 * f31;
    double cc7 = dlam * (fkk * fkk) + dmu * fij + hdd / hee;
    double d = 1.0 / cc7;
    double df = dlam * fkk, dg = dlam * fkk;
    double ramda = (dmu2 * f11 + dlam * fkk) * deps[0] + (dmu2 * f22 + dlam * fkk) * deps[1]
        + (dmu2 * f33 + dlam * fkk) * deps[2] + dmu * (f12 * deps[3] + f23 * deps[4] + f31 * deps[5]);
    if (ramda < 0.0) {
        double ww[6] = {dg + dmu2 * f11, dg + dmu2 * f22, dg + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
        double zz[6] = {df + dmu2 * f11, df + dmu2 * f22, df + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
        plastic_update(dept, d, ww, zz);
        adps[0] = ramda * d * f11; adps[1] = ramda * d * f22; adps[2] = ramda * d * f33;
        adps[3] = ramda * d * f12; adps[4] = ramda * d * f23; adps[5] = ramda * d * f31;
    }
}

/* elastic_plastic: Mohr-Coulomb (Drucker-Prager circumscribed cone with a
 * non-associated flow), CPP_8-1-consfactor.cpp:618-777.  Its mean stress uses
 * 0.333333333 (nine 3s) where the other models use ten. */
static void mc_model(double dept[6][6], const double* sig, const double* deps, const sphgpu_soil* so, double* adps)
{
    double sigct[6], e0, poi = so->poi, eps0 = so->eps0, zkapa = so->kapa;
    double fai = atan(tan(so->fai * 0.0174532925166667) / so->fs);
    double ci = so->c / so->fs;
    for (int a = 0; a < 6; a++) {
        sigct[a] = -sig[a];
        for (int b = 0; b < 6; b++) dept[a][b] = 0.0;
    }
    double sm = (sigct[0] + sigct[1] + sigct[2]) * 0.333333333;
    if (sm < 1.0) sm = 1.0;
    if (so->e > 1.0) e0 = so->e;
    else e0 = 3 * (1 - 2 * poi) * (1 + eps0) * fabs(sm) / zkapa;
    double dlam = e0 * poi / (1.0 + poi) / (1.0 - 2.0 * poi);
    double dmu = e0 * 0.5 / (1.0 + poi), dmu2 = dmu * 2.0;
    dept[0][0] = dlam + dmu2; dept[1][1] = dlam + dmu2; dept[2][2] = dlam + dmu2;
    dept[0][1] = dlam; dept[0][2] = dlam; dept[1][0] = dlam;
    dept[1][2] = dlam; dept[2][0] = dlam; dept[2][1] = dlam;
    dept[3][3] = dmu; dept[4][4] = dmu; dept[5][5] = dmu;
    double dx = sigct[0] - sm, dy = sigct[1] - sm, dz = sigct[2] - sm;
    double dxy = sigct[3], dyz = sigct[4], dzx = sigct[5];
    double sjj = 0.5 * (dx * dx + dy * dy + dz * dz) + dxy * dxy + dyz * dyz + dzx * dzx;
    double sj = sqrt(sjj);
    double yalf = sin(fai) / sqrt(9.0 + 3.0 * sin(fai) * sin(fai));
    double ykap = 3.0 * ci * cos(fai) / sqrt(9.0 + 3.0 * sin(fai) * sin(fai));
    if ((sj - yalf * sm * 3.0 - ykap) >= 0.0) {
        double f11 = -yalf + dx / sj * 0.5, f22 = -yalf + dy / sj * 0.5, f33 = -yalf + dz / sj * 0.5;
        double f12 = dxy / sj * 0.5, f23 = dyz / sj * 0.5, f31 = dzx / sj * 0.5;
        double fkk = f11 + f22 + f33;
        double g11 = dx / sj * 0.5, g22 = dy / sj * 0.5, g33 = dz / sj * 0.5;
        double g12 = dxy / sj * 0.5, g23 = dyz / sj * 0.5, g31 = dzx / sj * 0.5;
        double hdd = g11 + g22 + g33;
        double fij = 2.0 * (f11 * g11 + f22 * g22 + f33 * g33) + f12 * g12 + f23 * g23 + f31 * g31;
        double cc7 = dlam * (fkk * hdd) + dmu * fij;
        double d = 1.0 / cc7;
        double df = dlam * fkk, dg = dlam * hdd;
        double ramda = (dmu2 * f11 - 3.0 * dlam * yalf) * deps[0] + (dmu2 * f22 - 3.0 * dlam * yalf) * deps[1]
            + (dmu2 * f33 - 3.0 * dlam * yalf) * deps[2] + dmu * (f12 * deps[3] + f23 * deps[4] + f31 * deps[5]);
        double ttt = ramda * d;
        if (ttt < 0.0) {
            double ww[6] = {dg + dmu2 * g11, dg + dmu2 * g22, dg + dmu2 * g33, dmu * g12, dmu * g23, dmu * g31};
            double zz[6] = {df + dmu2 * f11, df + dmu2 * f22, df + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
            plastic_update(dept, d, ww, zz);
            adps[0] = ramda * d * f11; adps[1] = ramda * d * f22; adps[2] = ramda * d * f33;
            adps[3] = ramda * d * f12; adps[4] = ramda * d * f23; adps[5] = ramda * d * f31;
        }
    }
}

/* viscous_elastic: CPP_8-1-consfactor.cpp:88-126 (sets dsig directly; the
 * shear modulus is the material's c) */
static void visco_elastic(double* ds, const double* sig, const double* deps, const sphgpu_soil* so)
{
    double sigct[6], e0, poi = so->poi, eps0 = so->eps0, zkapa = so->kapa;
    for (int a = 0; a < 6; a++) sigct[a] = -sig[a];
    double sm = (sigct[0] + sigct[1] + sigct[2]) * 0.3333333333;
    if (sm < 1.0) sm = 1.0;
    if (so->e > 1.0) e0 = so->e;
    else e0 = 3 * (1 - 2 * poi) * (1 + eps0) * fabs(sm) / zkapa;
    double k = e0 * 0.3333333333 / (1.0 - 2.0 * poi);
    double g = so->c;
    double epkk = deps[0] + deps[1] + deps[2];
    ds[0] = 2.0 * g * (deps[0] - epkk * 0.3333333333) + k * epkk;
    ds[1] = 2.0 * g * (deps[1] - epkk * 0.3333333333) + k * epkk;
    ds[2] = 2.0 * g * (deps[2] - epkk * 0.3333333333) + k * epkk;
    ds[3] = 2.0 * g * deps[3];
    ds[4] = 2.0 * g * deps[4];
    ds[5] = 2.0 * g * deps[5];
}

/* dpmodel1 (yalf_dil = 0) and dpmodel_bui (yalf_dil from beta):
 * CPP_8-1-consfactor.cpp:284-448 and 451-615 */
static void dpmodel(double dept[6][6], const double* sig, const double* deps, const sphgpu_soil* so, double* adps, int bui)
{
    double dlam, dmu, sm;
    elastic_d(dept, sig, so, &dlam, &dmu, &sm);
    double dmu2 = dmu * 2.0;
    double fai = atan(tan(so->fai * 0.0174532925166667) / so->fs);
    double fai_dil = atan(tan(so->beta * 0.0174532925166667) / so->fs);
    double ci = so->c / so->fs;
    double sigct[6];
    for (int a = 0; a < 6; a++) sigct[a] = -sig[a];
    double dx = sigct[0] - sm, dy = sigct[1] - sm, dz = sigct[2] - sm;
    double dxy = sigct[3], dyz = sigct[4], dzx = sigct[5];
    double sjj = 0.5 * (dx * dx + dy * dy + dz * dz) + dxy * dxy + dyz * dyz + dzx * dzx;
    double sj = sqrt(sjj);
    double yalf = sin(fai) / sqrt(9.0 + 3.0 * sin(fai) * sin(fai));
    double ykap = 3.0 * ci * cos(fai) / sqrt(9.0 + 3.0 * sin(fai) * sin(fai));
    if ((sj - yalf * sm * 3.0 - ykap) >= 0.0) {
        double f11 = -yalf + dx / sj * 0.5, f22 = -yalf + dy / sj * 0.5, f33 = -yalf + dz / sj * 0.5;
        double f12 = dxy / sj * 0.5, f23 = dyz / sj * 0.5, f31 = dzx / sj * 0.5;
        double fkk = f11 + f22 + f33;
        double yalf_dil = bui ? sin(fai_dil) / sqrt(9.0 + 3.0 * sin(fai_dil) * sin(fai_dil)) : 0.0;
        double g11 = -yalf_dil + dx / sj * 0.5, g22 = -yalf_dil + dy / sj * 0.5, g33 = -yalf_dil + dz / sj * 0.5;
        double g12 = dxy / sj * 0.5, g23 = dyz / sj * 0.5, g31 = dzx / sj * 0.5;
        double hdd = g11 + g22 + g33;
        double fij = 2.0 * (f11 * g11 + f22 * g22 + f33 * g33) + f12 * g12 + f23 * g23 + f31 * g31;
        double cc7 = dlam * (fkk * hdd) + dmu * fij + hdd;
        double d = 1.0 / cc7;
        double df = dlam * fkk, dg = dlam * hdd;
        double ramda = (dmu2 * f11 - 3.0 * dlam * yalf) * deps[0]
            + (dmu2 * f22 - 3.0 * dlam * yalf) * deps[1]
            + (dmu2 * f33 - 3.0 * dlam * yalf) * deps[2]
            + dmu * (f12 * deps[3] + f23 * deps[4] + f31 * deps[5]);
        double ttt = ramda * d;
        if (ttt < 0.0) {
            double ww[6] = {dg + dmu2 * g11, dg + dmu2 * g22, dg + dmu2 * g33, dmu * g12, dmu * g23, dmu * g31};
            double zz[6] = {df + dmu2 * f11, df + dmu2 * f22, df + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
            for (int a = 0; a < 6; a++)
                for (int b = 0; b < 6; b++) dept[a][b] = dept[a][b] - d * ww[a] * zz[b];
            adps[0] = ramda * d * f11; adps[1] = ramda * d * f22; adps[2] = ramda * d * f33;
            adps[3] = ramda * d * f12; adps[4] = ramda * d * f23; adps[5] = ramda * d * f31;
        }
    }
}

/* sub_camunsatu: unsaturated subloading Cam-clay, CPP_8-4-consfactor-umcc.cpp:
 * 17-180.  Its elastic part takes the mean stress with 0.333333333; the
 * suction term rous follows the particle's degree of saturation, and the
 * plastic branch also sets the stress correction erfs. */
static void sub_camunsatu(double dept[6][6], double* erfs, const double* sig, const double* deps,
                          double satu, double dsatu, const sphgpu_soil* so, double* adps)
{
    double zkapa = so->kapa, poi = so->poi, eps0 = so->eps0;
    double qq = (so->epsr - so->epss) / (so->sitas - so->sitar);
    double sigct[6];
    for (int a = 0; a < 6; a++) sigct[a] = -sig[a];
    double ymf = 3.0 * (so->zmf - 1.0) / (so->zmf + 2.0) / so->fs;
    double sm = (sigct[0] + sigct[1] + sigct[2]) * 0.333333333;
    if (sm < 1.0) sm = 1.0;
    double e0;
    if (so->e > 1.0) e0 = so->e;
    else e0 = 3 * (1 - 2 * poi) * (1 + eps0) * fabs(sm) / zkapa;
    double hee = (so->ramda - so->kapa) / (1.0 + eps0);
    double dlam = e0 * poi / (1.0 + poi) / (1.0 - 2.0 * poi);
    double dmu = e0 * 0.5 / (1.0 + poi);
    double dmu2 = dmu * 2.0;
    dept[0][0] = dlam + dmu2; dept[1][1] = dlam + dmu2; dept[2][2] = dlam + dmu2;
    dept[0][1] = dlam; dept[0][2] = dlam; dept[1][0] = dlam;
    dept[1][2] = dlam; dept[2][0] = dlam; dept[2][1] = dlam;
    dept[3][3] = dmu; dept[4][4] = dmu; dept[5][5] = dmu;
    double dx = sigct[0] - sm, dy = sigct[1] - sm, dz = sigct[2] - sm;
    double dxy = sigct[3], dyz = sigct[4], dzx = sigct[5];
    double sjj = 0.5 * (dx * dx + dy * dy + dz * dz) + dxy * dxy + dyz * dyz + dzx * dzx;
    double tt1 = 1.0 / (ymf * ymf * sm * sm + 3.0 * sjj);
    double tt2 = 2.0 * ymf * ymf * sm * tt1 - 1.0 / sm;
    double f11 = tt2 * 0.333333333 + dx * tt1 * 3.0;
    double f22 = tt2 * 0.333333333 + dy * tt1 * 3.0;
    double f33 = tt2 * 0.333333333 + dz * tt1 * 3.0;
    double f12 = 3.0 * dxy * tt1, f23 = 3.0 * dyz * tt1, f31 = 3.0 * dzx * tt1;
    double rous = qq * (so->sitas - satu);
    double roue = hee * (1.0 + so->eps0) * log(so->sme0 / sm);
    double ttt = so->ann * roue + so->bnn * rous;
    ttt = pow(ttt, so->beta);
    double hdd = f11 + f22 + f33 + ttt / sm;
    double fkk = f11 + f22 + f33;
    double fij = 2.0 * (f11 * f11 + f22 * f22 + f33 * f33) + f12 * f12 + f23 * f23 + f31 * f31;
    double cc7 = dlam * (fkk * fkk) + dmu * fij + hdd / hee;
    double d = 1.0 / cc7;
    double df = dlam * fkk, dg = dlam * fkk;
    double ramda = (dmu2 * f11 + dlam * fkk) * deps[0] + (dmu2 * f22 + dlam * fkk) * deps[1]
        + (dmu2 * f33 + dlam * fkk) * deps[2] + dmu * (f12 * deps[3] + f23 * deps[4] + f31 * deps[5]);
    double omake = qq * dsatu / (so->ramda - so->kapa);
    ramda = ramda + omake;
    if (ramda < 0.0) {
        erfs[0] = omake * d * (dept[0][0] * f11 + dept[0][1] * f22 + dept[0][2] * f33);
        erfs[1] = omake * d * (dept[1][0] * f11 + dept[1][1] * f22 + dept[1][2] * f33);
        erfs[2] = omake * d * (dept[2][0] * f11 + dept[2][1] * f22 + dept[2][2] * f33);
        erfs[3] = omake * d * (dept[3][3] * f12);
        erfs[4] = omake * d * (dept[4][4] * f23);
        erfs[5] = omake * d * (dept[5][5] * f31);
        double ww[6] = {dg + dmu2 * f11, dg + dmu2 * f22, dg + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
        double zz[6] = {df + dmu2 * f11, df + dmu2 * f22, df + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
        plastic_update(dept, d, ww, zz);
        adps[0] = ramda * d * f11; adps[1] = ramda * d * f22; adps[2] = ramda * d * f33;
        adps[3] = ramda * d * f12; adps[4] = ramda * d * f23; adps[5] = ramda * d * f31;
    }
}

/* detA: determinant by cofactor expansion along the first row, recursively
 * (CPP_8-5-consfactor-focc.cpp:265-290) */
static double fo_det(double a[6][6], int n)
{
    double bak[6][6], sum = 0;
    if (n == 1) return a[0][0];
    for (int i = 0; i < n; i++) {
        for (int j = 1; j < n; j++) {
            int cc = 0;
            for (int k = 0; k < n; k++) {
                if (k == i) continue;
                bak[j - 1][cc++] = a[j][k];
            }
        }
        sum += (i % 2 == 0 ? 1 : -1) * a[0][i] * fo_det(bak, n - 1);
    }
    return sum;
}

/* getAStart: the adjugate, ans[j][i] = (-1)^(i+j) det(minor i, j)
 * (CPP_8-5-consfactor-focc.cpp:293-322) */
static void fo_adjugate(double a[6][6], int n, double ans[6][6])
{
    double tmp[6][6];
    if (n == 1) { ans[0][0] = 1.0; return; }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            for (int k = 0; k < n - 1; k++)
                for (int t = 0; t < n - 1; t++) tmp[k][t] = a[k >= i ? k + 1 : k][t >= j ? t + 1 : t];
            ans[j][i] = fo_det(tmp, n - 1);
            if ((i + j) % 2 == 1) ans[j][i] = -ans[j][i];
        }
}

/* fractional_mcc: fractional-order plastic model of MCC,
 * CPP_8-5-consfactor-focc.cpp:13-247.  dept is the inverse of the compliance
 * (elastic, plus the plastic part n m / hp when the Cam-clay loading index
 * ramda_cc is negative) by adjugate / determinant; cijkl keeps the elastic
 * compliance for fractional_plastic. */
static void fractional_mcc(double dept[6][6], double cijkl[6][6], const double* sig, const double* deps,
                           double e, const sphgpu_soil* so)
{
    double sigct[6], sij[6], smn[3][3], mij[6], nij[6], pijkl[6][6], total[6][6], adjoint[6][6];
    double p0 = 98000, pa = 98000;
    double poi = so->poi, h1 = so->damp1, h2 = so->damp2, ramda = so->ramda, mc = so->zmf;
    double alpha = so->ann, beta = so->bnn, c = so->c, zeta = so->zet, etao = so->etao, g0 = so->g0;
    for (int a = 0; a < 6; a++) {
        sigct[a] = -sig[a];
        for (int b = 0; b < 6; b++) { cijkl[a][b] = 0.0; pijkl[a][b] = 0.0; }
    }
    double sm = (sigct[0] + sigct[1] + sigct[2]) / 0.33333333;
    for (int a = 0; a < 6; a++) sij[a] = (a < 3) ? sigct[a] - sm : sigct[a];
    double q = 0.5 * (sij[0] * sij[0] + sij[1] * sij[1] + sij[2] * sij[2]) + sij[3] * sij[3] + sij[4] * sij[4] + sij[5] * sij[5];
    q = sqrt(3.0 * q);
    double ita = q / sm;
    if (ita == 0.0) {
        ita = 0.000001;
        q = ita * sm;
    }
    double g = g0 * (2.97 - e) * (2.97 - e) / (1.0 + e) * sqrt(sm * pa);
    double e0 = 2.0 * g * (1.0 + poi);
    double ymf = mc;
    double dlam = e0 * poi / (1.0 + poi) / (1.0 - 2.0 * poi);
    double dmu = e0 * 0.5 / (1.0 + poi);
    double dmu2 = dmu * 2.0;
    double tt1 = 1.0 / (ymf * ymf * sm * sm + q * q);
    double tt2 = 2.0 * ymf * ymf * sm * tt1 - 1.0 / sm;
    double f11 = tt2 * 0.33333333 + sij[0] * tt1 * 3.0;
    double f22 = tt2 * 0.33333333 + sij[1] * tt1 * 3.0;
    double f33 = tt2 * 0.33333333 + sij[2] * tt1 * 3.0;
    double f12 = 3.0 * sij[3] * tt1, f23 = 3.0 * sij[4] * tt1, f31 = 3.0 * sij[5] * tt1;
    double fkk = f11 + f22 + f33;
    double ramda_cc = (dmu2 * f11 + dlam * fkk) * deps[0] + (dmu2 * f22 + dlam * fkk) * deps[1]
        + (dmu2 * f33 + dlam * fkk) * deps[2] + dmu * (f12 * deps[3] + f23 * deps[4] + f31 * deps[5]);
    /* Lode angle */
    smn[0][0] = sij[0]; smn[0][1] = sij[3]; smn[0][2] = sij[5];
    smn[1][0] = sij[3]; smn[1][1] = sij[1]; smn[1][2] = sij[4];
    smn[2][0] = sij[5]; smn[2][1] = sij[4]; smn[2][2] = sij[2];
    double s_val = 0.0, skl = 0.0;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int k = 0; k < 3; k++) s_val = s_val + smn[a][b] * smn[b][k] * smn[k][a];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) skl = skl + smn[a][b] * smn[b][a];
    if (skl == 0.0) skl = 0.000001;
    double sita = 9.0 * s_val * 0.5 / pow(1.5 * skl, 1.5);
    if (sita < -1.0) sita = -1.0;
    else if (sita > 1.0) sita = 1.0;
    sita = asin(sita) * 0.33333333;
    c = pow(c, 4);
    double m = 2 * c / (1 + c + (1 - c) * sin(3.0 * sita));
    m = pow(m, 0.25);
    m = mc * m;
    double pc = pa * pow((etao - e) / ramda, 1 / zeta);
    double qc = q + m * (sm - pc);
    double df = (sm - p0 / 2) * mc * mc / q;
    double dg = ((sm - pc) + (2 - alpha) * (pc - sm * 0.5 - q * q / mc / mc / sm / 2)) / ((q - qc) + (2 - alpha) * qc);
    dg = pow(m, alpha + 1) * dg;
    for (int a = 0; a < 6; a++) {
        mij[a] = 1.0 / sqrt(1.0 + df * df) * ((a < 3) ? 3.0 * sij[a] * 0.5 / q + df * 0.33333333 : 3.0 * sij[a] * 0.5 / q);
        nij[a] = 1.0 / sqrt(1.0 + dg * dg) * ((a < 3) ? 3.0 * sij[a] * 0.5 / q + dg * 0.33333333 : 3.0 * sij[a] * 0.5 / q);
    }
    double order = beta * (e - etao + ramda * pow(sm / pa, zeta));
    double mf = mc * pow(2.71828, -order);
    double hp = (h1 - h2 * e) * (1 - e) * g * (mf - ita) / ita * pow(2.71828, order);
    cijkl[0][0] = 1.0 / e0; cijkl[1][1] = 1.0 / e0; cijkl[2][2] = 1.0 / e0;
    cijkl[0][1] = -poi / e0; cijkl[0][2] = -poi / e0; cijkl[1][0] = -poi / e0;
    cijkl[1][2] = -poi / e0; cijkl[2][0] = -poi / e0; cijkl[2][1] = -poi / e0;
    cijkl[3][3] = 1.0 / g; cijkl[4][4] = 1.0 / g; cijkl[5][5] = 1.0 / g;
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) pijkl[a][b] = nij[a] * mij[b] / hp;
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) total[a][b] = (ramda_cc < 0.0) ? cijkl[a][b] + pijkl[a][b] : cijkl[a][b];
    double det_a = fo_det(total, 6);
    fo_adjugate(total, 6, adjoint);
    /* a singular total falls back to the elastic compliance; the reference
     * switches on the first element, so every element takes it */
    if (det_a == 0.0) {
        det_a = fo_det(cijkl, 6);
        fo_adjugate(cijkl, 6, adjoint);
    }
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) dept[a][b] = adjoint[a][b] / det_a;
}

/* fractional_plastic: plastic strain rate = strain rate - C dsig,
 * CPP_8-5-consfactor-focc.cpp:250-264 */
static void fractional_plastic(const double* dsig, const double* deps, double* adps, double cijkl[6][6])
{
    double eeps[6];
    for (int a = 0; a < 6; a++) {
        eeps[a] = 0.0;
        for (int b = 0; b < 6; b++) eeps[a] = eeps[a] + cijkl[a][b] * dsig[b];
    }
    for (int a = 0; a < 6; a++) adps[a] = deps[a] - eeps[a];
}

/* TSSMP_before: the transformed stress of the SMP criterion from the
 * principal stresses of the last Stress_eigValue, CPP_7-3-TS.cpp:14-67 */
static void tssmp_before(orc_ctx* c, int i, double alpha)
{
    double* s = &c->sig[i * 6];
    const double* sp = &c->strep[i * 3];
    double qc = 0.0, sx[6];
    c->tsqc[i] = 0.0;
    sx[0] = -s[0] + c->vsig[i];
    sx[1] = -s[1] + c->vsig[i];
    sx[2] = -s[2] + c->vsig[i];
    sx[3] = -s[3]; sx[4] = -s[4]; sx[5] = -s[5];
    double q = c->divq[i];
    double I1 = -(sp[0] + sp[1] + sp[2]);
    double I2 = sp[0] * sp[1] + sp[1] * sp[2] + sp[2] * sp[1];
    double I3 = -sp[0] * sp[1] * sp[2];
    if ((I1 * I1 - 3.0 * I2) >= 1.0e-7) {
        double temp = 3.0 * sqrt((I1 * I2 - I3) / (I1 * I2 - 9.0 * I3)) - 1.0;
        if (fabs(temp) >= 1.0e-7)
            qc = alpha * sqrt(I1 * I1 - 3.0 * I2) + 2.0 * (1.0 - alpha) * I1 / (3.0 * sqrt((I1 * I2 - I3) / (I1 * I2 - 9.0 * I3)) - 1.0);
        else
            qc = 0.0;
    } else
        qc = 0.0;
    c->tsqc[i] = qc;
    for (int a = 0; a < 6; a++) c->tssig[i * 6 + a] = s[a];
    if (q != 0.0) {
        s[0] = -I1 * 0.33333333 - qc / q * sx[0];
        s[1] = -I1 * 0.33333333 - qc / q * sx[1];
        s[2] = -I1 * 0.33333333 - qc / q * sx[2];
        s[3] = -qc / q * sx[3];
        s[4] = -qc / q * sx[4];
        s[5] = -qc / q * sx[5];
    }
}

/* TSSMP_after: the stress rate back to the real stress space; sig and tssig
 * exchange, CPP_7-3-TS.cpp:69-105 */
static void tssmp_after(orc_ctx* c, int i, double* ds)
{
    double q = c->divq[i], qc = c->tsqc[i], temp[6];
    double* s = &c->sig[i * 6];
    double* ts = &c->tssig[i * 6];
    double dvsig = (ds[0] + ds[1] + ds[2]) / 3.0;
    if (qc != 0.0) {
        ds[0] = dvsig + q / qc * (ds[0] - dvsig);
        ds[1] = dvsig + q / qc * (ds[1] - dvsig);
        ds[2] = dvsig + q / qc * (ds[2] - dvsig);
        ds[3] = q / qc * ds[3];
        ds[4] = q / qc * ds[4];
        ds[5] = q / qc * ds[5];
    }
    for (int a = 0; a < 6; a++) temp[a] = ts[a];
    for (int a = 0; a < 6; a++) ts[a] = s[a];
    for (int a = 0; a < 6; a++) s[a] = temp[a];
}

/* moisturesuct: suction from the degree of saturation on the wetting or
 * drying curve, CPP_7-2-constitutive.cpp:323-338 (its first tan, for
 * saturations within 1e-4 of the residual one, is overwritten) */
static double moisturesuct(double satu, double dsatu, const sphgpu_soil* so)
{
    const double pi_ = 3.141592653;   /* Header_Parameters.h:10 */
    double temp = tan(pi_ * (so->sitas - satu) / (so->sitas - so->sitar) / 2.0);
    if (dsatu > 0.0) return log(1 + exp(so->c2 * so->sw) * temp) / so->c2;
    return log(1 + exp(so->c1 * so->sd) * temp) / so->c1;
}

/* saturation: degree of saturation of soil particles from their water
 * neighbours (flagum == 1), CPP_7-1-strain.cpp:222-281 */
static void saturation(orc_ctx* c)
{
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] != 2) continue;   /* the sums of other particles are unused */
        const sphgpu_soil* so = &c->so[i];
        double cof = so->sitas - so->sitar, sitas = so->sitas, sitar = so->sitar;
        double tempup = 0.0, tempdown = 0.0;
        int nc = c->ninflu[i];
        for (int nj = 1; nj <= nc; nj++) {
            int j = c->influ[i * NB + nj];
            if (c->type[j] == 1) {
                double w = c->wij[((size_t)i * NB + nj) * 4 + 3];
                tempup = tempup + c->mass[j] / c->rho[j] * cof * w;
                tempdown = tempdown + c->mass[j] / c->rho[j] * w;
            }
        }
        double psatu = c->satu[i];
        if (tempdown != 0.0) c->satu[i] = tempup / tempdown + sitar;
        else c->satu[i] = tempup + sitar;
        c->dsatu[i] = c->satu[i] - psatu;
        if (c->dsatu[i] < 0) {
            c->satu[i] = c->satu[i] - c->dsatu[i];
            c->dsatu[i] = 0.0;
        }
        if (c->satu[i] > sitas) c->satu[i] = sitas;
        else if (c->satu[i] < sitar) c->satu[i] = sitar;
        c->suct[i] = moisturesuct(c->satu[i], c->dsatu[i], so);
    }
}

/* DPModel_check: stress-scaling return, CPP_8-1-consfactor.cpp:779-819 */
static void dp_check(double* sig, double* dsig, const sphgpu_soil* so, double dt)
{
    double ts[6];
    double fai = atan(tan(so->fai * 0.0174532925166667) / so->fs);
    double ci = so->c / so->fs;
    double sm = (sig[0] + sig[1] + sig[2]) / 3.0;
    double dx = sig[0] - sm, dy = sig[1] - sm, dz = sig[2] - sm;
    double sj_2 = 0.5 * (dx * dx + dy * dy + dz * dz) + sig[3] * sig[3] + sig[4] * sig[4] + sig[5] * sig[5];
    double sj = sqrt(sj_2);
    for (int a = 0; a < 6; a++) ts[a] = sig[a] + dsig[a] * dt;
    double i_1 = ts[0] + ts[1] + ts[2];
    double alpha_fai = sin(fai) / sqrt(9.0 + 3.0 * sin(fai) * sin(fai));
    double k_c = 3.0 * ci * cos(fai) / sqrt(9.0 + 3.0 * sin(fai) * sin(fai));
    double rn = (-alpha_fai * i_1 + k_c) / sj;
    if (rn < 1.0) {
        ts[0] = rn * (ts[0] - i_1 / 3.0) + i_1 / 3.0;
        ts[1] = rn * (ts[1] - i_1 / 3.0) + i_1 / 3.0;
        ts[2] = rn * (ts[2] - i_1 / 3.0) + i_1 / 3.0;
        ts[3] = rn * ts[3];
        ts[4] = rn * ts[4];
        ts[5] = rn * ts[5];
    }
    for (int a = 0; a < 6; a++) dsig[a] = (ts[a] - sig[a]) / dt;
}

/* Jaumann rate terms: CPP_7-2-constitutive.cpp:236-253 (also 297-307) */
static void jaumann(double* ds, const double* s, const double* w)
{
#define WE(a, b) w[(a) * 3 + (b)]
    ds[0] = ds[0] + (WE(0, 0) * s[0] + WE(0, 1) * s[3] + WE(0, 2) * s[5]) - (s[0] * WE(0, 0) + s[3] * WE(1, 0) + s[5] * WE(2, 0));
    ds[1] = ds[1] + (WE(1, 0) * s[3] + WE(1, 1) * s[1] + WE(1, 2) * s[4]) - (s[3] * WE(0, 1) + s[1] * WE(1, 1) + s[4] * WE(2, 1));
    ds[2] = ds[2] + (WE(2, 0) * s[5] + WE(2, 1) * s[4] + WE(2, 2) * s[2]) - (s[5] * WE(0, 2) + s[4] * WE(1, 2) + s[2] * WE(2, 2));
    ds[3] = ds[3] + (WE(0, 0) * s[3] + WE(0, 1) * s[1] + WE(0, 2) * s[4]) - (s[0] * WE(0, 1) + s[3] * WE(1, 1) + s[5] * WE(2, 1));
    ds[4] = ds[4] + (WE(1, 0) * s[5] + WE(1, 1) * s[4] + WE(1, 2) * s[2]) - (s[3] * WE(0, 2) + s[1] * WE(1, 2) + s[4] * WE(2, 2));
    ds[5] = ds[5] + (WE(0, 0) * s[5] + WE(0, 1) * s[4] + WE(0, 2) * s[2]) - (s[0] * WE(0, 2) + s[3] * WE(1, 2) + s[5] * WE(2, 2));
#undef WE
}

/* strain_to_stress: CPP_7-2-constitutive.cpp:13-321.  Soil models restated:
 * elastic (matype%10 = 0, 6), subloading Cam-clay (1), Drucker-Prager (2,
 * with DPModel_check), unsaturated Cam-clay (3), anisotropic Cam-clay (4, an
 * empty model), Bui DP (5, with DPModel_check), viscous-elastic (7),
 * fractional-order MCC (8) and Mohr-Coulomb (9), each inside the TSSMP
 * transformation when flts >= 1. */
static int strain_to_stress(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    double dt = P->dt;
    for (int i = 0; i < c->n; i++) {
        int ti = c->type[i];
        double* s = &c->sig[i * 6];
        double* de = &c->deps[i * 6];
        double* ep = &c->eps[i * 6];
        if (ti == 1) {
            double strain_min = c->fl[i].strain_min, viscos1, d[6];
            double depsmax = (de[0] + de[1] + de[2]) / 3.0;
            ep[0] = de[0] - depsmax;
            ep[1] = de[1] - depsmax;
            ep[2] = de[2] - depsmax;
            depsmax = 0.666666666666667 * (ep[0] * ep[0] + ep[1] * ep[1]
                + ep[2] * ep[2] + de[3] * de[3] * 0.25 +
                de[4] * de[4] * 0.25 + de[5] * de[5] * 0.25);
            depsmax = sqrt(depsmax);
            if (c->fl[i].bhtype == 1) {
                double fai = c->fl[i].fai * 0.0174532925199;
                double tao = c->pre[i] * tan(fai) + c->fl[i].c;
                if (depsmax < strain_min) viscos1 = c->fl[i].vis + tao / strain_min;
                else viscos1 = c->fl[i].vis + tao / depsmax;
            } else
                viscos1 = c->fl[i].vis;
            d[0] = 2.0 * de[0] - 2.0 * (de[0] + de[1] + de[2]) / 3.0;
            d[1] = 2.0 * de[1] - 2.0 * (de[0] + de[1] + de[2]) / 3.0;
            d[2] = 2.0 * de[2] - 2.0 * (de[0] + de[1] + de[2]) / 3.0;
            d[3] = de[3]; d[4] = de[4]; d[5] = de[5];
            for (int a = 0; a < 6; a++) s[a] = (a < 3) ? -c->pre[i] - viscos1 * d[a] : -viscos1 * d[a];
        } else if (ti == 3) {
            double viscos1 = c->fl[i].vis, d[6];
            d[0] = 2.0 * de[0] - 2.0 * (de[0] + de[1] + de[2]) / 3.0;
            d[1] = 2.0 * de[1] - 2.0 * (de[0] + de[1] + de[2]) / 3.0;
            d[2] = 2.0 * de[2] - 2.0 * (de[0] + de[1] + de[2]) / 3.0;
            d[3] = de[3]; d[4] = de[4]; d[5] = de[5];
            for (int a = 0; a < 6; a++) s[a] = (a < 3) ? -c->pre[i] - viscos1 * d[a] : -viscos1 * d[a];
        } else if (ti == 2) {
            double dept[6][6], adps[6] = {0, 0, 0, 0, 0, 0}, erfs[6] = {0, 0, 0, 0, 0, 0}, cijkl[6][6];
            double dl, dm, sm;
            double* ds = &c->dsig[i * 6];
            int mt = c->matype[i] % 10;
            const int m = c->matype[i];
            /* matype 30-49 and >= 60 match no branch of the reference's dispatch */
            if ((m >= 30 && m < 50) || m >= 60) return SPHGPU_E_UNSUPPORTED;
            for (int a = 0; a < 6; a++)
                for (int b = 0; b < 6; b++) { dept[a][b] = 0.0; cijkl[a][b] = 0.0; }
            /* transformed stress of the SMP criterion, step 1 (:99-101) */
            if (P->flts >= 1) tssmp_before(c, i, P->alphats);
            if (c->l < P->inip || mt == 0 || mt == 6) {
                elastic_d(dept, s, &c->so[i], &dl, &dm, &sm);
            } else if (mt == 1) {
                sub_camclay(dept, s, de, &c->so[i], adps);
            } else if (mt == 2 || mt == 5) {
                dpmodel(dept, s, de, &c->so[i], adps, mt == 5);
            } else if (mt == 3) {
                sub_camunsatu(dept, erfs, s, de, c->satu[i], c->dsatu[i], &c->so[i], adps);
            } else if (mt == 4) {
                /* sub_camanisotropy (CPP_8-2-consfactor-amcc.cpp:17-99): its body is
                 * commented out, so dept stays zero */
            } else if (mt == 8) {
                fractional_mcc(dept, cijkl, s, de, c->e[i], &c->so[i]);
            } else if (mt == 9) {
                mc_model(dept, s, de, &c->so[i], adps);
            } else {
                visco_elastic(ds, s, de, &c->so[i]);
            }
            if (c->l < P->inip || mt != 7) {
                for (int a = 0; a < 6; a++)
                    for (int b = 0; b < 6; b++) ds[a] += dept[a][b] * de[b];
                /* depp0 = dept; its largest diagonal entry 0-2, as
                 * soil_damping_vibration takes it (CPP_9-1:186-188) */
                double st = fmax(0.0, dept[0][0]);
                st = fmax(st, dept[1][1]);
                st = fmax(st, dept[2][2]);
                c->stiff[i] = st;
            }
            if (!(c->l < P->inip) && (mt == 2 || mt == 5)) dp_check(s, ds, &c->so[i], dt);
            jaumann(ds, s, &c->weps[i * 9]);
            /* fractional_plastic for matype 8, 18, 28 (:255-258).  In elastic steps
             * (l < inip) the reference reads cijkl uninitialised there; only the
             * output-only adps depends on it, and a zero compliance is taken. */
            if (m == 8 || m == 18 || m == 28) fractional_plastic(ds, de, adps, cijkl);
            /* step 2: the rate back to the real stress; sig restored (:261-262) */
            if (P->flts >= 1) tssmp_after(c, i, ds);
            for (int a = 0; a < 6; a++) {
                c->adps[i * 6 + a] = c->adps[i * 6 + a] + adps[a] * dt;
                ep[a] = ep[a] + de[a] * dt;
                s[a] = s[a] + ds[a] * dt + erfs[a];
            }
            deq(c, i);
            shearstrain(c, i);
            poro_cal(c, i, dt);
        } else if (ti == 4) {
            double dept[6][6], e0 = P->structure.e, poi = P->structure.poi;
            double* ds = &c->dsig[i * 6];
            for (int a = 0; a < 6; a++) for (int b = 0; b < 6; b++) dept[a][b] = 0.0;
            double dlam = e0 * poi / (1.0 + poi) / (1.0 - 2.0 * poi);
            double dmu = e0 * 0.5 / (1.0 + poi), dmu2 = dmu * 2.0;
            dept[0][0] = dlam + dmu2; dept[1][1] = dlam + dmu2; dept[2][2] = dlam + dmu2;
            dept[0][1] = dlam; dept[0][2] = dlam; dept[1][0] = dlam;
            dept[1][2] = dlam; dept[2][0] = dlam; dept[2][1] = dlam;
            dept[3][3] = dmu; dept[4][4] = dmu; dept[5][5] = dmu;
            for (int a = 0; a < 6; a++)
                for (int b = 0; b < 6; b++) ds[a] += dept[a][b] * de[b];
            {
                double st = fmax(0.0, dept[0][0]);
                st = fmax(st, dept[1][1]);
                st = fmax(st, dept[2][2]);
                c->stiff[i] = st;
            }
            jaumann(ds, s, &c->weps[i * 9]);
            for (int a = 0; a < 6; a++) {
                ep[a] = ep[a] + de[a] * dt;
                s[a] = s[a] + ds[a] * dt;
            }
            deq(c, i);
            shearstrain(c, i);
            poro_cal(c, i, dt);
        }
    }
    return 0;
}

/* free_surface_check: CPP_7-2-constitutive.cpp:453-506 */
static void free_surface_check(orc_ctx* c)
{
    double tmax = c->P.threshold_max, tmin = c->P.threshold_min, incline = tmax - tmin;
    for (int i = 0; i < c->n; i++) {
        double color = 0.0;
        int ti = c->type[i];
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), tj = c->type[j];
            if (ti == tj && (ti != 0 && ti != 7))
                color = color + c->mass[j] / c->rho[j] * 1.0 * W(i, nj, 3);
            else if (ti != tj && (ti > 0 && ti < 5)) {
                if (tj == 0) color = color + c->mass[j] / c->rho[j] * 1.0 * W(i, nj, 3);
            }
        }
        double* s = &c->sig[i * 6];
        if (ti == 1) {
            if (color < tmin / 2.0) {
                for (int k = 0; k < 3; k++) s[k] = -1.0;
                for (int k = 3; k < 6; k++) s[k] = 0.0;
            } else if (color >= tmin / 2.0 && color < tmax / 2.0) {
                double xishu = (2.0 * color - tmin) / incline;
                for (int k = 0; k < 6; k++) s[k] = xishu * s[k];
            }
        } else if (ti == 2) {
            if (color < tmin) {
                for (int k = 0; k < 3; k++) s[k] = -1.0;
                for (int k = 3; k < 6; k++) s[k] = 0.0;
            } else if (color >= tmin && color < tmax) {
                double xishu = (color - tmin) / incline * 1.0;
                for (int k = 0; k < 6; k++) s[k] = xishu * s[k];
            }
            stress_adjust(c, i);
            deq(c, i);
        }
    }
}

/* eejcb: Jacobi eigen-solver, CPP_7-1-strain.cpp:341-437 */
static int eejcb(double a[], int n, double v[], double eps, int jt)
{
    int i, j, p = 0, q = 0, u, w, t, s, l = 1;
    double fm, cn, sn, omega, x, y, d;
    for (i = 0; i <= n - 1; i++) {
        v[i * n + i] = 1.0;
        for (j = 0; j <= n - 1; j++)
            if (i != j) v[i * n + j] = 0.0;
    }
    while (1) {
        fm = 0.0;
        for (i = 0; i <= n - 1; i++)
            for (j = 0; j <= n - 1; j++) {
                d = fabs(a[i * n + j]);
                if ((i != j) && (d > fm)) { fm = d; p = i; q = j; }
            }
        if (fm < eps) return 1;
        if (l > jt) return -1;
        l = l + 1;
        u = p * n + q; w = p * n + p; t = q * n + p; s = q * n + q;
        x = -a[u];
        y = (a[s] - a[w]) / 2.0;
        omega = x / sqrt(x * x + y * y);
        if (y < 0.0) omega = -omega;
        sn = 1.0 + sqrt(1.0 - omega * omega);
        sn = omega / sqrt(2.0 * sn);
        cn = sqrt(1.0 - sn * sn);
        fm = a[w];
        a[w] = fm * cn * cn + a[s] * sn * sn + a[u] * omega;
        a[s] = fm * sn * sn + a[s] * cn * cn - a[u] * omega;
        a[u] = 0.0;
        a[t] = 0.0;
        for (j = 0; j <= n - 1; j++)
            if ((j != p) && (j != q)) {
                u = p * n + j; w = q * n + j;
                fm = a[u];
                a[u] = fm * cn + a[w] * sn;
                a[w] = -fm * sn + a[w] * cn;
            }
        for (i = 0; i <= n - 1; i++)
            if ((i != p) && (i != q)) {
                u = i * n + p; w = i * n + q;
                fm = a[u];
                a[u] = fm * cn + a[w] * sn;
                a[w] = -fm * sn + a[w] * cn;
            }
        for (i = 0; i <= n - 1; i++) {
            u = i * n + p; w = i * n + q;
            fm = v[u];
            v[u] = fm * cn + v[w] * sn;
            v[w] = -fm * sn + v[w] * cn;
        }
    }
    return 1;
}

/* Stress_eigValue: CPP_7-1-strain.cpp:283-332 */
static void stress_eig(orc_ctx* c)
{
    for (int i = 0; i < c->n; i++) {
        double st[9], ev[9];
        const double* s = &c->sig[i * 6];
        for (int k = 0; k < 9; k++) ev[k] = 0.0;
        st[0] = s[0]; st[1] = s[3]; st[2] = s[5];
        st[3] = s[3]; st[4] = s[1]; st[5] = s[4];
        st[6] = s[5]; st[7] = s[4]; st[8] = s[2];
        eejcb(st, 3, ev, 0.001, 7);
        for (int k = 0; k < 3; k++) c->strep[i * 3 + k] = st[k * 3 + k];
        for (int k = 0; k < 3; k++) {
            c->beta_ts[i * 9 + k * 3 + 0] = ev[k * 3];
            c->beta_ts[i * 9 + k * 3 + 1] = ev[k * 3 + 1];
            c->beta_ts[i * 9 + k * 3 + 2] = ev[k * 3 + 2];
            c->beta[i * 9 + 0 * 3 + k] = ev[k * 3];
            c->beta[i * 9 + 1 * 3 + k] = ev[k * 3 + 1];
            c->beta[i * 9 + 2 * 3 + k] = ev[k * 3 + 2];
        }
    }
}

/* ------------------------------------------------------------------------- */
/* momentum: CPP_9-4-derivation_stress.cpp                                   */

/* one pair of the symmetric stress-divergence sum, the 9 lines shared by
 * fluid_acceleration_water/air (:55-65) and the soil/structure forms */
static void stress_pair(double tu[3][3], double mj, const double* aj, const double* ai,
                        double rj, double ri, const double* w, double sgn)
{
    if (sgn > 0) {
        tu[0][0] = tu[0][0] + mj * (aj[0] / rj / rj + ai[0] / ri / ri) * w[0];
        tu[0][1] = tu[0][1] + mj * (aj[3] / rj / rj + ai[3] / ri / ri) * w[1];
        tu[0][2] = tu[0][2] + mj * (aj[5] / rj / rj + ai[5] / ri / ri) * w[2];
        tu[1][0] = tu[1][0] + mj * (aj[3] / rj / rj + ai[3] / ri / ri) * w[0];
        tu[1][1] = tu[1][1] + mj * (aj[1] / rj / rj + ai[1] / ri / ri) * w[1];
        tu[1][2] = tu[1][2] + mj * (aj[4] / rj / rj + ai[4] / ri / ri) * w[2];
        tu[2][0] = tu[2][0] + mj * (aj[5] / rj / rj + ai[5] / ri / ri) * w[0];
        tu[2][1] = tu[2][1] + mj * (aj[4] / rj / rj + ai[4] / ri / ri) * w[1];
        tu[2][2] = tu[2][2] + mj * (aj[2] / rj / rj + ai[2] / ri / ri) * w[2];
    } else {
        tu[0][0] = tu[0][0] + mj * (aj[0] / rj / rj - ai[0] / ri / ri) * w[0];
        tu[0][1] = tu[0][1] + mj * (aj[3] / rj / rj - ai[3] / ri / ri) * w[1];
        tu[0][2] = tu[0][2] + mj * (aj[5] / rj / rj - ai[5] / ri / ri) * w[2];
        tu[1][0] = tu[1][0] + mj * (aj[3] / rj / rj - ai[3] / ri / ri) * w[0];
        tu[1][1] = tu[1][1] + mj * (aj[1] / rj / rj - ai[1] / ri / ri) * w[1];
        tu[1][2] = tu[1][2] + mj * (aj[4] / rj / rj - ai[4] / ri / ri) * w[2];
        tu[2][0] = tu[2][0] + mj * (aj[5] / rj / rj - ai[5] / ri / ri) * w[0];
        tu[2][1] = tu[2][1] + mj * (aj[4] / rj / rj - ai[4] / ri / ri) * w[1];
        tu[2][2] = tu[2][2] + mj * (aj[2] / rj / rj - ai[2] / ri / ri) * w[2];
    }
}

/* fluid_acceleration_water / _air and the minor forms: :12-351 */
static void fluid_acceleration(orc_ctx* c, int me, int other, int minor)
{
    double g[3] = {c->P.gx, c->P.gy, c->P.gz};
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] != me) continue;
        double poro = c->fl[i].porosity, tu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int k = 0; k < 3; k++) c->ax[i * 3 + k] = g[k];
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[i] == c->type[j] || c->type[j] == other) {
                double ai[6], aj[6];
                for (int k = 0; k < 6; k++) { ai[k] = poro * c->sig[i * 6 + k]; aj[k] = poro * c->sig[j * 6 + k]; }
                stress_pair(tu, c->mass[j], aj, ai, c->rho[j], c->rho[i], &W(i, nj, 0), minor ? -1.0 : 1.0);
            }
        }
        c->ax[i * 3 + 0] += tu[0][0] + tu[0][1] + tu[0][2];
        c->ax[i * 3 + 1] += tu[1][0] + tu[1][1] + tu[1][2];
        c->ax[i * 3 + 2] += tu[2][0] + tu[2][1] + tu[2][2];
    }
}

/* soil_acceleration_noreg: :354-428 */
static void soil_acceleration(orc_ctx* c)
{
    double g[3] = {c->P.gx, c->P.gy, c->P.gz};
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] != 2) continue;
        double poro = c->so[i].porosity, tu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int k = 0; k < 3; k++) c->ax[i * 3 + k] = g[k];
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[i] != c->type[j]) continue;
            double satu = c->satu[j], prei[3], prej[3];
            const double* w = &W(i, nj, 0);
            for (int k = 0; k < 3; k++) {
                prei[k] = (1 - poro) * (-satu * c->prew[i] + (1 - satu) * c->prea[i]);
                prej[k] = (1 - poro) * (-satu * c->prew[j] + (1 - satu) * c->prea[j]);
            }
            stress_pair(tu, c->mass[j], &c->sig[j * 6], &c->sig[i * 6], c->rho[j], c->rho[i], w, 1.0);
            double mj = c->mass[j], rj = c->rho[j], di = c->so[i].dens;
            tu[0][0] = tu[0][0] + mj * (prej[0] / rj / rj + prei[0] / di / di) * w[0];
            tu[1][1] = tu[1][1] + mj * (prej[1] / rj / rj + prei[1] / di / di) * w[1];
            tu[2][2] = tu[2][2] + mj * (prej[2] / rj / rj + prei[2] / di / di) * w[2];
        }
        c->ax[i * 3 + 0] += tu[0][0] + tu[0][1] + tu[0][2];
        c->ax[i * 3 + 1] += tu[1][0] + tu[1][1] + tu[1][2];
        c->ax[i * 3 + 2] += tu[2][0] + tu[2][1] + tu[2][2];
    }
}

/* structure_acceleration_noreg: :431-505 */
static void structure_acceleration(orc_ctx* c)
{
    double g[3] = {c->P.gx, c->P.gy, c->P.gz};
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] != 4) continue;
        double tu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int k = 0; k < 3; k++) c->ax[i * 3 + k] = g[k];
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[i] != c->type[j]) continue;
            double satu = c->satu[j], prei[3], prej[3];
            const double* w = &W(i, nj, 0);
            for (int k = 0; k < 3; k++) {
                prei[k] = -satu * c->prew[i] + (1 - satu) * c->prea[i];
                prej[k] = -satu * c->prew[j] + (1 - satu) * c->prea[j];
            }
            stress_pair(tu, c->mass[j], &c->sig[j * 6], &c->sig[i * 6], c->rho[j], c->rho[i], w, 1.0);
            double mj = c->mass[j], rj = c->rho[j], ri = c->rho[i];
            tu[0][0] = tu[0][0] + mj * (prej[0] / rj / rj - prei[0] / ri / ri) * w[0];
            tu[1][1] = tu[1][1] + mj * (prej[1] / rj / rj - prei[1] / ri / ri) * w[1];
            tu[2][2] = tu[2][2] + mj * (prej[2] / rj / rj - prei[2] / ri / ri) * w[2];
        }
        c->ax[i * 3 + 0] += tu[0][0] + tu[0][1] + tu[0][2];
        c->ax[i * 3 + 1] += tu[1][0] + tu[1][1] + tu[1][2];
        c->ax[i * 3 + 2] += tu[2][0] + tu[2][1] + tu[2][2];
    }
}

/* artificial_viscosity: CPP_9-3-artificialvis.cpp:12-99 */
static void artificial_viscosity(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    int ndim = P->ndim;
    for (int i = 0; i < c->n; i++) {
        double tu[3] = {0, 0, 0};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), k;
            if (!(c->type[i] == c->type[j] && c->type[i] != 7)) continue;
            double a = 0.0, b = 0.0, cc = 0.0, inprod = 0.0, dst = 0.0, myu, paix, dvx[3], dx[3];
            for (k = 0; k < ndim; k++) {
                dvx[k] = c->vxp[i * 3 + k] - c->vxp[j * 3 + k];
                dx[k] = c->xp[i * 3 + k] - c->xp[j * 3 + k];
                dst = dst + dx[k] * dx[k];
                inprod = inprod + dvx[k] * dx[k];
            }
            double hl = (c->hl[j] + c->hl[i]) * 0.5;
            double rou = (c->rho[j] + c->rho[i]) * 0.5;
            if (c->type[i] == 1) { cc = c->fl[i].vpu; a = P->art_vis[0][0]; b = P->art_vis[0][1]; }
            if (c->type[i] == 2) { cc = c->so[i].vpu; a = P->art_vis[1][0]; b = P->art_vis[1][1]; }
            if (c->type[i] == 3) { cc = c->fl[i].vpu; a = P->art_vis[2][0]; b = P->art_vis[2][1]; }
            if (inprod < 0.0) {
                dst = sqrt(dst);
                myu = hl * inprod / (dst * dst + 0.01 * hl * hl);
                paix = (-a * cc * myu + b * myu * myu) / rou;
            } else
                paix = 0.0;
            for (k = 0; k < ndim; k++) tu[k] = tu[k] + c->mass[j] * paix * W(i, nj, k);
        }
        if (c->type[i] != 7)
            for (int k = 0; k < ndim; k++) c->ax[i * 3 + k] = c->ax[i * 3 + k] - tu[k];
    }
}

/* matrix_multiply / inverse_mat of the artificial stress:
 * CPP_9-5-artificialstress.cpp:13-26, 297-317 (the inverse is left zero when
 * |det| <= 1e-5) */
static void mat3_mul(double a[3][3], double b[3][3], double c[3][3])
{
    for (int r = 0; r < 3; r++)
        for (int q = 0; q < 3; q++) c[r][q] = a[r][0] * b[0][q] + a[r][1] * b[1][q] + a[r][2] * b[2][q];
}

static void mat3_inv(double A[3][3], double B[3][3])
{
    double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[1][0] * (A[0][1] * A[2][2] - A[0][2] * A[2][1])
        + A[2][0] * (A[0][1] * A[1][2] - A[0][2] * A[1][1]);
    if (fabs(det) > 1.0e-5) {
        B[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) / det;
        B[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) / det;
        B[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) / det;
        B[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) / det;
        B[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) / det;
        B[1][2] = (A[1][0] * A[0][2] - A[0][0] * A[1][2]) / det;
        B[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) / det;
        B[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) / det;
        B[2][2] = (A[0][0] * A[1][1] - A[1][0] * A[0][1]) / det;
    }
}

/* artificial_stress_2d / artificial_stress_3d: CPP_9-5-artificialstress.cpp:28-295.
 * R_i from the tensile principal stresses of each soil particle, then
 * a_i += sum_j m_j f_ij^n (R_i + R_j) grad W_ij over soil neighbours, with
 * f_ij^n = (W(q) / W(dr))^2.55. */
static void artificial_stress(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    int ndim = P->ndim;
    double xishu = P->art_stre_coe;
    const double pi_ = 3.141592653;   /* Header_Parameters.h:10 */
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] != 2) continue;
        double R[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double* s = &c->sig[i * 6];
        double rho = c->rho[i];
        if (ndim == 2) {
            double sita;
            if (fabs(s[0] - s[1]) < 1.0e-6) {
                if (s[3] > 0.0) sita = -pi_ * 0.78539816325;
                else if (s[3] < 0.0) sita = pi_ * 0.78539816325;
                else sita = 0.0;
            } else
                sita = 0.5 * atan(2.0 * s[3] / (s[0] - s[1]));
            double sxx = cos(sita) * cos(sita) * s[0] + 2.0 * sin(sita) * cos(sita) * s[3] + sin(sita) * sin(sita) * s[1];
            double syy = sin(sita) * sin(sita) * s[0] - 2.0 * sin(sita) * cos(sita) * s[3] + cos(sita) * cos(sita) * s[1];
            double rxx = (sxx > 0.0) ? -xishu * sxx / rho / rho : 0.0;
            double ryy = (syy > 0.0) ? -xishu * syy / rho / rho : 0.0;
            R[0][0] = rxx * cos(sita) * cos(sita) + ryy * sin(sita) * sin(sita);
            R[1][1] = rxx * sin(sita) * sin(sita) + ryy * cos(sita) * cos(sita);
            R[0][1] = (rxx - ryy) * sin(sita) * cos(sita);
            R[1][0] = R[0][1];
        } else {
            double sp[3] = {c->strep[i * 3], c->strep[i * 3 + 1], c->strep[i * 3 + 2]}, r[3];
            for (int k = 0; k < 3; k++) r[k] = (sp[k] > 0.0) ? -xishu * sp[k] / rho / rho : 0.0;
            double bi[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, bti[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            double tmp[3][3], st[3][3] = {{r[0], 0, 0}, {0, r[1], 0}, {0, 0, r[2]}};
            double be[3][3], bt[3][3];
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    be[a][b] = c->beta[i * 9 + a * 3 + b];
                    bt[a][b] = c->beta_ts[i * 9 + a * 3 + b];
                }
            mat3_inv(be, bi);
            mat3_inv(bt, bti);
            mat3_mul(bi, st, tmp);
            mat3_mul(tmp, bti, R);
        }
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) c->rij[i * 9 + a * 3 + b] = R[a][b];
    }
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] != 2) continue;
        double tu[3] = {0, 0, 0};
        const double* Ri = &c->rij[i * 9];
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[j] != 2) continue;
            double dst = 0.0;
            for (int k = 0; k < 3; k++) dst = dst + (c->xp[i * 3 + k] - c->xp[j * 3 + k]) * (c->xp[i * 3 + k] - c->xp[j * 3 + k]);
            dst = sqrt(dst);
            double hl = (c->hl[i] + c->hl[j]) * 0.5;
            double q = dst / hl, f;
            if (q >= 0.0 && q < 1.0) f = pow((0.666666666666667 - q * q + 0.5 * q * q * q) * 3.82300884955752, 2.55);
            else if (q >= 1.0 && q < 2.0) f = pow((2.0 - q) * (2.0 - q) * (2.0 - q) * 0.629737609329447, 2.55);
            else f = 0.0;
            const double* Rj = &c->rij[j * 9];
            const double* w = &W(i, nj, 0);
            double m = c->mass[j];
            if (ndim == 2) {
                tu[0] = tu[0] + m * f * (Ri[0] + Rj[0]) * w[0] + m * f * (Ri[1] + Rj[1]) * w[1];
                tu[1] = tu[1] + m * f * (Ri[3] + Rj[3]) * w[0] + m * f * (Ri[4] + Rj[4]) * w[1];
            } else {
                for (int a = 0; a < 3; a++)
                    tu[a] = tu[a] + m * f * (Ri[a * 3] + Rj[a * 3]) * w[0] + m * f * (Ri[a * 3 + 1] + Rj[a * 3 + 1]) * w[1]
                        + m * f * (Ri[a * 3 + 2] + Rj[a * 3 + 2]) * w[2];
            }
        }
        for (int k = 0; k < ndim; k++) c->ax[i * 3 + k] = c->ax[i * 3 + k] + tu[k];
    }
}

/* boundary_moving_stress_effect: CPP_9-4-derivation_stress.cpp:631-721 */
static void boundary_moving_stress_effect(orc_ctx* c)
{
    for (int i = 0; i < c->n; i++) {
        int ti = c->type[i];
        if (ti == 0 || ti == 7) continue;
        double tu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[j] != 0) continue;
            double a[6] = {0, 0, 0, 0, 0, 0};
            const double* s = &c->sig[i * 6];
            if (ti == 1 || ti == 3) {
                for (int k = 0; k < 6; k++) a[k] = s[k];
            } else if (ti == 2 || ti == 4) {
                double satu = c->satu[i];
                a[0] = s[0] - satu * c->prew[i] + (1 - satu) * c->prea[i];
                a[1] = s[1] - satu * c->prew[i] + (1 - satu) * c->prea[i];
                a[2] = s[2] - satu * c->prew[i] + (1 - satu) * c->prea[i];
                a[3] = s[3]; a[4] = s[4]; a[5] = s[5];
            }
            stress_pair(tu, c->mass[j], a, a, c->rho[j], c->rho[i], &W(i, nj, 0), 1.0);
        }
        c->ax[i * 3 + 0] += tu[0][0] + tu[0][1] + tu[0][2];
        c->ax[i * 3 + 1] += tu[1][0] + tu[1][1] + tu[1][2];
        c->ax[i * 3 + 2] += tu[2][0] + tu[2][1] + tu[2][2];
    }
}

/* boundary_stress_effect_tran: CPP_9-4-derivation_stress.cpp:725-846, the wall
 * stress of flbndy 3/4/13/14 with the wall's Shepard-extrapolated stress of
 * the particle's phase */
static void boundary_stress_effect_tran(orc_ctx* c)
{
    for (int i = 0; i < c->n; i++) {
        int ti = c->type[i];
        if (ti == 0 || ti == 7) continue;
        double tu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double* wall = ti == 1 ? c->sb_water : ti == 2 ? c->sb_soil : ti == 3 ? c->sb_air : ti == 4 ? c->sb_struct : 0;
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[j] != 0) continue;
            double ai[6] = {0, 0, 0, 0, 0, 0}, aj[6] = {0, 0, 0, 0, 0, 0};
            const double* s = &c->sig[i * 6];
            if (ti == 2) {
                double satu = c->satu[i];
                ai[0] = s[0] - satu * c->prew[i] + (1 - satu) * c->prea[i];
                ai[1] = s[1] - satu * c->prew[i] + (1 - satu) * c->prea[i];
                ai[2] = s[2] - satu * c->prew[i] + (1 - satu) * c->prea[i];
                ai[3] = s[3]; ai[4] = s[4]; ai[5] = s[5];
            } else if (ti == 1 || ti == 3 || ti == 4) {
                for (int k = 0; k < 6; k++) ai[k] = s[k];
            }
            if (wall)
                for (int k = 0; k < 6; k++) aj[k] = wall[j * 6 + k];
            stress_pair(tu, c->mass[j], aj, ai, c->rho[j], c->rho[i], &W(i, nj, 0), 1.0);
        }
        c->ax[i * 3 + 0] += tu[0][0] + tu[0][1] + tu[0][2];
        c->ax[i * 3 + 1] += tu[1][0] + tu[1][1] + tu[1][2];
        c->ax[i * 3 + 2] += tu[2][0] + tu[2][1] + tu[2][2];
    }
}

/* boundary_effect_free_struct: CPP_9-4-derivation_stress.cpp:900-990, the wall
 * stress of flbndy 5 (and any flbndy outside 1-4, 13, 14): the particle's own
 * stress mirrored into the wall, with the shear components of a fluid's
 * mirror negated */
static void boundary_effect_free_struct(orc_ctx* c)
{
    for (int i = 0; i < c->n; i++) {
        int ti = c->type[i];
        if (ti == 0 || ti == 7) continue;
        double tu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[j] != 0) continue;
            double ai[6] = {0, 0, 0, 0, 0, 0}, aj[6] = {0, 0, 0, 0, 0, 0};
            const double* s = &c->sig[i * 6];
            if (ti == 1 || ti == 3) {
                for (int k = 0; k < 6; k++) ai[k] = s[k];
                aj[0] = ai[0]; aj[1] = ai[1]; aj[2] = ai[2];
                aj[3] = -ai[3]; aj[4] = -ai[4]; aj[5] = -ai[5];
            } else if (ti == 2 || ti == 4) {
                double satu = c->satu[i];
                ai[0] = s[0] - satu * c->prew[i] + (1 - satu) * c->prea[i];
                ai[1] = s[1] - satu * c->prew[i] + (1 - satu) * c->prea[i];
                ai[2] = s[2] - satu * c->prew[i] + (1 - satu) * c->prea[i];
                ai[3] = s[3]; ai[4] = s[4]; ai[5] = s[5];
                for (int k = 0; k < 6; k++) aj[k] = ai[k];
            }
            stress_pair(tu, c->mass[j], aj, ai, c->rho[j], c->rho[i], &W(i, nj, 0), 1.0);
        }
        c->ax[i * 3 + 0] += tu[0][0] + tu[0][1] + tu[0][2];
        c->ax[i * 3 + 1] += tu[1][0] + tu[1][1] + tu[1][2];
        c->ax[i * 3 + 2] += tu[2][0] + tu[2][1] + tu[2][2];
    }
}

/* coupled_Water_Soil_Structure (ss acc_type 2): CPP_9-4-derivation_stress.cpp:
 * 507-629, the stress divergence between structure and soil / water pairs
 * (plain stresses; water with a structure neighbour takes the difference form) */
static void coupled_water_soil_structure(orc_ctx* c)
{
    for (int i = 0; i < c->n; i++) {
        int ti = c->type[i];
        if (!(ti == 4 || ti == 2 || ti == 1)) continue;
        double tu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), tj = c->type[j];
            double sg = 0.0;
            if ((ti == 4 && tj == 2) || (ti == 2 && tj == 4) || (ti == 4 && tj == 1)) sg = 1.0;
            else if (ti == 1 && tj == 4) sg = -1.0;
            else continue;
            stress_pair(tu, c->mass[j], &c->sig[j * 6], &c->sig[i * 6], c->rho[j], c->rho[i], &W(i, nj, 0), sg);
        }
        c->ax[i * 3 + 0] += tu[0][0] + tu[0][1] + tu[0][2];
        c->ax[i * 3 + 1] += tu[1][0] + tu[1][1] + tu[1][2];
        c->ax[i * 3 + 2] += tu[2][0] + tu[2][1] + tu[2][2];
    }
}

/* Soil-water drag coefficient beta of interact2 (Tsuji et al. 1993 / Shi et al.
 * 2018, CPP_10-interact1.cpp:154-176) and interact3 (Peng et al. 2017,
 * :294-306), for soil particle s and water particle w; rho_w is the density
 * the reference reads (pPar[j].rho with i soil, pPar[i].rho with i water). */
static double drag_beta(const orc_ctx* c, int form, int s, int w, double mag_v, double rho_w)
{
    double por = c->porosity[s], ds = c->so[s].ds, dens = c->fl[w].dens, vis = c->fl[w].vis;
    double re, cd, beta;
    if (form == 2) {
        re = mag_v * dens * por * ds / vis;
        if (re > 1000.0) cd = 0.43;
        else if (fabs(re) > 0.0001) cd = 24.0 * (1.0 + 0.15 * pow(re, 0.687)) / re;
        else cd = 0.0;
        if (por <= 0.8) {
            beta = 150.0 * (1.0 - por) * (1.0 - por) / por / por / ds / ds * vis;
            beta = beta + 1.75 * (1.0 - por) / ds / por * dens * mag_v;
        } else
            beta = 0.75 * cd * mag_v * dens * (1.0 - por) / ds * pow(por, -2.7);
    } else {
        re = mag_v * dens * ds / vis;
        cd = por * por * por * ds * ds * 0.0066666667 / (1.0 - por) / (1.0 - por);
        if (re > 60.0) beta = vis / cd + 1.75 / sqrt(150.0) * rho_w * mag_v / sqrt(cd) / pow(por, 1.5);
        else beta = vis / cd;
    }
    return beta;
}

/* interact1 (Darcy, CPP_10-interact1.cpp:15-110), interact2 (Tsuji, :114-263)
 * and interact3 (Peng, :267-405): the same pass, limiter and soil-air term;
 * they differ in the soil-water pair term. */
static void interact(orc_ctx* c, int form)
{
    const sphgpu_params* P = &c->P;
    int ndim = P->ndim;
    double xishu = P->interc, dt = P->dt;
    double g_acc = sqrt(P->gx * P->gx + P->gy * P->gy + P->gz * P->gz);
    for (int i = 0; i < c->n; i++) {
        double tu[3] = {0, 0, 0};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), k;
            if (c->type[i] == c->type[j]) continue;
            double inprod = 0.0, mag_v = 0.0, dx[3], dvx[3];
            for (k = 0; k < ndim; k++) {
                dx[k] = c->xp[i * 3 + k] - c->xp[j * 3 + k];
                dvx[k] = c->vxp[i * 3 + k] - c->vxp[j * 3 + k];
                mag_v = mag_v + dvx[k] * dvx[k];
                inprod = inprod + dx[k] * dvx[k];
            }
            mag_v = sqrt(mag_v);
            if (!(inprod < 0)) continue;
            int ti = c->type[i], tj = c->type[j];
            double w3 = W(i, nj, 3);
            if (form > 1 && ((ti == 2 && tj == 1) || (ti == 1 && tj == 2))) {
                double beta = (ti == 2) ? drag_beta(c, form, i, j, mag_v, c->rho[j]) : drag_beta(c, form, j, i, mag_v, c->rho[i]);
                for (k = 0; k < ndim; k++)
                    tu[k] = tu[k] + c->mass[j] / c->rho[j] * w3 * beta * (c->vxp[i * 3 + k] - c->vxp[j * 3 + k]);
            } else if (ti == 2 && tj == 1) {
                for (k = 0; k < ndim; k++)
                    tu[k] = tu[k] + c->satu[i] * c->satu[i] * c->porosity[i] * c->porosity[i] * c->fl[j].dens * g_acc * dvx[k] / c->cop[i] * c->mass[j] / c->rho[j] * w3;
            } else if (ti == 1 && tj == 2) {
                for (k = 0; k < ndim; k++)
                    tu[k] = tu[k] + c->satu[j] * c->satu[j] * c->porosity[j] * c->porosity[j] * c->fl[i].dens * g_acc * dvx[k] / c->cop[j] * c->mass[j] / c->rho[j] * w3;
            } else if (ti == 2 && tj == 3) {
                for (k = 0; k < ndim; k++)
                    tu[k] = tu[k] + (1 - c->satu[i]) * (1 - c->satu[i]) * c->porosity[i] * c->porosity[i] * c->fl[j].dens * g_acc * dvx[k] * 2000 * c->mass[j] / c->rho[j] * w3;
            } else if (ti == 3 && tj == 2) {
                for (k = 0; k < ndim; k++)
                    tu[k] = tu[k] + (1 - c->satu[j]) * (1 - c->satu[j]) * c->porosity[j] * c->porosity[j] * c->fl[i].dens * g_acc * dvx[k] * 2000 * c->mass[j] / c->rho[j] * w3;
            }
        }
        if (c->type[i] != 0 && c->type[i] != 7) {
            for (int k = 0; k < ndim; k++) {
                double* ax = &c->ax[i * 3 + k];
                double axp = c->axp[i * 3 + k], vxp = c->vxp[i * 3 + k];
                c->interf[i * 3 + k] = tu[k];
                double vx1 = vxp + 0.5 * (axp + *ax) * dt;
                double vx2 = vxp + 0.5 * (axp + *ax - c->interf[i * 3 + k] * xishu / c->rho[i]) * dt;
                if (vx1 * vx2 <= 0.0) {
                    c->interf[i * 3 + k] = 0.0;
                    *ax = -2.0 * vxp / dt - axp;
                } else
                    *ax -= c->interf[i * 3 + k] * xishu / c->rho[i];
            }
        }
    }
}

/* soil_damping_geostress: CPP_9-4-derivation_stress.cpp:849-896 */
static void soil_damping_geostress(orc_ctx* c)
{
    int ndim = c->P.ndim;
    double dt = c->P.dt;
    for (int i = 0; i < c->n; i++) {
        if (!(c->type[i] == 2 || c->type[i] == 4)) continue;
        double cd = c->cd[i], damp[3] = {0, 0, 0};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[i] == c->type[j])
                for (int k = 0; k < ndim; k++)
                    damp[k] = damp[k] + c->mass[j] / c->rho[j] * cd * (c->vxp[i * 3 + k] - c->vxp[j * 3 + k]) * W(i, nj, 3);
        }
        for (int k = 0; k < ndim; k++) {
            double* ax = &c->ax[i * 3 + k];
            double axp = c->axp[i * 3 + k], vxp = c->vxp[i * 3 + k];
            double vx1 = vxp + 0.5 * (axp + *ax) * dt;
            double vx2 = vxp + 0.5 * (axp + *ax - damp[k]) * dt;
            if (vx1 * vx2 <= 0.0) *ax = -2.0 * vxp / dt - axp;
            else *ax -= damp[k];
        }
    }
}

/* ff_stress_2d_solid / _3d_solid: CPP_19-FreeFieldParticles.cpp:21-76 (the
 * soil form's copy, CPP_19-FreeFieldParticles_soil.cpp:21-68, is the same) */
static void ff_stress(int ndim, double* sg, const double* va, const double* vb, double e, double poi, double dens,
                      int type)
{
    double g = e * 0.5 / (1 + poi);
    double k = e * 0.333333333333333 / (1 - 2.0 * poi);
    double c_p = sqrt((k + 4.0 * g * 0.333333333333333) / dens);
    double c_s = sqrt(g / dens);
    sg[0] = 0.0; sg[1] = 0.0; sg[2] = 0.0;
    if (ndim == 2) {
        if (type == 1) {
            sg[0] = -c_p * dens * (va[0] - vb[0]);
            sg[1] = -c_s * dens * (va[1] - vb[1]);
        } else if (type == 2) {
            sg[0] = -c_s * dens * (va[0] - vb[0]);
            sg[1] = -c_p * dens * (va[1] - vb[1]);
        }
    } else {
        if (type == 1) {
            sg[0] = -c_p * dens * (va[0] - vb[0]);
            sg[1] = -c_s * dens * (va[1] - vb[1]);
            sg[2] = -c_s * dens * (va[2] - vb[2]);
        } else if (type == 2) {
            sg[0] = -c_s * dens * (va[0] - vb[0]);
            sg[1] = -c_p * dens * (va[1] - vb[1]);
            sg[2] = -c_s * dens * (va[2] - vb[2]);
        } else if (type == 3) {
            sg[0] = -c_s * dens * (va[0] - vb[0]);
            sg[1] = -c_s * dens * (va[1] - vb[1]);
            sg[2] = -c_p * dens * (va[2] - vb[2]);
        }
    }
}

/* free_field_solid of the walls: CPP_19-FreeFieldParticles.cpp:79-141.  The
 * elastic constants are those of pFFBound, a default-constructed Para_Soil
 * (e = poi = 0, CPP_1-SPHLoops.cpp:253; Class_ParticleProperty.cpp:28-31) */
static void free_field_walls(orc_ctx* c)
{
    const int ndim = c->P.ndim;
    const double e = 0.0, poi = 0.0;
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] != 2) continue;
        double t[3] = {0, 0, 0};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (!(c->type[j] == 0 && c->matype[j] == 5)) continue;
            double sg[3];
            ff_stress(ndim, sg, &c->vx[i * 3], &c->interfss[j * 3], e, poi, c->rho[j], c->permtype[j]);
            for (int k = 0; k < 3; k++) t[k] = t[k] + c->mass[j] / c->rho[j] * sg[k] / c->rho[i] * W(i, nj, k);
        }
        for (int k = 0; k < ndim; k++) c->ax[i * 3 + k] = c->ax[i * 3 + k] + t[k];
    }
}

/* free_field_solid of the soil: CPP_19-FreeFieldParticles_soil.cpp:71-175,
 * between soil of matype >= 50 (the free-field columns) and the rest */
static void free_field_soil(orc_ctx* c)
{
    const int ndim = c->P.ndim;
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] != 2) continue;
        const int ff = c->matype[i] >= 50;
        double t[3] = {0, 0, 0};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (!(c->type[j] == 2 && (c->matype[j] >= 50) != ff)) continue;
            double sg[3];
            if (!ff)
                ff_stress(ndim, sg, &c->vx[i * 3], &c->vx[j * 3], c->so[j].e, c->so[j].poi, c->rho[j], c->permtype[j]);
            else
                ff_stress(ndim, sg, &c->vx[j * 3], &c->vx[i * 3], c->so[i].e, c->so[i].poi, c->rho[i], c->permtype[i]);
            for (int k = 0; k < 3; k++) t[k] = t[k] + c->mass[j] / c->rho[j] * sg[k] / c->rho[i] * W(i, nj, k);
        }
        for (int k = 0; k < ndim; k++) c->ax[i * 3 + k] = c->ax[i * 3 + k] + t[k];
    }
}

/* the load of time t: 0 outside [sttime, edtime], else 1 (largest magnitude
 * under 1000) or 2, the entry in v (CPP_9-1:21-35, 85-99) */
static int vib_load(const orc_ctx* c, double* v)
{
    double time1 = c->t - c->vib_sttime, time2 = c->t - c->vib_edtime;
    if (!(time1 >= 0.0 && time2 <= 0.0)) return 0;
    double q = time1 / c->vib_ttime * (double)c->vib_nsteps;
    int nstep = (q >= (double)(c->vib_nsteps - 1)) ? c->vib_nsteps - 1 : (int)q;
    for (int k = 0; k < 3; k++) v[k] = c->vib_loads[nstep * 3 + k];
    double m = fmax(0.0, fabs(v[0]));
    m = fmax(m, fabs(v[1]));
    m = fmax(m, fabs(v[2]));
    return m < 1000.0 ? 1 : 2;
}

/* vibration_acceleration (CPP_9-1:10-78, flv 1, walls of matype 3 and 5) and
 * vibration_velocity (CPP_9-1:80-160, flv 2, walls of matype 4 and 5) */
static void vibration_load(orc_ctx* c, int velocity)
{
    const int ndim = c->P.ndim;
    double v[3];
    const int ld = vib_load(c, v);
    for (int i = 0; i < c->n; i++) {
        const int m = c->matype[i];
        if (c->type[i] != 0 || !(m == (velocity ? 4 : 3) || m == 5)) continue;
        for (int k = 0; k < ndim; k++) {
            if (ld == 1) {
                if (velocity) c->interfss[i * 3 + k] = v[k];
                else c->interf[i * 3 + k] = v[k];
            } else {
                c->interf[i * 3 + k] = 0.0;
                c->interfss[i * 3 + k] = 0.0;
            }
        }
    }
}

/* soil_damping_vibration: CPP_9-1-acceleration_vibration.cpp:162-224 */
static void soil_damping_vibration(orc_ctx* c)
{
    const int ndim = c->P.ndim;
    const double dt = c->P.dt;
    for (int i = 0; i < c->n; i++) {
        if (!(c->type[i] == 2 || c->type[i] == 4)) continue;
        double damp[3] = {0, 0, 0}, tempdown = 0.0;
        const double stiff = c->stiff[i];
        const double cd = c->so[i].damp1 + c->so[i].damp2 * sqrt(stiff / c->rhop[i] / c->hl[i] / c->hl[i]);
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[i] == c->type[j]) {
                for (int k = 0; k < ndim; k++)
                    damp[k] = damp[k] + c->mass[j] / c->rho[j] * cd * (c->vxp[i * 3 + k] - c->vxp[j * 3 + k]) * W(i, nj, 3);
                tempdown = tempdown + c->mass[j] / c->rho[j] * W(i, nj, 3);
            }
        }
        for (int k = 0; k < ndim; k++) {
            if (fabs(tempdown) < 1.0e-7) tempdown = 1.0e-7;
            double* ax = &c->ax[i * 3 + k];
            double axp = c->axp[i * 3 + k], vxp = c->vxp[i * 3 + k];
            double vx1 = vxp + 0.5 * (axp + *ax) * dt;
            double vx2 = vxp + 0.5 * (axp + *ax - damp[k] / tempdown) * dt;
            if (vx1 * vx2 <= 0.0) *ax = -2.0 * vxp / dt - axp;
            else *ax -= damp[k] / tempdown;
        }
    }
}

/* veocity_update: CPP_11-xsph.cpp:11-142 */
static void velocity_update(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    int ndim = P->ndim, l = c->l, inip = P->inip;
    double dt = P->dt;
    for (int i = 0; i < c->n; i++) {
        int ti = c->type[i], mt = c->matype[i];
        double *vx = &c->vx[i * 3], *vxp = &c->vxp[i * 3], *ax = &c->ax[i * 3], *axp = &c->axp[i * 3];
        double *itf = &c->interf[i * 3], *itss = &c->interfss[i * 3];
        if (P->if_move == 0) {
            if (ti == 0 && mt < 2) {
                for (int k = 0; k < ndim; k++) { itf[k] = 0.0; double ath = (itf[k] + itf[k]) * 0.5; itss[k] = itss[k] + ath * dt; }
            } else if (ti == 0 && mt == 3) {
                for (int k = 0; k < ndim; k++) { double ath = (itf[k] + itf[k]) * 0.5; itss[k] = itss[k] + ath * dt; }
            } else if (ti == 0 && mt == 5 && P->flv == 1) {
                for (int k = 0; k < ndim; k++) { double ath = (itf[k] + itf[k]) * 0.5; itss[k] = itss[k] + ath * dt; }
            } else if (ti != 0) {
                for (int k = 0; k < ndim; k++) { double ath = (axp[k] + ax[k]) * 0.5; vx[k] = vxp[k] + ath * dt; }
            }
        } else if (P->if_move == 1) {
            if ((ti == 0 && mt == 2) && l > inip) {
                for (int k = 0; k < ndim; k++) itss[k] = P->move_vx[k];
            } else if (ti == 0) {
                for (int k = 0; k < ndim; k++) itss[k] = 0.0;
            } else {
                for (int k = 0; k < ndim; k++) { double ath = (axp[k] + ax[k]) * 0.5; vx[k] = vxp[k] + ath * dt; }
            }
        } else if (P->if_move == 2 || P->if_move == 3) {
            int tmove = (P->if_move == 2) ? 2 : 4;
            if ((ti == tmove && c->etype[i] == 5) && l > inip) {
                for (int k = 0; k < ndim; k++) { axp[k] = 0.0; vxp[k] = P->move_vx[k]; vx[k] = P->move_vx[k]; ax[k] = 0.0; }
            }
            for (int k = 0; k < ndim; k++) { double ath = (axp[k] + ax[k]) * 0.5; vx[k] = vxp[k] + ath * dt; }
        }
    }
}

/* xsph: CPP_11-xsph.cpp:145-256 (flbndy 1 virtual-velocity form) */
static void xsph(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    int ndim = P->ndim, bndytype = P->flbndy;
    for (int i = 0; i < c->n; i++) {
        double tu[3] = {0, 0, 0}, down = 0.0, xishu = 0.0, vxj[3];
        int ti = c->type[i];
        for (int k = 0; k < ndim; k++) c->vx_temp[i * 3 + k] = 0.0;
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), tj = c->type[j], k;
            double w3 = W(i, nj, 3);
            if (ti == tj && (ti != 0 && ti != 7)) {
                if (ti == 1) xishu = P->xsph[0];
                else if (ti == 2) xishu = P->xsph[1];
                else if (ti == 3) xishu = P->xsph[2];
                else if (ti == 4) xishu = P->xsph[1];
                for (k = 0; k < ndim; k++)
                    tu[k] = tu[k] + xishu * c->mass[j] * (c->vx[j * 3 + k] - c->vx[i * 3 + k]) * w3 / c->rho[j];
                down = down + c->mass[j] * w3 / c->rho[j];
            } else if ((ti == 1 || ti == 2 || ti == 3 || ti == 4) && tj == 0) {
                vxj[0] = vxj[1] = vxj[2] = 0.0;
                if (bndytype == 1) { vxj[0] = c->vx[i * 3]; vxj[1] = c->vx[i * 3 + 1]; vxj[2] = c->vx[i * 3 + 2]; }
                (void)vxj;   /* computed and unused by the reference (:187-233) */
                if (ti == 1) xishu = 0.006;
                else if (ti == 2) xishu = P->xsph[1] / 5.0;
                else if (ti == 3) xishu = 0.006;
                else if (ti == 4) xishu = P->xsph[1] / 5.0;
                for (k = 0; k < ndim; k++)
                    tu[k] = tu[k] + xishu * c->mass[j] * (c->vx[j * 3 + k] - c->vx[i * 3 + k]) * w3 / c->rho[j];
                down = down + c->mass[j] * w3 / c->rho[j];
            }
        }
        if (ti != 0 && ti != 7) {
            if (fabs(down) > 1.0e-7 && (ti == 2 || ti == 4))
                for (int k = 0; k < ndim; k++) c->vx_temp[i * 3 + k] = c->vx[i * 3 + k] + tu[k] / down;
            else
                for (int k = 0; k < ndim; k++) c->vx_temp[i * 3 + k] = c->vx[i * 3 + k] + tu[k];
        }
    }
    for (int i = 0; i < c->n; i++)
        if (c->type[i] != 0 && c->type[i] != 7)
            for (int k = 0; k < ndim; k++) c->vx[i * 3 + k] = c->vx_temp[i * 3 + k];
}

/* tmboundary: CPP_13-boundary.cpp:125-177 */
static void tmboundary(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    int ndim = P->ndim;
    double dr = P->dr, a = 0.30, b = 0.30;
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] == 0 || c->type[i] == 7) continue;
        double tu[3] = {0, 0, 0};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), k;
            if (c->type[j] != 0) continue;
            double inprod = 0.0, dst = 0.0;
            for (k = 0; k < ndim; k++) {
                inprod = inprod + (c->vx[i * 3 + k] - c->interfss[j * 3 + k]) * (c->xp[i * 3 + k] - c->xp[j * 3 + k]);
                dst = dst + (c->xp[i * 3 + k] - c->xp[j * 3 + k]) * (c->xp[i * 3 + k] - c->xp[j * 3 + k]);
            }
            if (inprod < 0.0) {
                dst = sqrt(dst);
                double db = a * dr;
                double beta = 1 + db / (dst - b * dr);
                beta = fmin(1.5, beta);
                for (k = 0; k < ndim; k++)
                    tu[k] = tu[k] + (1 - beta) * (c->xp[i * 3 + k] - c->xp[j * 3 + k]) * inprod / dst / dst;
            }
        }
        for (int k = 0; k < ndim; k++) c->vx[i * 3 + k] = c->vx[i * 3 + k] + tu[k];
    }
}

/* velocity_set_domain: CPP_13-boundary.cpp:71-122, fluid particles only, with
 * a = b = coe_bndy */
static void velocity_set_domain(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    int ndim = P->ndim;
    double dr = P->dr, a = P->coe_bndy, b = P->coe_bndy;
    for (int i = 0; i < c->n; i++) {
        if (!(c->type[i] == 1 || c->type[i] == 3)) continue;
        double tu[3] = {0, 0, 0};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), k;
            if (c->type[j] != 0) continue;
            double inprod = 0.0, dst = 0.0;
            for (k = 0; k < ndim; k++) {
                inprod = inprod + (c->vx[i * 3 + k] - c->interfss[j * 3 + k]) * (c->xp[i * 3 + k] - c->xp[j * 3 + k]);
                dst = dst + (c->xp[i * 3 + k] - c->xp[j * 3 + k]) * (c->xp[i * 3 + k] - c->xp[j * 3 + k]);
            }
            if (inprod < 0.0) {
                dst = sqrt(dst);
                double db = a * dr;
                double beta = 1 + db / (dst - b * dr);
                beta = fmin(1.5, beta);
                for (k = 0; k < ndim; k++)
                    tu[k] = tu[k] + (1 - beta) * (c->xp[i * 3 + k] - c->xp[j * 3 + k]) * inprod / dst / dst;
            }
        }
        for (int k = 0; k < ndim; k++) c->vx[i * 3 + k] = c->vx[i * 3 + k] + tu[k];
    }
}

/* the wall particles of i's list in list order with their distances, sorted
 * as clParti_Pair::dist_sorting does (Class_particle.cpp:343-359): four
 * passes that swap the ids but not the distances */
static int wall_pairs_sorted(const orc_ctx* c, int i, int* ids, int* last_id)
{
    double dsts[NB];
    int k = 0;
    *last_id = 0;
    for (int nj = 1; nj <= c->ninflu[i]; nj++) {
        int j = NBR(i, nj);
        if (c->type[j] != 0) continue;
        double dx = c->xp[i * 3] - c->xp[j * 3], dy = c->xp[i * 3 + 1] - c->xp[j * 3 + 1];
        double dz = c->xp[i * 3 + 2] - c->xp[j * 3 + 2];
        double d = dx * dx + dy * dy + dz * dz;
        ids[k] = j;
        dsts[k] = sqrt(d);
        k++;
        if (c->matype[j] > 2) *last_id = j;
    }
    for (int a = 0; a < 4; a++)
        for (int b = a + 1; b < k; b++)
            if (dsts[a] > dsts[b]) { int t = ids[a]; ids[a] = ids[b]; ids[b] = t; }
    return k;
}

/* tm_boundary_2d / tm_boundary_3d: CPP_13-boundary.cpp:179-615.  The line of
 * the two nearest walls (2-D) keeps the C = 1 of clLine() (cal_line sets only
 * A and B); the plane through the three nearest walls (3-D) keeps the D its
 * variable last held: 1 from clPlane(), or the value plane_two_points set,
 * which persists through later particles of the same loop in the reference
 * (ORC_INPLACE); in ORC_JACOBI order every particle starts from D = 1.  The
 * walls' Shepard sums keep the reference's [0][0] index in components 1 and 2. */
static void tm_boundary(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    const int nd = P->ndim;
    const double dr = P->dr;
    double plane_d = 1.0;
    int ids[NB];
    for (int i = 0; i < c->n; i++) {
        int ti = c->type[i];
        if (ti == 0 || ti == 7) continue;
        int id = 0;
        int total = wall_pairs_sorted(c, i, ids, &id);
        double* vb = &c->vel_bndy[i * 3];
        const double* vi = &c->vx[i * 3];
        if (total >= (nd == 2 ? 2 : 3)) {
            const double* p4 = &c->xp[i * 3];
            const double* p1 = &c->xp[ids[0] * 3];
            const double* p2 = &c->xp[ids[1] * 3];
            double dst;
            if (nd == 2) {
                /* cal_line (:645-650) and cal_dpline (:617-628) */
                double den = p2[1] * p1[0] - p1[1] * p2[0];
                double A = (p1[1] - p2[1]) / den, B = (p2[0] - p1[0]) / den, C = 1.0;
                double num = fabs(A * p4[0] + B * p4[1] + C);
                double tmp = sqrt(A * A + B * B);
                dst = (tmp > 1.0e-3) ? num / tmp : 0.0;
            } else {
                const double* p3 = &c->xp[ids[2] * 3];
                double pc1[3], pc2[3], A, B, C;
                /* cal_plane (:653-666) of (p1, p2, p4) and (p1, p3, p4) */
                double den1 = -p1[0] * (p2[1] * p4[2] - p4[1] * p2[2]) - p2[0] * (p4[1] * p1[2] - p1[1] * p4[2]) -
                              p4[0] * (p1[1] * p2[2] - p2[1] * p1[2]);
                pc1[0] = p1[1] * (p2[2] - p4[2]) + p2[1] * (p4[2] - p1[2]) + p4[1] * (p1[2] - p2[2]);
                pc1[1] = p1[2] * (p2[0] - p4[0]) + p2[2] * (p4[0] - p1[0]) + p4[2] * (p1[0] - p2[0]);
                pc1[2] = p1[0] * (p2[1] - p4[1]) + p2[0] * (p4[1] - p1[1]) + p4[0] * (p1[1] - p2[1]);
                pc1[0] = pc1[0] / den1; pc1[1] = pc1[1] / den1; pc1[2] = pc1[2] / den1;
                double den2 = -p1[0] * (p3[1] * p4[2] - p4[1] * p3[2]) - p3[0] * (p4[1] * p1[2] - p1[1] * p4[2]) -
                              p4[0] * (p1[1] * p3[2] - p3[1] * p1[2]);
                pc2[0] = p1[1] * (p3[2] - p4[2]) + p3[1] * (p4[2] - p1[2]) + p4[1] * (p1[2] - p3[2]);
                pc2[1] = p1[2] * (p3[0] - p4[0]) + p3[2] * (p4[0] - p1[0]) + p4[2] * (p1[0] - p3[0]);
                pc2[2] = p1[0] * (p3[1] - p4[1]) + p3[0] * (p4[1] - p1[1]) + p4[0] * (p1[1] - p3[1]);
                pc2[0] = pc2[0] / den2; pc2[1] = pc2[1] / den2; pc2[2] = pc2[2] / den2;
                double cs = pc1[0] * pc2[0] + pc1[1] * pc2[1] + pc1[2] * pc2[2];
                cs = cs / sqrt(pc1[0] * pc1[0] + pc1[1] * pc1[1] + pc1[2] * pc1[2]) /
                     sqrt(pc2[0] * pc2[0] + pc2[1] * pc2[1] + pc2[2] * pc2[2]);
                if (c->mode == ORC_JACOBI) plane_d = 1.0;
                if (fabs(cs) > 0.999999) {
                    /* plane_two_points(p4, p1) (:684-708) */
                    double a = p4[0] - p1[0], b = p4[1] - p1[1], cc = p4[2] - p1[2];
                    double tmp = -a * p1[0] - b * p1[1] - cc * p1[2];
                    if (fabs(tmp) > 1.0e-6) { A = a / tmp; B = b / tmp; C = cc / tmp; plane_d = 1.0; }
                    else { A = a; B = b; C = cc; plane_d = 0.0; }
                } else {
                    double den = -p1[0] * (p2[1] * p3[2] - p3[1] * p2[2]) - p2[0] * (p3[1] * p1[2] - p1[1] * p3[2]) -
                                 p3[0] * (p1[1] * p2[2] - p2[1] * p1[2]);
                    A = p1[1] * (p2[2] - p3[2]) + p2[1] * (p3[2] - p1[2]) + p3[1] * (p1[2] - p2[2]);
                    B = p1[2] * (p2[0] - p3[0]) + p2[2] * (p3[0] - p1[0]) + p3[2] * (p1[0] - p2[0]);
                    C = p1[0] * (p2[1] - p3[1]) + p2[0] * (p3[1] - p1[1]) + p3[0] * (p1[1] - p2[1]);
                    A = A / den; B = B / den; C = C / den;
                }
                /* cal_dpplane (:631-642) */
                double num = fabs(A * p4[0] + B * p4[1] + C * p4[2] + plane_d);
                double tmp = sqrt(A * A + B * B + C * C);
                dst = (tmp > 1.0e-3) ? num / tmp : 0.0;
            }
            double da = (dst > 0.6 * dr) ? dst - 0.5 * dr : 0.1 * dr;
            double db = 0.5 * dr, beta;
            if (fabs(da) > 1.0e-6) { beta = 1.0 + db / da; beta = fmin(1.5, beta); }
            else beta = 1.5;
            const double* its = &c->interfss[id * 3];
            vb[0] = (1.0 - beta) * vi[0] + beta * its[0];
            vb[1] = (1.0 - beta) * vi[1] + beta * its[1];
            vb[2] = (nd == 2) ? 0.0 : (1.0 - beta) * vi[2] + beta * its[2];
        } else {
            vb[0] = vi[0]; vb[1] = vi[1]; vb[2] = vi[2];
        }
    }
    /* the walls: Shepard sums of the moving particles' virtual velocities per phase */
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] != 0) continue;
        double up[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, down[4] = {0, 0, 0, 0};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), tj = c->type[j];
            if (tj < 1 || tj > 4) continue;
            int p = tj - 1;
            const double* vb = &c->vel_bndy[j * 3];
            double w3 = W(i, nj, 3), mj = c->mass[j], rj = c->rho[j];
            up[p][0] = up[p][0] + mj * vb[0] * w3 / rj;
            up[p][1] = up[p][0] + mj * vb[1] * w3 / rj;
            up[p][2] = up[p][0] + mj * vb[2] * w3 / rj;
            down[p] = down[p] + mj * w3 / rj;
        }
        double* out[4] = {c->vb_water, c->vb_soil, c->vb_air, c->vb_struct};
        for (int p = 0; p < 4; p++)
            for (int k = 0; k < 3; k++) out[p][i * 3 + k] = (fabs(down[p]) > 1.0e-6) ? up[p][k] / down[p] : 0.0;
    }
}

/* ------------------------------------------------------------------------- */
/* soil-structure contact: interaction_ss_rigid / _deformable / _penalty      */
/* (CPP_10-1-interact_ss.cpp:17-1036) with their geometry helpers (:1039-1369) */
/* in the order one thread runs them: the forces a structure particle takes   */
/* from its contacting particles accumulate in particle order.               */

typedef struct { double x, y, z; } orc_pt;

static double ss_dpline(orc_pt p, double A, double B, double C)
{   /* cal_dpline (:1224-1236) */
    double dst = fabs(A * p.x + B * p.y + C), tmp = sqrt(A * A + B * B);
    return (tmp > 1.0e-3) ? dst / tmp : 0.0;
}

static double ss_dpplane(orc_pt p, double A, double B, double C, double D)
{   /* cal_dpplane (:1238-1250) */
    double dst = fabs(A * p.x + B * p.y + C * p.z + D), tmp = sqrt(A * A + B * B + C * C);
    return (tmp > 1.0e-3) ? dst / tmp : 0.0;
}

/* linear_interpolate (:1187-1202) */
static void ss_interp(orc_pt P1, orc_pt P2, orc_pt r, double m1, double m2, const double* v1, const double* v2,
                      double* m, double* v)
{
    double xk1 = 0.0;
    double xk2 = sqrt((P2.x - P1.x) * (P2.x - P1.x) + (P2.y - P1.y) * (P2.y - P1.y) + (P2.z - P1.z) * (P2.z - P1.z));
    double xp = sqrt((r.x - P1.x) * (r.x - P1.x) + (r.y - P1.y) * (r.y - P1.y) + (r.z - P1.z) * (r.z - P1.z));
    *m = (m1 * fabs(xp - xk2) + m2 * fabs(xp - xk1)) / fabs(xk2 - xk1);
    for (int k = 0; k < 3; k++) v[k] = (v1[k] * fabs(xp - xk2) + v2[k] * fabs(xp - xk1)) / fabs(xk2 - xk1);
}

/* linear_interpolate_force (:1204-1222) */
static void ss_interp_force(orc_pt P1, orc_pt P2, orc_pt r, const double* f, double* f1, double* f2)
{
    double xk1 = 0.0;
    double xk2 = sqrt((P2.x - P1.x) * (P2.x - P1.x) + (P2.y - P1.y) * (P2.y - P1.y) + (P2.z - P1.z) * (P2.z - P1.z));
    double xp = sqrt((r.x - P1.x) * (r.x - P1.x) + (r.y - P1.y) * (r.y - P1.y) + (r.z - P1.z) * (r.z - P1.z));
    for (int k = 0; k < 3; k++) f1[k] = -fabs(xp - xk2) / fabs(xk1 - xk2) * f[k];
    for (int k = 0; k < 3; k++) f2[k] = -fabs(xp - xk1) / fabs(xk1 - xk2) * f[k];
}

static orc_pt ss_point(const orc_ctx* c, int i) { orc_pt p = {c->xp[i * 3], c->xp[i * 3 + 1], c->xp[i * 3 + 2]}; return p; }

static void interaction_ss(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    const int form = P->ss_type, nd = P->ndim, n = c->n;
    const double dt = P->dt, dr = P->dr, myu = P->ss_myu, zeta = P->ss_zeta;
    const double reach = (form == 1) ? 0.5 * dr : dr;
    int ids[NB];
    double dsts[NB];
    for (int i = 0; i < n * 3; i++) { c->ss_fn[i] = 0.0; c->ss_ft[i] = 0.0; }
    for (int i = 0; i < n; i++) {
        int ti = c->type[i];
        if (!(ti == 1 || ti == 2)) continue;
        int total = 0;
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[j] != 4) continue;
            double d = (c->xp[i * 3] - c->xp[j * 3]) * (c->xp[i * 3] - c->xp[j * 3]) +
                       (c->xp[i * 3 + 1] - c->xp[j * 3 + 1]) * (c->xp[i * 3 + 1] - c->xp[j * 3 + 1]) +
                       (c->xp[i * 3 + 2] - c->xp[j * 3 + 2]) * (c->xp[i * 3 + 2] - c->xp[j * 3 + 2]);
            ids[total] = j;
            dsts[total] = sqrt(d);
            total++;
        }
        for (int a = 0; a < 4; a++)   /* clParti_Pair::dist_sorting */
            for (int b = a + 1; b < total; b++)
                if (dsts[a] > dsts[b]) { int t = ids[a]; ids[a] = ids[b]; ids[b] = t; }
        if (total < (nd == 2 ? 2 : 3)) continue;
        const double mi = c->mass[i];
        const double* vpi = &c->vxp[i * 3];
        double* fn = &c->ss_fn[i * 3];
        double* ft = &c->ss_ft[i * 3];
        orc_pt p4 = ss_point(c, i);
        int id1 = ids[0], id2 = ids[1];
        orc_pt p1 = ss_point(c, id1), p2 = ss_point(c, id2);
        if (nd == 2) {
            /* cal_line (:1055-1060), C = 1 from clLine() */
            double den = p2.y * p1.x - p1.y * p2.x;
            double A = (p1.y - p2.y) / den, B = (p2.x - p1.x) / den, C = 1.0;
            double dp = ss_dpline(p4, A, B, C);
            /* cal_mappoint_line (:1094-1125) */
            double tmp = sqrt(A * A + B * B);
            orc_pt P1 = {p4.x + dp * A / tmp, p4.y + dp * B / tmp, 0.0}, P2 = {p4.x - dp * A / tmp, p4.y - dp * B / tmp, 0.0};
            orc_pt outp = (ss_dpline(P1, A, B, C) < 1.0e-3) ? P1 : P2;
            outp.z = 0.0;
            /* check_ifinside_line (:1290-1305) on (p1, p2, outp with z = 0) */
            double v0x = p2.x - p1.x, v0y = p2.y - p1.y, v0z = p2.z - p1.z;
            double v1x = outp.x - p1.x, v1y = outp.y - p1.y, v1z = 0.0 - p1.z;
            double dot00 = v0x * v0x + v0y * v0y + v0z * v0z, dot01 = v0x * v1x + v0y * v1y + v0z * v1z;
            double u = 1.0 / dot00 * dot01;
            int inside = !(u < 0 || u > 1);
            if (!(inside && dp < reach)) continue;
            /* clLine::set_normal, check_ifoutward2D (:1252-1270) */
            double nx = 0.0, ny = 0.0, tot = sqrt(A * A + B * B);
            if (tot > 1.0e-10) { nx = A / tot; ny = B / tot; }
            double dot = (outp.x - p4.x) * nx + (outp.y - p4.y) * ny + 0.0 * 0.0;
            if (!(dot <= 0.0)) { nx = -nx; ny = -ny; }
            double ms, vs[3];
            ss_interp(p1, p2, outp, c->mass[id1], c->mass[id2], &c->vxp[id1 * 3], &c->vxp[id2 * 3], &ms, vs);
            vs[0] -= vpi[0];
            vs[1] -= vpi[1];
            if (form != 1) {
                vs[0] *= ms / (ms + mi);
                vs[1] *= ms / (ms + mi);
            }
            /* decomposition_velocity2D (:1346-1356) */
            double v = vs[0] * nx + vs[1] * ny;
            double vn[2] = {v * nx, v * ny}, vt[2] = {vs[0] - vn[0], vs[1] - vn[1]};
            if (form == 3) {
                double mag = (1.0 - zeta) * 2.0 * mi * (dr - dp) / dt / dt;
                fn[0] = mag * nx; fn[1] = mag * ny;
            } else {
                fn[0] = mi * vn[0] / dt; fn[1] = mi * vn[1] / dt;
            }
            ft[0] = mi * vt[0] / dt; ft[1] = mi * vt[1] / dt;
            double mag_fn = sqrt(fn[0] * fn[0] + fn[1] * fn[1]);
            double mag_ft = sqrt(ft[0] * ft[0] + ft[1] * ft[1]);
            if (mag_ft > (mag_fn * myu)) {
                vt[0] = vt[0] * myu * mag_fn / mag_ft;
                vt[1] = vt[1] * myu * mag_fn / mag_ft;
                ft[0] = mi * vt[0] / dt; ft[1] = mi * vt[1] / dt;
            }
            double f1n[3], f2n[3], f1t[3], f2t[3];
            ss_interp_force(p1, p2, outp, fn, f1n, f2n);
            ss_interp_force(p1, p2, outp, ft, f1t, f2t);
            for (int k = 0; k < 3; k++) c->ss_fn[id1 * 3 + k] += f1n[k];
            for (int k = 0; k < 3; k++) c->ss_fn[id2 * 3 + k] += f2n[k];
            for (int k = 0; k < 3; k++) c->ss_ft[id1 * 3 + k] += f1t[k];
            for (int k = 0; k < 3; k++) c->ss_ft[id2 * 3 + k] += f2t[k];
        } else {
            int id3 = ids[2];
            orc_pt p3 = ss_point(c, id3);
            /* cal_plane (:1063-1076), D = 1 from clPlane() */
            double den = -p1.x * (p2.y * p3.z - p3.y * p2.z) - p2.x * (p3.y * p1.z - p1.y * p3.z) - p3.x * (p1.y * p2.z - p2.y * p1.z);
            double A = p1.y * (p2.z - p3.z) + p2.y * (p3.z - p1.z) + p3.y * (p1.z - p2.z);
            double B = p1.z * (p2.x - p3.x) + p2.z * (p3.x - p1.x) + p3.z * (p1.x - p2.x);
            double C = p1.x * (p2.y - p3.y) + p2.x * (p3.y - p1.y) + p3.x * (p1.y - p2.y);
            A = A / den; B = B / den; C = C / den;
            const double D = 1.0;
            double dp = ss_dpplane(p4, A, B, C, D);
            /* cal_mappoint_plane (:1127-1160) */
            double tmp = sqrt(A * A + B * B + C * C);
            orc_pt P1 = {p4.x + dp * A / tmp, p4.y + dp * B / tmp, p4.z + dp * C / tmp};
            orc_pt P2 = {p4.x - dp * A / tmp, p4.y - dp * B / tmp, p4.z - dp * C / tmp};
            orc_pt outp = (ss_dpplane(P1, A, B, C, D) < 1.0e-3) ? P1 : P2;
            /* check_ifinside_triangle (:1307-1344) of (p1, p2, p3, outp) */
            double v0[3] = {p3.x - p1.x, p3.y - p1.y, p3.z - p1.z};
            double v1[3] = {p2.x - p1.x, p2.y - p1.y, p2.z - p1.z};
            double v2[3] = {outp.x - p1.x, outp.y - p1.y, outp.z - p1.z};
            double dot00 = v0[0] * v0[0] + v0[1] * v0[1] + v0[2] * v0[2];
            double dot01 = v0[0] * v1[0] + v0[1] * v1[1] + v0[2] * v1[2];
            double dot02 = v0[0] * v2[0] + v0[1] * v2[1] + v0[2] * v2[2];
            double dot11 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
            double dot12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
            double inv = 1 / (dot00 * dot11 - dot01 * dot01);
            double u = (dot11 * dot02 - dot01 * dot12) * inv;
            int inside = 1;
            if (u < 0 || u > 1) inside = 0;
            else {
                double v = (dot00 * dot12 - dot01 * dot02) * inv;
                if (v < 0 || v > 1) inside = 0;
                else inside = (u + v <= 1);
            }
            if (!(inside && dp < reach)) continue;
            /* clPlane::set_normal, check_ifoutward3D (:1272-1288) */
            double nx = 0.0, ny = 0.0, nz = 0.0, tot = sqrt(A * A + B * B + C * C);
            if (tot > 1.0e-10) { nx = A / tot; ny = B / tot; nz = C / tot; }
            double dot = (outp.x - p4.x) * nx + (outp.y - p4.y) * ny + (outp.z - p4.z) * nz;
            if (!(dot <= 0.0)) { nx = -nx; ny = -ny; nz = -nz; }
            /* cal_line3D (:1078-1092) of (p1, p2) and (p3, outp); cal_intersect_lines3D (:1162-1185) */
            double d1 = sqrt((p2.x - p1.x) * (p2.x - p1.x) + (p2.y - p1.y) * (p2.y - p1.y) + (p2.z - p1.z) * (p2.z - p1.z));
            double a1 = (p2.x - p1.x) / d1, b1 = (p2.y - p1.y) / d1, c1 = (p2.z - p1.z) / d1;
            double d2 = sqrt((outp.x - p3.x) * (outp.x - p3.x) + (outp.y - p3.y) * (outp.y - p3.y) + (outp.z - p3.z) * (outp.z - p3.z));
            double a2 = (outp.x - p3.x) / d2, b2 = (outp.y - p3.y) / d2;
            double flag = a1 * b2 - a2 * b1;
            if (!(fabs(flag) > 1.0e-3)) continue;
            double tu = a2 * (p1.y - p3.y) - b2 * (p1.x - p3.x);
            double t = tu / flag;
            orc_pt sectp = {p1.x + a1 * t, p1.y + b1 * t, p1.z + c1 * t};
            double tms, tvs[3], ms, vs[3];
            ss_interp(p1, p2, sectp, c->mass[id1], c->mass[id2], &c->vxp[id1 * 3], &c->vxp[id2 * 3], &tms, tvs);
            ss_interp(p3, sectp, outp, c->mass[id3], tms, &c->vxp[id3 * 3], tvs, &ms, vs);
            for (int k = 0; k < 3; k++) {
                vs[k] -= vpi[k];
                if (form != 1) vs[k] *= ms / (ms + mi);
            }
            /* decomposition_velocity3D (:1358-1369) */
            double v = vs[0] * nx + vs[1] * ny + vs[2] * nz;
            double vn[3] = {v * nx, v * ny, v * nz}, vt[3] = {vs[0] - vn[0], vs[1] - vn[1], vs[2] - vn[2]};
            if (form == 3) {
                double mag = (1.0 - zeta) * 2.0 * mi * (dr - dp) / dt / dt;
                fn[0] = mag * nx; fn[1] = mag * ny; fn[2] = mag * nz;
            } else {
                for (int k = 0; k < 3; k++) fn[k] = mi * vn[k] / dt;
            }
            for (int k = 0; k < 3; k++) ft[k] = mi * vt[k] / dt;
            double mag_fn = sqrt(fn[0] * fn[0] + fn[1] * fn[1] + fn[2] * fn[2]);
            double mag_ft = sqrt(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
            if (mag_ft > (mag_fn * myu)) {
                for (int k = 0; k < 3; k++) vt[k] = vt[k] * myu * mag_fn / mag_ft;
                for (int k = 0; k < 3; k++) ft[k] = mi * vt[k] / dt;
            }
            double f1n[3], f3n[3], f1t[3], f3t[3], g1n[3], g2n[3], g1t[3], g2t[3];
            ss_interp_force(p3, sectp, outp, fn, f1n, f3n);
            ss_interp_force(p3, sectp, outp, ft, f1t, f3t);
            for (int k = 0; k < 3; k++) c->ss_fn[id3 * 3 + k] += f1n[k];
            for (int k = 0; k < 3; k++) c->ss_ft[id3 * 3 + k] += f1t[k];
            ss_interp_force(p1, p2, sectp, f3n, g1n, g2n);
            ss_interp_force(p1, p2, sectp, f3t, g1t, g2t);
            for (int k = 0; k < 3; k++) c->ss_fn[id1 * 3 + k] -= g1n[k];
            for (int k = 0; k < 3; k++) c->ss_fn[id2 * 3 + k] -= g2n[k];
            for (int k = 0; k < 3; k++) c->ss_ft[id1 * 3 + k] -= g1t[k];
            for (int k = 0; k < 3; k++) c->ss_ft[id2 * 3 + k] -= g2t[k];
        }
    }
    /* the per-thread sums into interfss and the acceleration (:1008-1034) */
    for (int i = 0; i < n; i++) {
        int ti = c->type[i];
        if (!(ti == 1 || ti == 2 || ti == 4)) continue;
        for (int k = 0; k < 3; k++) {
            c->interfss[i * 3 + k] = 0.0;
            if (form != 3) c->interfss[i * 3 + k] += zeta * (c->ss_ft[i * 3 + k] + c->ss_fn[i * 3 + k]);
            else c->interfss[i * 3 + k] += c->ss_ft[i * 3 + k] + c->ss_fn[i * 3 + k];
        }
        for (int k = 0; k < 3; k++) c->ax[i * 3 + k] += c->interfss[i * 3 + k] / c->mass[i];
    }
}

/* boundary_free_solid (flbndy 5): CPP_13-boundary.cpp:1239-1516.  The rigid
 * contact of interaction_ss_rigid against the wall particles, with the walls'
 * velocities (interfss), applied to the particle's own acceleration only:
 * types 1-4 in 2-D; every particle in 3-D, as the reference's 3-D loop has no
 * type test. */
static void boundary_free_solid(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    const int nd = P->ndim, n = c->n;
    const double dt = P->dt, dr = P->dr, myu = P->ss_myu, zeta = P->ss_zeta;
    int ids[NB];
    double dsts[NB];
    for (int i = 0; i < n; i++) {
        int ti = c->type[i];
        if (nd == 2 && !(ti == 1 || ti == 2 || ti == 3 || ti == 4)) continue;
        int total = 0;
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj);
            if (c->type[j] != 0) continue;
            double d = (c->xp[i * 3] - c->xp[j * 3]) * (c->xp[i * 3] - c->xp[j * 3]) +
                       (c->xp[i * 3 + 1] - c->xp[j * 3 + 1]) * (c->xp[i * 3 + 1] - c->xp[j * 3 + 1]) +
                       (c->xp[i * 3 + 2] - c->xp[j * 3 + 2]) * (c->xp[i * 3 + 2] - c->xp[j * 3 + 2]);
            ids[total] = j;
            dsts[total] = sqrt(d);
            total++;
        }
        for (int a = 0; a < 4; a++)
            for (int b = a + 1; b < total; b++)
                if (dsts[a] > dsts[b]) { int t = ids[a]; ids[a] = ids[b]; ids[b] = t; }
        if (total < (nd == 2 ? 2 : 3)) continue;
        const double mi = c->mass[i];
        const double* vpi = &c->vxp[i * 3];
        double fn[3] = {0, 0, 0}, ft[3] = {0, 0, 0};
        orc_pt p4 = ss_point(c, i);
        int id1 = ids[0], id2 = ids[1];
        orc_pt p1 = ss_point(c, id1), p2 = ss_point(c, id2);
        if (nd == 2) {
            double den = p2.y * p1.x - p1.y * p2.x;
            double A = (p1.y - p2.y) / den, B = (p2.x - p1.x) / den, C = 1.0;
            double dp = ss_dpline(p4, A, B, C);
            double tmp = sqrt(A * A + B * B);
            orc_pt Q1 = {p4.x + dp * A / tmp, p4.y + dp * B / tmp, 0.0}, Q2 = {p4.x - dp * A / tmp, p4.y - dp * B / tmp, 0.0};
            orc_pt outp = (ss_dpline(Q1, A, B, C) < 1.0e-3) ? Q1 : Q2;
            outp.z = 0.0;
            double v0x = p2.x - p1.x, v0y = p2.y - p1.y, v0z = p2.z - p1.z;
            double v1x = outp.x - p1.x, v1y = outp.y - p1.y, v1z = 0.0 - p1.z;
            double dot00 = v0x * v0x + v0y * v0y + v0z * v0z, dot01 = v0x * v1x + v0y * v1y + v0z * v1z;
            double u = 1.0 / dot00 * dot01;
            if ((u < 0 || u > 1) || !(dp < 0.5 * dr)) continue;
            double nx = 0.0, ny = 0.0, tot = sqrt(A * A + B * B);
            if (tot > 1.0e-10) { nx = A / tot; ny = B / tot; }
            double dot = (outp.x - p4.x) * nx + (outp.y - p4.y) * ny + 0.0 * 0.0;
            if (!(dot <= 0.0)) { nx = -nx; ny = -ny; }
            double ms, vs[3];
            ss_interp(p1, p2, outp, c->mass[id1], c->mass[id2], &c->interfss[id1 * 3], &c->interfss[id2 * 3], &ms, vs);
            vs[0] -= vpi[0];
            vs[1] -= vpi[1];
            double v = vs[0] * nx + vs[1] * ny;
            double vn[2] = {v * nx, v * ny}, vt[2] = {vs[0] - vn[0], vs[1] - vn[1]};
            fn[0] = mi * vn[0] / dt; fn[1] = mi * vn[1] / dt;
            ft[0] = mi * vt[0] / dt; ft[1] = mi * vt[1] / dt;
            double mag_fn = sqrt(fn[0] * fn[0] + fn[1] * fn[1]), mag_ft = sqrt(ft[0] * ft[0] + ft[1] * ft[1]);
            if (mag_ft > (mag_fn * myu)) {
                vt[0] = vt[0] * myu * mag_fn / mag_ft;
                vt[1] = vt[1] * myu * mag_fn / mag_ft;
                ft[0] = mi * vt[0] / dt; ft[1] = mi * vt[1] / dt;
            }
            c->ax[i * 3 + 0] += zeta * (ft[0] + fn[0]) / mi;
            c->ax[i * 3 + 1] += zeta * (ft[1] + fn[1]) / mi;
            c->ax[i * 3 + 2] += 0.0;
        } else {
            int id3 = ids[2];
            orc_pt p3 = ss_point(c, id3);
            double den = -p1.x * (p2.y * p3.z - p3.y * p2.z) - p2.x * (p3.y * p1.z - p1.y * p3.z) - p3.x * (p1.y * p2.z - p2.y * p1.z);
            double A = p1.y * (p2.z - p3.z) + p2.y * (p3.z - p1.z) + p3.y * (p1.z - p2.z);
            double B = p1.z * (p2.x - p3.x) + p2.z * (p3.x - p1.x) + p3.z * (p1.x - p2.x);
            double C = p1.x * (p2.y - p3.y) + p2.x * (p3.y - p1.y) + p3.x * (p1.y - p2.y);
            A = A / den; B = B / den; C = C / den;
            const double D = 1.0;
            double dp = ss_dpplane(p4, A, B, C, D);
            double tmp = sqrt(A * A + B * B + C * C);
            orc_pt Q1 = {p4.x + dp * A / tmp, p4.y + dp * B / tmp, p4.z + dp * C / tmp};
            orc_pt Q2 = {p4.x - dp * A / tmp, p4.y - dp * B / tmp, p4.z - dp * C / tmp};
            orc_pt outp = (ss_dpplane(Q1, A, B, C, D) < 1.0e-3) ? Q1 : Q2;
            double a0[3] = {p3.x - p1.x, p3.y - p1.y, p3.z - p1.z};
            double a1[3] = {p2.x - p1.x, p2.y - p1.y, p2.z - p1.z};
            double a2[3] = {outp.x - p1.x, outp.y - p1.y, outp.z - p1.z};
            double dot00 = a0[0] * a0[0] + a0[1] * a0[1] + a0[2] * a0[2];
            double dot01 = a0[0] * a1[0] + a0[1] * a1[1] + a0[2] * a1[2];
            double dot02 = a0[0] * a2[0] + a0[1] * a2[1] + a0[2] * a2[2];
            double dot11 = a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2];
            double dot12 = a1[0] * a2[0] + a1[1] * a2[1] + a1[2] * a2[2];
            double inv = 1 / (dot00 * dot11 - dot01 * dot01);
            double u = (dot11 * dot02 - dot01 * dot12) * inv;
            int inside = 1;
            if (u < 0 || u > 1) inside = 0;
            else {
                double v = (dot00 * dot12 - dot01 * dot02) * inv;
                inside = (v < 0 || v > 1) ? 0 : (u + v <= 1);
            }
            if (!(inside && dp < 0.5 * dr)) continue;
            double nx = 0.0, ny = 0.0, nz = 0.0, tot = sqrt(A * A + B * B + C * C);
            if (tot > 1.0e-10) { nx = A / tot; ny = B / tot; nz = C / tot; }
            double dot = (outp.x - p4.x) * nx + (outp.y - p4.y) * ny + (outp.z - p4.z) * nz;
            if (!(dot <= 0.0)) { nx = -nx; ny = -ny; nz = -nz; }
            double d1 = sqrt((p2.x - p1.x) * (p2.x - p1.x) + (p2.y - p1.y) * (p2.y - p1.y) + (p2.z - p1.z) * (p2.z - p1.z));
            double la = (p2.x - p1.x) / d1, lb = (p2.y - p1.y) / d1, lc = (p2.z - p1.z) / d1;
            double d2 = sqrt((outp.x - p3.x) * (outp.x - p3.x) + (outp.y - p3.y) * (outp.y - p3.y) + (outp.z - p3.z) * (outp.z - p3.z));
            double ma = (outp.x - p3.x) / d2, mb = (outp.y - p3.y) / d2;
            double flag = la * mb - ma * lb;
            if (!(fabs(flag) > 1.0e-3)) continue;
            double tu = ma * (p1.y - p3.y) - mb * (p1.x - p3.x);
            double t = tu / flag;
            orc_pt sectp = {p1.x + la * t, p1.y + lb * t, p1.z + lc * t};
            double tms, tvs[3], ms, vs[3];
            ss_interp(p1, p2, sectp, c->mass[id1], c->mass[id2], &c->interfss[id1 * 3], &c->interfss[id2 * 3], &tms, tvs);
            ss_interp(p3, sectp, outp, c->mass[id3], tms, &c->interfss[id3 * 3], tvs, &ms, vs);
            for (int k = 0; k < 3; k++) vs[k] -= vpi[k];
            double v = vs[0] * nx + vs[1] * ny + vs[2] * nz;
            double vn[3] = {v * nx, v * ny, v * nz}, vt[3] = {vs[0] - vn[0], vs[1] - vn[1], vs[2] - vn[2]};
            for (int k = 0; k < 3; k++) { fn[k] = mi * vn[k] / dt; ft[k] = mi * vt[k] / dt; }
            double mag_fn = sqrt(fn[0] * fn[0] + fn[1] * fn[1] + fn[2] * fn[2]);
            double mag_ft = sqrt(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
            if (mag_ft > (mag_fn * myu)) {
                for (int k = 0; k < 3; k++) vt[k] = vt[k] * myu * mag_fn / mag_ft;
                for (int k = 0; k < 3; k++) ft[k] = mi * vt[k] / dt;
            }
            for (int k = 0; k < 3; k++) c->ax[i * 3 + k] += zeta * (ft[k] + fn[k]) / mi;
        }
    }
}

/* no_slip_tran / free_slip_tran: CPP_13-boundary.cpp:711-958 and 960-1237.
 * Each wall particle's Shepard sums over its water, soil, air and structure
 * neighbours give its stress per phase (soil with the pore terms) and its
 * virtual velocity per phase: the wall's own velocity minus the phase's mean
 * velocity (no-slip), or plus the phase's mean tangential velocity taken from
 * neighbours more than 0.1 dr away (free-slip).  (The reference's rho_* are
 * formed but never read; they are not kept.) */
static void tran_walls(orc_ctx* c, int free_slip)
{
    const double dr = c->P.dr;
    double* sig_out[4] = {c->sb_water, c->sb_soil, c->sb_air, c->sb_struct};
    double* vel_out[4] = {c->vb_water, c->vb_soil, c->vb_air, c->vb_struct};
    for (int i = 0; i < c->n; i++) {
        if (c->type[i] != 0) continue;
        double us[4][6], uv[4][3], down[4];
        for (int p = 0; p < 4; p++) {
            for (int k = 0; k < 6; k++) us[p][k] = 0.0;
            for (int k = 0; k < 3; k++) uv[p][k] = 0.0;
            down[p] = 0.0;
        }
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), tj = c->type[j];
            if (tj < 1 || tj > 4) continue;
            int p = tj - 1;
            double mj = c->mass[j], rj = c->rho[j], w3 = W(i, nj, 3);
            const double* sj = &c->sig[j * 6];
            const double* vj = &c->vx[j * 3];
            if (tj == 2) {
                double satu = c->satu[j];
                for (int k = 0; k < 3; k++)
                    us[p][k] = us[p][k] + mj * (sj[k] - satu * c->prew[j] + (1 - satu) * c->prea[j]) * w3 / rj;
                for (int k = 3; k < 6; k++) us[p][k] = us[p][k] + mj * sj[k] * w3 / rj;
            } else {
                for (int k = 0; k < 6; k++) us[p][k] = us[p][k] + mj * sj[k] * w3 / rj;
            }
            if (free_slip) {
                double v1[3] = {c->xp[i * 3] - c->xp[j * 3], c->xp[i * 3 + 1] - c->xp[j * 3 + 1],
                                c->xp[i * 3 + 2] - c->xp[j * 3 + 2]};
                double dst = sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
                double inprod = vj[0] * v1[0] + vj[1] * v1[1] + vj[2] * v1[2];
                if (dst > 0.1 * dr)
                    for (int k = 0; k < 3; k++)
                        uv[p][k] = uv[p][k] + mj * (vj[k] - inprod * v1[k] / dst / dst) * w3 / rj;
            } else {
                for (int k = 0; k < 3; k++) uv[p][k] = uv[p][k] + mj * vj[k] * w3 / rj;
            }
            down[p] = down[p] + mj * w3 / rj;
        }
        const double* its = &c->interfss[i * 3];
        for (int p = 0; p < 4; p++) {
            if (fabs(down[p]) > 1.0e-6) {
                for (int k = 0; k < 6; k++) sig_out[p][i * 6 + k] = us[p][k] / down[p];
                for (int k = 0; k < 3; k++)
                    vel_out[p][i * 3 + k] = free_slip ? its[k] + uv[p][k] / down[p] : its[k] - uv[p][k] / down[p];
            } else {
                for (int k = 0; k < 6; k++) sig_out[p][i * 6 + k] = 0.0;
                for (int k = 0; k < 3; k++) vel_out[p][i * 3 + k] = its[k];
            }
        }
    }
}

/* check_domain: CPP_13-boundary.cpp:20-68, in the sequential order (vbx is
 * taken from the first wall particle with matype > 2 and applies to the
 * particles after it) */
static void check_domain(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    double bmax[3] = {P->xmax, P->ymax, P->zmax}, bmin[3] = {P->xmin, P->ymin, P->zmin};
    double vbx[3] = {0, 0, 0}, dr = P->dr;
    int flag = 0, dim = P->ndim;
    for (int i = 0; i < c->n; i++) {
        int ti = c->type[i];
        if (ti != 0 && ti != 7) {
            const double* xp = &c->xp[i * 3];
            int hit = 0;
            if (xp[0] - bmax[0] >= -0.5 * dr) hit = 1;
            if (xp[0] - bmin[0] <= 0.5 * dr) hit = 1;
            if (xp[1] - bmax[1] >= -0.5 * dr) hit = 1;
            if (xp[1] - bmin[1] <= 0.5 * dr) hit = 1;
            if (xp[2] - bmax[2] >= -0.5 * dr && dim == 3) hit = 1;
            if (xp[2] - bmin[2] <= 0.5 * dr && dim == 3) hit = 1;
            if (hit) for (int k = 0; k < 3; k++) c->vx[i * 3 + k] = vbx[k];
        } else if (ti == 0 && c->matype[i] > 2 && flag == 0) {
            flag = 1;
            for (int k = 0; k < 3; k++) vbx[k] = c->interfss[i * 3 + k];
        }
    }
}

/* update: CPP_12-1-update.cpp:11-55 */
static void update(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    int ndim = P->ndim, loop = c->l - P->inip;
    double dt = P->dt;
    for (int i = 0; i < c->n; i++) {
        for (int k = 0; k < ndim; k++) {
            if (c->type[i] != 0) {
                double s = (c->vx[i * 3 + k] + c->vxp[i * 3 + k]) * dt * 0.5;
                c->x[i * 3 + k] = c->xp[i * 3 + k] + s;
                if (loop == 0) c->ux[i * 3 + k] = 0.0;
                else c->ux[i * 3 + k] = c->ux[i * 3 + k] + (c->vx[i * 3 + k] + c->vxp[i * 3 + k]) * dt * 0.5;
                c->xp[i * 3 + k] = c->x[i * 3 + k];
                c->vxp[i * 3 + k] = c->vx[i * 3 + k];
                c->axp[i * 3 + k] = c->ax[i * 3 + k];
                c->rhop[i] = c->rho[i];
            } else {
                int mt = c->matype[i];
                if (mt == 2 || mt == 3 || mt == 4 || mt == 5) {
                    c->x[i * 3 + k] = c->xp[i * 3 + k] + (c->interfss[i * 3 + k] + c->interfss[i * 3 + k]) * dt * 0.5;
                    c->ux[i * 3 + k] = c->ux[i * 3 + k] + (c->interfss[i * 3 + k] + c->interfss[i * 3 + k]) * dt * 0.5;
                    c->xp[i * 3 + k] = c->x[i * 3 + k];
                    c->rhop[i] = c->rho[i];
                    c->prep[i] = c->pre[i];
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------- */

int orc_nnps(orc_ctx* c, int* ninflu, int* influ, double* wij)
{
    int err = parttocell(c);
    if (err) return err;
    err = partisearching(c);
    if (ninflu) memcpy(ninflu, c->ninflu, sizeof(int) * c->n);
    if (influ) memcpy(influ, c->influ, sizeof(int) * (size_t)c->n * NB);
    if (wij) memcpy(wij, c->wij, sizeof(double) * (size_t)c->n * NB * 4);
    return err;
}

/* inverse_mat_2D / inverse_mat_3D: CPP_3-NNPS.cpp:499-558 */
static void inverse_2d(double A[3][3], double B[3][3])
{
    double det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
    if (fabs(det) > 1.0e-5) {
        B[0][0] = A[1][1] / det; B[0][1] = -A[0][1] / det;
        B[1][0] = -A[1][0] / det; B[1][1] = A[0][0] / det;
    } else {
        B[0][0] = 1.0; B[0][1] = 0.0; B[1][0] = 0.0; B[1][1] = 1.0;
    }
}

static void inverse_3d(double A[3][3], double B[3][3])
{
    double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[1][0] * (A[0][1] * A[2][2] - A[0][2] * A[2][1])
        + A[2][0] * (A[0][1] * A[1][2] - A[0][2] * A[1][1]);
    if (fabs(det) > 1.0e-5) {
        B[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) / det;
        B[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) / det;
        B[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) / det;
        B[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) / det;
        B[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) / det;
        B[1][2] = (A[1][0] * A[0][2] - A[0][0] * A[1][2]) / det;
        B[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) / det;
        B[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) / det;
        B[2][2] = (A[0][0] * A[1][1] - A[1][0] * A[0][1]) / det;
    } else {
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) B[a][b] = (a == b) ? 1.0 : 0.0;
    }
}

/* kernel_gradient_correction: CPP_3-NNPS.cpp:376-496.  For soil and structure
 * particles, the kernel gradients of every pair are multiplied by the inverse
 * of L = sum_j m_j / rho_j (x_j - x_i) (x) grad W_ij over same-phase, wall and
 * soil/structure neighbours. */
static void kernel_gradient_correction(orc_ctx* c)
{
    int ndim = c->P.ndim;
    for (int i = 0; i < c->n; i++) {
        int ti = c->type[i];
        if (!(ti == 2 || ti == 4)) continue;
        double L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Li[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            int j = NBR(i, nj), tj = c->type[j];
            int take = (ti == 2 && (tj == 2 || tj == 0 || tj == 4)) || (ti == 4 && (tj == 4 || tj == 0 || tj == 2));
            if (!take) continue;
            double xij[3];
            for (int k = 0; k < ndim; k++) xij[k] = c->xp[j * 3 + k] - c->xp[i * 3 + k];
            for (int a = 0; a < ndim; a++)
                for (int b = 0; b < ndim; b++)
                    L[a][b] = L[a][b] + c->mass[j] / c->rho[j] * xij[a] * W(i, nj, b);
        }
        if (ndim == 2) inverse_2d(L, Li);
        else inverse_3d(L, Li);
        for (int nj = 1; nj <= c->ninflu[i]; nj++) {
            double* w = &W(i, nj, 0);
            double r0 = Li[0][0] * w[0] + Li[0][1] * w[1] + Li[0][2] * w[2];
            double r1 = Li[1][0] * w[0] + Li[1][1] * w[1] + Li[1][2] * w[2];
            double r2 = Li[2][0] * w[0] + Li[2][1] * w[1] + Li[2][2] * w[2];
            w[0] = r0; w[1] = r1; w[2] = r2;
        }
    }
}

/* rainini (CPP_15-1-rain.cpp:11-23) for rtype 1: lp steps between rows,
 * nrain / nhor in integer arithmetic */
int orc_set_rain(orc_ctx* c, const sphgpu_rain* rain)
{
    if (!rain) return SPHGPU_E_ARG;
    if (rain->rtype != 1) return SPHGPU_E_UNSUPPORTED;
    c->rain = *rain;
    if (c->rain.nhor == 0) c->rain.nhor = 35;      /* initial_pro's default, CPP_2-initialf.cpp:201-202 */
    double temp = c->rain.nrain / c->rain.nhor + 1.0;
    c->lp = (int)((c->P.loop - c->P.inip) / temp);
    c->vrain = c->rain.drop_velocity;
    c->rain_set = 1;
    return 0;
}

int orc_set_vibration(orc_ctx* c, double ttime, int nsteps, double sttime, double edtime, const double* loads)
{
    if (nsteps < 1) return 7;
    if (!loads || !(ttime > 0.0)) return SPHGPU_E_ARG;
    free(c->vib_loads);
    c->vib_loads = (double*)malloc(sizeof(double) * 3 * (size_t)nsteps);
    memcpy(c->vib_loads, loads, sizeof(double) * 3 * (size_t)nsteps);
    c->vib_ttime = ttime; c->vib_nsteps = nsteps; c->vib_sttime = sttime; c->vib_edtime = edtime;
    c->vib_set = 1;
    return 0;
}

int orc_get_rain(const orc_ctx* c, sphgpu_rain* rain)
{
    if (!rain) return SPHGPU_E_ARG;
    *rain = c->rain;
    return 0;
}

/* rainpro (CPP_15-1-rain.cpp:43-85): the next row of waiting rain
 * particles, from index ntotal - nrain on while each next particle's vertical
 * coordinate stays within 0.1 dr of the one before it (compared before that
 * one is lowered), becomes water falling at vrain, lowered to 0.95 of its
 * height; the reference's loop reads one particle past the array after the
 * last one, which this restatement does not */
static void rainpro(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    const int nd = P->ndim, n = c->n;
    const double g = (nd == 2) ? P->gy : P->gz;
    int k = n - c->rain.nrain;
    if (c->rain.nrain <= 0) return;
    for (;;) {
        c->rain.nrain = c->rain.nrain - 1;
        const double temp_xp = c->xp[k * 3 + nd - 1];
        c->xp[k * 3 + nd - 1] = 0.95 * c->xp[k * 3 + nd - 1];
        c->type[k] = 1;
        c->matype[k] = 0;
        c->etype[k] = 7;
        c->rhop[k] = c->fl[k].porosity * c->fl[k].dens;
        c->hl[k] = P->dr;
        c->mass[k] = (nd == 2) ? c->rhop[k] * c->hl[k] * c->hl[k] : c->rhop[k] * c->hl[k] * c->hl[k] * c->hl[k];
        for (int d = 0; d < 3; d++) { c->vxp[k * 3 + d] = 0.0; c->vx[k * 3 + d] = 0.0; }
        c->vxp[k * 3 + nd - 1] = c->vrain;
        c->prep[k] = c->rhop[k] * P->dr * (-g) * c->rain.press_factor;
        c->satu[k] = 0.99;
        k++;
        if (!(k <= n - 1 && fabs(c->xp[k * 3 + nd - 1] - temp_xp) < 0.1 * P->dr)) break;
    }
}

/* partidel (CPP_15-2-partidel.cpp:19-58): water within dr of 7 dr past
 * either x end of the domain box and above y = 0.12 stops and leaves the
 * calculation as type 7 */
static void partidel(orc_ctx* c)
{
    const sphgpu_params* P = &c->P;
    for (int i = 0; i < c->n; i++) {
        const double dx1 = fabs(c->xp[i * 3] - P->xmax - 7.0 * P->dr);
        const double dx2 = fabs(c->xp[i * 3] - P->xmin + 7.0 * P->dr);
        const double dy1 = c->xp[i * 3 + 1] - 0.12;
        if (c->type[i] == 1 && (dx1 < P->dr || dx2 < P->dr) && dy1 > 0.0) {
            c->type[i] = 7;
            for (int d = 0; d < 3; d++) { c->vxp[i * 3 + d] = 0.0; c->vx[i * 3 + d] = 0.0; c->ax[i * 3 + d] = 0.0; }
        }
    }
}

static int check_supported(const sphgpu_params* P)
{
    if (!(P->flbndy >= 1 && P->flbndy <= 5) && P->flbndy != 13 && P->flbndy != 14) return SPHGPU_E_UNSUPPORTED;
    if (P->flknl < 1 || P->flknl > 4) return SPHGPU_E_UNSUPPORTED;
    if (P->flv < 0 || P->flv > 2) return SPHGPU_E_UNSUPPORTED;
    if (P->fli < 0 || P->fli > 3 || P->ss_type < 0 || P->ss_type > 3) return SPHGPU_E_UNSUPPORTED;
    return 0;
}

/* one pass of the main loop body, CPP_1-SPHLoops.cpp:523-753 */
int orc_step(orc_ctx* c, int nsteps)
{
    const sphgpu_params* P = &c->P;
    int err = check_supported(P);
    if (err) return err;
    if (P->flr == 1 && !c->rain_set) return SPHGPU_E_STATE;
    if (P->flv >= 1 && !c->vib_set) return SPHGPU_E_STATE;
    for (int s = 0; s < nsteps; s++) {
        c->t = c->t + P->dt;
        if (P->flr == 1 && (c->l - P->inip) > 0 && c->lp > 0 && (c->l - P->inip) % c->lp == 0) rainpro(c);
        err = parttocell(c);
        if (err) return err;
        err = partisearching(c);
        if (err) return err;
        if (P->flknl > 2) kernel_gradient_correction(c);
        density(c);
        strain_noreg(c);
        if (c->l % P->step_regu == 0) regularise(c, c->eps);
        if (P->flagum == 1) saturation(c);
        if (P->fli == 1) cal_permeability(c);
        eos(c);
        err = strain_to_stress(c);
        if (err) return err;
        if (c->l % P->step_regu == 0) regularise(c, c->sig);
        free_surface_check(c);
        stress_eig(c);
        fluid_acceleration(c, 1, 3, P->water_acc_type != 0);
        fluid_acceleration(c, 3, 1, P->air_acc_type != 0);
        soil_acceleration(c);
        structure_acceleration(c);
        artificial_viscosity(c);
        if (P->art_stre_coe > 0.0) artificial_stress(c);
        if (P->flbndy == 1 || P->flbndy == 2) boundary_moving_stress_effect(c);
        else if (P->flbndy == 3 || P->flbndy == 4 || P->flbndy == 13 || P->flbndy == 14) boundary_stress_effect_tran(c);
        else boundary_effect_free_struct(c);
        if (P->flv != 0) { free_field_walls(c); free_field_soil(c); }
        if (P->ss_type >= 1 && P->ss_type <= 3 && P->ss_acc_type == 2) coupled_water_soil_structure(c);
        if (P->flv == 1) vibration_load(c, 0);
        if (P->fli >= 1) interact(c, P->fli);
        if (P->ss_type >= 1 && P->ss_type <= 3) interaction_ss(c);
        if (c->l <= P->inip) soil_damping_geostress(c);
        if (P->flv > 0) soil_damping_vibration(c);
        if (P->flbndy == 5) boundary_free_solid(c);
        velocity_update(c);
        if (P->flv == 2) vibration_load(c, 1);
        if (P->if_move != 2) xsph(c);
        if (P->flbndy == 1) tmboundary(c);
        else if (P->flbndy == 2) { velocity_set_domain(c); tm_boundary(c); }
        else if (P->flbndy == 3) tran_walls(c, 0);
        else if (P->flbndy == 4) tran_walls(c, 1);
        else if (P->flbndy == 13) { velocity_set_domain(c); tran_walls(c, 0); }
        else if (P->flbndy == 14) { velocity_set_domain(c); tran_walls(c, 1); }
        check_domain(c);
        update(c);
        if (P->flr == 1) partidel(c);
        c->l++;
    }
    return 0;
}
