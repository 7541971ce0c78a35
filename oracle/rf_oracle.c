/*
 * rf_oracle.c -- CPU restatement of nonstationary_random_2D / _3D
 * (CPP_17-3-Nonstationary-RF.cpp).  TEST INFRASTRUCTURE ONLY: the checker of
 * the engine's correlation-matrix random field.  Single-threaded; every sum in
 * the order the reference's loops take it with one thread.
 */
#include "rf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define RF_PI 3.141592653            /* Header_Parameters.h:10 */
#define RF_MAXP 39                    /* spv_cell::parti_id[40], 1-based (Class_spatial_variability.h:69-77) */

/* Cholesky (CPP_17-3:45-74): row-oriented, the diagonal's radicand floored
 * at 1e-6 */
static void cholesky(const double* A, double* L, int n)
{
    for (int k = 0; k < n; k++) {
        double sum = 0;
        for (int i = 0; i < k; i++) sum += L[(size_t)k * n + i] * L[(size_t)k * n + i];
        sum = A[(size_t)k * n + k] - sum;
        L[(size_t)k * n + k] = sqrt(sum > 1.0e-6 ? sum : 1.0e-6);
        for (int i = k + 1; i < n; i++) {
            sum = 0;
            for (int j = 0; j < k; j++) sum += L[(size_t)i * n + j] * L[(size_t)k * n + j];
            L[(size_t)i * n + k] = (A[(size_t)i * n + k] - sum) / L[(size_t)k * n + k];
        }
        for (int j = 0; j < k; j++) L[(size_t)j * n + k] = 0;
    }
}

/* The cells of one call (CPP_17-3:97-156, 480-545; 17-5:111-176, 434-500):
 * counts, each particle's cell (-1 for none) and the centres.  Returns 0, 41,
 * 42 or 100, as orc_rf_cholesky documents. */
typedef struct rf_cells {
    int nc[3], total;
    double base[3], cdx;
    int* cell;
    double* cx;
} rf_cells;

static void rf_cells_free(rf_cells* g)
{
    free(g->cell);
    free(g->cx);
    g->cell = NULL;
    g->cx = NULL;
}

static int rf_cells_make(int nd, int n, const double* xp, const int* type, double dr, const orc_rf_spec* s,
                         rf_cells* g)
{
    double xmin[3] = {0, 0, 0}, xmax[3] = {0, 0, 0};
    g->cell = NULL;
    g->cx = NULL;
    /* the non-boundary box widened by 10% per side (CPP_17-3:100-105, 483-489) */
    for (int d = 0; d < nd; d++) {
        xmin[d] = s->nb_min[d] - 0.1 * (s->nb_max[d] - s->nb_min[d]);
        xmax[d] = s->nb_max[d] + 0.1 * (s->nb_max[d] - s->nb_min[d]);
    }
    g->cdx = s->cell_ndx * dr;
    for (int d = 0; d < 3; d++) { g->nc[d] = 1; g->base[d] = 0.0; }
    for (int d = 0; d < nd; d++) g->nc[d] = (int)((xmax[d] - xmin[d]) / g->cdx) + 1;
    g->total = g->nc[0] * g->nc[1] * g->nc[2];
    if (!(g->total > 0 && g->total < 15000)) return 41;
    for (int d = 0; d < nd; d++) g->base[d] = -(g->nc[d] * g->cdx - (xmax[d] - xmin[d])) / 2.0 + 0.01 * dr + xmin[d];
    /* cell of each particle (2-D: water and soil; 3-D: every particle) */
    g->cell = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* count = (int*)calloc((size_t)g->total, sizeof(int));
    int err = 0;
    for (int i = 0; i < n && !err; i++) {
        g->cell[i] = -1;
        if (nd == 2 && !(type[i] == 1 || type[i] == 2)) continue;
        int np[3] = {0, 0, 0};
        for (int d = 0; d < nd; d++) np[d] = (int)(fabs(xp[(size_t)i * 3 + d] - g->base[d]) / g->cdx);
        const int c = (nd == 2) ? np[1] * g->nc[0] + np[0] : np[2] * g->nc[0] * g->nc[1] + np[1] * g->nc[0] + np[0];
        /* a particle beyond the cells (the reference indexes past its array
         * there): refused */
        if (c < 0 || c >= g->total || np[0] >= g->nc[0] || np[1] >= g->nc[1] || (nd == 3 && np[2] >= g->nc[2])) {
            err = 100;
            break;
        }
        if (count[c] < RF_MAXP) { count[c]++; g->cell[i] = c; }
        else err = 42;
    }
    free(count);
    if (err) { rf_cells_free(g); return err; }
    /* cell centres */
    g->cx = (double*)malloc(sizeof(double) * 3 * (size_t)g->total);
    for (int k = 0; k < g->nc[2]; k++)
        for (int j = 0; j < g->nc[1]; j++)
            for (int i = 0; i < g->nc[0]; i++) {
                const int c = k * g->nc[0] * g->nc[1] + j * g->nc[0] + i;
                g->cx[c * 3 + 0] = g->base[0] + ((double)i + 0.5) * g->cdx;
                g->cx[c * 3 + 1] = g->base[1] + ((double)j + 0.5) * g->cdx;
                g->cx[c * 3 + 2] = (nd == 3) ? g->base[2] + ((double)k + 0.5) * g->cdx : 0.0;
            }
    return 0;
}

/* The factor L of the cell centres' correlation matrix with the lengths and
 * kernel of s (CPP_17-3:210-228, 600-620; 17-5:188-204, 511-530) */
static double* rf_factor(int nd, const rf_cells* g, const orc_rf_spec* s)
{
    const int total = g->total;
    const double* cx = g->cx;
    double* C = (double*)malloc(sizeof(double) * (size_t)total * total);
    double* L = (double*)calloc((size_t)total * total, sizeof(double));
    const double lx = s->rl[0], ly = s->rl[1], lz = s->rl[2];
    const double be = s->beta * RF_PI / 180.0, be1 = s->beta_1 * RF_PI / 180.0;
    for (int k = 0; k < total; k++)
        for (int j = 0; j < total; j++) {
            const double dx = fabs(cx[k * 3] - cx[j * 3]), dy = fabs(cx[k * 3 + 1] - cx[j * 3 + 1]);
            double acf;
            if (nd == 2) {
                if (s->flag_auto == 1) acf = exp(-2.0 * (dx / lx + dy / ly));
                else if (s->flag_auto == 2) acf = exp(-RF_PI * (pow(dx / lx, 2) + pow(dy / ly, 2)));
                else acf = exp(-2.0 * ((dx * cos(be) + dy * sin(be)) / lx + (-dx * sin(be) + dy * cos(be)) / ly));
            } else {
                const double dz = fabs(cx[k * 3 + 2] - cx[j * 3 + 2]);
                const double t0 = dx * cos(be1) + dy * sin(be1);
                const double t1 = (-dx * sin(be1) + dy * cos(be1)) * cos(be) + dz * sin(be);
                const double t2 = -(-dx * sin(be1) + dy * cos(be1)) * sin(be) + dz * cos(be);
                if (s->flag_auto == 1) acf = exp(-2.0 * (dx / lx + dy / ly + dz / lz));
                else if (s->flag_auto == 2) acf = exp(-RF_PI * (pow(dx / lx, 2) + pow(dy / ly, 2) + pow(dz / lz, 2)));
                else acf = exp(-2.0 * (t0 / lx + t1 / ly + t2 / lz));
            }
            C[(size_t)k * total + j] = acf;
        }
    cholesky(C, L, total);
    free(C);
    return L;
}

/* E = L zeta (matrix_multi, CPP_17-3:20-30; one column of 17-5:21-33): the
 * zeta values at stride zs */
static void rf_gemv(const double* L, int total, const double* zeta, int zs, double* E)
{
    for (int i = 0; i < total; i++) {
        double t = 0.0;
        for (int j = 0; j < total; j++) t = t + L[(size_t)i * total + j] * zeta[(size_t)j * zs];
        E[i] = t;
    }
}

/* the value of each cell, written into its particles of the field's phase
 * (CPP_17-3:235-450, 17-5:222-402, 545-735): the depth trend of a normal field
 * from soil_max (soil members) or water_max (fluid members), of a lognormal
 * one from soil_max for every member, as the reference has it.  depth_axis:
 * the centre coordinate read as depth; log_exp: lognormal values as exp(.)
 * (17-5) rather than pow(e, .) (17-3) */
static void rf_assign(int n, const int* type, const rf_cells* g, const double* E, const orc_rf_spec* s,
                      int dist_type, int depth_axis, int log_exp, double* out)
{
    const int soil = s->no <= 3;
    const int want = soil ? 2 : 1;
    for (int i = 0; i < n; i++) {
        const int c = g->cell[i];
        if (c < 0 || type[i] != want) continue;
        const double depth = g->cx[c * 3 + depth_axis];
        double v;
        if (dist_type == 1) {
            const double top = soil ? s->soil_max : s->water_max;
            if (top > depth) v = s->mean_value + s->coe_depth * (top - depth) + s->sd_value * E[c];
            else v = s->mean_value + s->sd_value * E[c];
        } else if (dist_type == 2) {
            double m = (s->soil_max > depth) ? s->mean_value + s->coe_depth * (s->soil_max - depth) : s->mean_value;
            const double sd = sqrt(log(1.0 + (s->sd_value / m) * (s->sd_value / m)));
            m = log(m) - 0.5 * sd * sd;
            v = log_exp ? exp(m + sd * E[c]) : pow(exp(1), m + sd * E[c]);
        } else continue;
        out[i] = v;
    }
}

int orc_rf_cholesky(int nd, int n, const double* xp, const int* type, double dr, const orc_rf_spec* s,
                    const double* zeta, int nzeta, double* out, int* ncell)
{
    for (int i = 0; i < n; i++) out[i] = NAN;
    rf_cells g;
    int err = rf_cells_make(nd, n, xp, type, dr, s, &g);
    *ncell = (err == 41) ? 0 : g.total;
    if (err) return err;
    if (nzeta < g.total) { rf_cells_free(&g); return 41; }
    double* L = rf_factor(nd, &g, s);
    double* E = (double*)malloc(sizeof(double) * (size_t)g.total);
    rf_gemv(L, g.total, zeta, 1, E);
    rf_assign(n, type, &g, E, s, s->type, nd - 1, 0, out);
    free(L); free(E);
    rf_cells_free(&g);
    return 0;
}

/* the correlation coefficient of the underlying normals and the rows of the
 * 2 x 2 factor (CPP_17-5:206-225, 761-779) */
static void rf_pair_factor(const orc_rf_spec* s0, const orc_rf_spec* s1, double coe, double cm[4])
{
    double coefficient;
    if (s0->type == 2) {
        coefficient = log(1.0 + coe * (s0->sd_value / s0->mean_value) * (s1->sd_value / s1->mean_value));
        coefficient = coefficient / sqrt(log(1.0 + s0->sd_value * s0->sd_value / s0->mean_value / s0->mean_value) *
                                         log(1.0 + s1->sd_value * s1->sd_value / s1->mean_value / s1->mean_value));
    } else coefficient = coe;
    cm[0] = 1.0; cm[1] = coefficient; cm[2] = 0.0; cm[3] = sqrt(1.0 - coefficient * coefficient);
}

int orc_rf_cholesky_corr(int nd, int n, const double* xp, const int* type, double dr, const orc_rf_spec* s0,
                         const orc_rf_spec* s1, double coe, const double* u2, int nu, double* out, int* ncell)
{
    for (int i = 0; i < 2 * n; i++) out[i] = NAN;
    rf_cells g;
    int err = rf_cells_make(nd, n, xp, type, dr, s0, &g);
    *ncell = (err == 41) ? 0 : g.total;
    if (err) return err;
    if (nu < g.total) { rf_cells_free(&g); return 41; }
    const int total = g.total;
    /* both members take the friction field's lengths and type (psv_temp) */
    double* L = rf_factor(nd, &g, s0);
    double cm[4];
    rf_pair_factor(s0, s1, coe, cm);
    /* zeta = u2 cov (matrix_multi(vec_zeta_1, covariance_mat, ...)) */
    double* z = (double*)malloc(sizeof(double) * 2 * (size_t)total);
    for (int i = 0; i < total; i++)
        for (int j = 0; j < 2; j++) {
            double t = 0.0;
            for (int k = 0; k < 2; k++) t = t + u2[(size_t)i * 2 + k] * cm[k * 2 + j];
            z[(size_t)i * 2 + j] = t;
        }
    double* E = (double*)malloc(sizeof(double) * (size_t)total);
    const orc_rf_spec* sp[2] = {s0, s1};
    for (int j = 0; j < 2; j++) {
        rf_gemv(L, total, z + j, 2, E);
        /* the fluid members of the 3-D field read their depth on y */
        const int axis = (nd == 3 && sp[j]->no >= 4) ? 1 : nd - 1;
        rf_assign(n, type, &g, E, sp[j], s0->type, axis, 1, out + (size_t)j * n);
    }
    free(L); free(z); free(E);
    rf_cells_free(&g);
    return 0;
}

int orc_rv_corr(int n, const int* type, const orc_rf_spec* s0, const orc_rf_spec* s1, double coe, const double u2[2],
                double* out)
{
    for (int i = 0; i < 2 * n; i++) out[i] = NAN;
    double cm[4], z1[2];
    rf_pair_factor(s0, s1, coe, cm);
    for (int j = 0; j < 2; j++) {
        double t = 0.0;
        for (int k = 0; k < 2; k++) t = t + u2[k] * cm[k * 2 + j];
        z1[j] = t;
    }
    /* friction takes zeta_1[1], cohesion zeta_1[0] (CPP_17-5:783-863) */
    const orc_rf_spec* sp[2] = {s0, s1};
    const int want = s0->no <= 3 ? 2 : 1;
    for (int j = 0; j < 2; j++) {
        double mean = sp[j]->mean_value, sd = sp[j]->sd_value, v;
        const double zz = z1[1 - j];
        if (s0->type == 1) v = mean + sd * zz;
        else if (s0->type == 2) {
            sd = sqrt(log(1.0 + (sd / mean) * (sd / mean)));
            mean = log(mean) - 0.5 * sd * sd;
            v = exp(mean + sd * zz);
        } else continue;
        for (int i = 0; i < n; i++)
            if (type[i] == want) out[(size_t)j * n + i] = v;
    }
    return 0;
}
