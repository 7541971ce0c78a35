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

int orc_rf_cholesky(int nd, int n, const double* xp, const int* type, double dr, const orc_rf_spec* s,
                    const double* zeta, int nzeta, double* out, int* ncell)
{
    double xmin[3] = {0, 0, 0}, xmax[3] = {0, 0, 0}, base[3] = {0, 0, 0};
    /* the non-boundary box widened by 10% per side (CPP_17-3:100-105, 483-489) */
    for (int d = 0; d < nd; d++) {
        xmin[d] = s->nb_min[d] - 0.1 * (s->nb_max[d] - s->nb_min[d]);
        xmax[d] = s->nb_max[d] + 0.1 * (s->nb_max[d] - s->nb_min[d]);
    }
    const double cdx = s->cell_ndx * dr;
    int nc[3] = {1, 1, 1};
    for (int d = 0; d < nd; d++) nc[d] = (int)((xmax[d] - xmin[d]) / cdx) + 1;
    const int total = nc[0] * nc[1] * nc[2];
    *ncell = total;
    for (int i = 0; i < n; i++) out[i] = NAN;
    if (!(total > 0 && total < 15000)) return 41;
    if (nzeta < total) return 41;
    for (int d = 0; d < nd; d++) base[d] = -(nc[d] * cdx - (xmax[d] - xmin[d])) / 2.0 + 0.01 * dr + xmin[d];
    /* cell of each particle (2-D: water and soil; 3-D: every particle) */
    int* cell = (int*)malloc(sizeof(int) * (size_t)n);
    int* count = (int*)calloc((size_t)total, sizeof(int));
    int err = 0;
    for (int i = 0; i < n && !err; i++) {
        cell[i] = -1;
        if (nd == 2 && !(type[i] == 1 || type[i] == 2)) continue;
        int np[3] = {0, 0, 0};
        for (int d = 0; d < nd; d++) np[d] = (int)(fabs(xp[(size_t)i * 3 + d] - base[d]) / cdx);
        const int c = (nd == 2) ? np[1] * nc[0] + np[0] : np[2] * nc[0] * nc[1] + np[1] * nc[0] + np[0];
        /* a particle beyond the cells (the reference indexes past its array
         * there): refused */
        if (c < 0 || c >= total || np[0] >= nc[0] || np[1] >= nc[1] || (nd == 3 && np[2] >= nc[2])) {
            err = 100;
            break;
        }
        if (count[c] < RF_MAXP) { count[c]++; cell[i] = c; }
        else err = 42;
    }
    if (err) { free(cell); free(count); return err; }
    /* cell centres */
    double* cx = (double*)malloc(sizeof(double) * 3 * (size_t)total);
    for (int k = 0; k < nc[2]; k++)
        for (int j = 0; j < nc[1]; j++)
            for (int i = 0; i < nc[0]; i++) {
                const int c = k * nc[0] * nc[1] + j * nc[0] + i;
                cx[c * 3 + 0] = base[0] + ((double)i + 0.5) * cdx;
                cx[c * 3 + 1] = base[1] + ((double)j + 0.5) * cdx;
                cx[c * 3 + 2] = (nd == 3) ? base[2] + ((double)k + 0.5) * cdx : 0.0;
            }
    /* the correlation matrix (CPP_17-3:210-224, 600-616) */
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
    /* E = L zeta (matrix_multi, CPP_17-3:20-30) */
    double* E = (double*)malloc(sizeof(double) * (size_t)total);
    for (int i = 0; i < total; i++) {
        double t = 0.0;
        for (int j = 0; j < total; j++) t = t + L[(size_t)i * total + j] * zeta[j];
        E[i] = t;
    }
    /* the value of each cell, written into its particles of the field's
     * phase (CPP_17-3:235-450): the depth trend of a normal field from
     * soil_max (soil members) or water_max (fluid members), of a lognormal
     * one from soil_max for every member, as the reference has it */
    const int soil = s->no <= 3;
    const int want = soil ? 2 : 1;
    const int ax = nd - 1;
    for (int i = 0; i < n; i++) {
        const int c = cell[i];
        if (c < 0 || type[i] != want) continue;
        const double depth = cx[c * 3 + ax];
        double v;
        if (s->type == 1) {
            const double top = soil ? s->soil_max : s->water_max;
            if (top > depth) v = s->mean_value + s->coe_depth * (top - depth) + s->sd_value * E[c];
            else v = s->mean_value + s->sd_value * E[c];
        } else {
            double m = (s->soil_max > depth) ? s->mean_value + s->coe_depth * (s->soil_max - depth) : s->mean_value;
            const double sd = sqrt(log(1.0 + (s->sd_value / m) * (s->sd_value / m)));
            m = log(m) - 0.5 * sd * sd;
            v = pow(exp(1), m + sd * E[c]);
        }
        out[i] = v;
    }
    free(cell); free(count); free(cx); free(C); free(L); free(E);
    return 0;
}
