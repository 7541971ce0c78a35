/*
 * kl_oracle.c -- CPU restatement of the reference's Karhunen-Loeve random
 * field generator (CPP_17-1_K-L_expansion_non.cpp, CPP_17-2_K-L_expansion_corr.cpp).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the engine's K-L path
 * (sphgpu_kl_generate); the engine never links it.
 *
 * The reference draws the standard-normal coefficients from a time-seeded
 * std::default_random_engine (generate_SND, CPP_17-1:24-33); here they are
 * an input (xi), so a run is reproducible and comparable.  Everything else
 * follows the reference's arithmetic in its order:
 *   orc_kl_solve_wi      solve_wi      (CPP_17-1:275-345): bisection roots of
 *                        2/l - w tan(w a) (odd terms) and 2/l tan(w a) + w (even)
 *   orc_kl_ramdai        solve_ramdai  (CPP_17-1:348-442): 1-D eigenvalues
 *                        4 l / (4 + w^2 l^2), their products over the 2 or 3
 *                        axes and the K largest by repeated first-maximum
 *                        search (ties: lowest index in (m, n, k) scan order)
 *   orc_kl_field         solve_h_2D / solve_h_3D (CPP_17-1:486-700): the
 *                        eigenfunctions solve_faii (:44-59), the truncated sum
 *                        H = sum_j sqrt(lambda_j) phi_j(x) xi_j and the normal
 *                        or lognormal map with the depth trend
 * The reference fixes K = klterm = 200 (CPP_17-1:20); K is a parameter here.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "kl_oracle.h"

static const double KL_PI = 3.141592653;      /* Header_Parameters.h:10 */
#define KL_PREC 1.0e-6                        /* CPP_17-1:21 */

void orc_kl_solve_wi(double* wi, const double a_x[3], const double rl[3], int ndim, int K)
{
    double* up = (double*)malloc(sizeof(double) * K);
    double* lo = (double*)malloc(sizeof(double) * K);
    for (int d = 0; d < ndim; d++) {
        const double a = a_x[d], dira = rl[d];
        for (int i = 0; i < K; i++) {
            if ((i + 1) % 2 == 1) {
                up[i] = (i + 0.5) * KL_PI / a;
                lo[i] = i * KL_PI / a;
            } else {
                up[i] = (i + 1.0) * KL_PI / a;
                lo[i] = (i + 0.5) * KL_PI / a;
            }
        }
        for (int i = 0; i < K; i++) {
            double x1 = lo[i] + KL_PREC, x2 = up[i] - KL_PREC, xm, f1, fm;
            if ((i + 1) % 2 == 1) {
                xm = (x1 + x2) * 0.5;
                do {
                    f1 = 2.0 / dira - x1 * tan(x1 * a);
                    fm = 2.0 / dira - xm * tan(xm * a);
                    if ((f1 * fm) < 0.0) x2 = xm;
                    else x1 = xm;
                    xm = (x1 + x2) * 0.5;
                } while (fabs(fm) > KL_PREC);
            } else {
                xm = (x1 + x2) / 2.0;
                do {
                    f1 = 2.0 / dira * tan(x1 * a) + x1;
                    fm = 2.0 / dira * tan(xm * a) + xm;
                    if ((f1 * fm) < 0.0) x2 = xm;
                    else x1 = xm;
                    xm = (x1 + x2) * 0.5;
                } while (fabs(fm) > KL_PREC);
            }
            wi[i * 3 + d] = xm;
        }
    }
    free(up);
    free(lo);
}

static double ramdai(double dirac, double w) { return 4.0 * dirac / (4.0 + w * w * dirac * dirac); }

int orc_kl_ramdai(double* eigval, int* order, const double* wi, const double rl[3], int ndim, int K)
{
    double* r = (double*)malloc(sizeof(double) * 3 * K);
    for (int i = 0; i < K; i++) order[i * 3 + 0] = order[i * 3 + 1] = order[i * 3 + 2] = i;
    for (int d = 0; d < ndim; d++)
        for (int i = 0; i < K; i++) r[i * 3 + d] = ramdai(rl[d], wi[i * 3 + d]);
    const size_t total = (ndim == 2) ? (size_t)K * K : (size_t)K * K * K;
    double* prod = (double*)malloc(sizeof(double) * total);
    if (!prod) { free(r); return 1; }
    if (ndim == 2) {
        for (int i = 0; i < K; i++)
            for (int j = 0; j < K; j++) prod[(size_t)i * K + j] = r[i * 3 + 0] * r[j * 3 + 1];
    } else {
        for (int i = 0; i < K; i++)
            for (int j = 0; j < K; j++)
                for (int k = 0; k < K; k++)
                    prod[((size_t)i * K + j) * K + k] = r[i * 3 + 0] * r[j * 3 + 1] * r[k * 3 + 2];
    }
    /* K largest in the order of repeated first-maximum search */
    for (int t = 0; t < K; t++) {
        double best = -1.0;
        size_t at = 0;
        int found = 0;
        for (size_t q = 0; q < total; q++)
            if (best < prod[q]) { best = prod[q]; at = q; found = 1; }
        eigval[t] = best;
        if (found) {
            if (ndim == 2) {
                order[t * 3 + 0] = (int)(at / K);
                order[t * 3 + 1] = (int)(at % K);
            } else {
                order[t * 3 + 0] = (int)(at / ((size_t)K * K));
                order[t * 3 + 1] = (int)((at / K) % K);
                order[t * 3 + 2] = (int)(at % K);
            }
            prod[at] = -1.0;
        }
    }
    free(prod);
    free(r);
    return 0;
}

static double faii(double x, double a, double wi, int i)
{
    double alphai;
    if ((i + 1) % 2 == 1) {
        alphai = 1.0 / sqrt(sin(2.0 * wi * a) / 2.0 / wi + a);
        return alphai * cos(wi * x);
    }
    alphai = 1.0 / sqrt(-sin(2.0 * wi * a) / 2.0 / wi + a);
    return alphai * sin(wi * x);
}

int orc_kl_field(int ndim, int n, const double* xp, const int* type, const orc_kl_spec* s, const double* wi,
                 const double* eigval, const int* order, const double* xi, int K, double* out, int* written)
{
    double* ev = (double*)malloc(sizeof(double) * K);
    for (int i = 0; i < n; i++) {
        written[i] = 0;
        const int t = type[i];
        if (t == 0 || t == 7) continue;
        double xa[3];
        for (int d = 0; d < ndim; d++) xa[d] = xp[(size_t)i * 3 + d] - s->x_trans[d];
        for (int j = 0; j < K; j++) {
            double f = 1.0, fd[3];
            for (int d = 0; d < ndim; d++) {
                const int id = order[j * 3 + d];
                fd[d] = faii(xa[d], s->a[d], wi[id * 3 + d], id);
            }
            f = (ndim == 2) ? fd[0] * fd[1] : fd[0] * fd[1] * fd[2];
            ev[j] = f;
        }
        double mean;
        if (t == 2) mean = s->mean_value + (s->soil_max - xp[(size_t)i * 3 + 1]) * s->coe_depth;
        else if (t == 1) mean = s->mean_value + (s->water_max - xp[(size_t)i * 3 + 1]) * s->coe_depth;
        else mean = s->mean_value;
        double sigma;
        if (s->type == 1) {
            sigma = s->sd_value;
        } else if (s->type == 2) {
            sigma = sqrt(log(1.0 + (s->sd_value / mean) * (s->sd_value / mean)));
            mean = log(mean) - 0.5 * sigma * sigma;
        } else {
            free(ev);
            return 14;
        }
        double h = 0.0;
        for (int j = 0; j < K; j++) h = h + sqrt(eigval[j]) * ev[j] * xi[j];
        const int soil_field = (s->no >= 0 && s->no <= 3);
        if ((soil_field && t == 2) || (!soil_field && t == 1)) {
            out[i] = (s->type == 1) ? mean + h * sigma : exp(mean + h * sigma);
            written[i] = 1;
        }
    }
    free(ev);
    return 0;
}

void orc_kl_domain(int ndim, const double nb_min[3], const double nb_max[3], double a[3], double x_trans[3])
{
    double xmin[3] = {0, 0, 0}, xmax[3] = {0, 0, 0};
    for (int d = 0; d < ndim; d++) {
        xmin[d] = nb_min[d] - 0.2 * (nb_max[d] - nb_min[d]);
        xmax[d] = nb_max[d] + 0.2 * (nb_max[d] - nb_min[d]);
    }
    for (int d = 0; d < 3; d++) {
        x_trans[d] = (d < ndim) ? (xmax[d] + xmin[d]) / 2.0 : 0.0;
        a[d] = (d < ndim) ? (xmax[d] - xmin[d]) / 2.0 : 0.0;
    }
}

void orc_kl_correlate(const double* u2, double coefficient, double* xi_fai, double* xi_c, int K)
{
    /* covariance_mat = [1, coefficient; 0, sqrt(1 - coefficient^2)] and
     * zeta = uu_cfai (K x 2) * covariance_mat (CPP_17-2:120-168) */
    const double cm[4] = {1.0, coefficient, 0.0, sqrt(1.0 - coefficient * coefficient)};
    for (int i = 0; i < K; i++) {
        double z0 = 0.0, z1 = 0.0;
        z0 = z0 + u2[i * 2 + 0] * cm[0];
        z0 = z0 + u2[i * 2 + 1] * cm[2];
        z1 = z1 + u2[i * 2 + 0] * cm[1];
        z1 = z1 + u2[i * 2 + 1] * cm[3];
        xi_fai[i] = z0;
        xi_c[i] = z1;
    }
}
