/*
 * rf_oracle.h -- CPU restatement of the reference's correlation-matrix
 * (Cholesky) random field, nonstationary_random_2D / _3D
 * (CPP_17-3-Nonstationary-RF.cpp:76-458, 460-849; flspv 3), of its
 * correlated form (nonstationary_correlated_random_2D / _3D,
 * CPP_17-5-Nonstationary-Correlated-RF.cpp:87-735; flspv 4) and of the
 * correlated random variables (random_variable_generate, CPP_17-5:738-863;
 * flspv 5).
 * TEST INFRASTRUCTURE ONLY (the checker of the engine's sphgpu_rf_generate,
 * sphgpu_rf_generate_corr and sphgpu_rv_generate_corr).
 */
#ifndef RF_ORACLE_H
#define RF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One field: Para_SpatialVariability (no, type, mean, sd, lengths,
 * coe_depth), the Flag_SpatialVariability members the generator reads
 * (cell_ndx, flag_auto, beta, beta_1, Class_spatial_variability.h:9-28) and
 * the Cell_Con values (the non-boundary box, soil_max / water_max along the
 * depth axis). */
typedef struct orc_rf_spec {
    int no;                  /* 0 soil fai, 1 soil c, 2 soil cop, 3 soil ds, 4 fluid fai, 5 fluid c */
    int type;                /* 1 normal, 2 lognormal */
    double mean_value, sd_value, coe_depth;
    double rl[3];
    double cell_ndx;
    int flag_auto;
    double beta, beta_1;     /* degrees */
    double nb_min[3], nb_max[3];
    double soil_max, water_max;
} orc_rf_spec;

/* The field for n particles (positions xp, n x 3; types), with the cell
 * normals zeta (one per cell, cells numbered as the reference numbers them;
 * *ncell receives their count).  out[i] gets the value the field writes into
 * particle i, NaN where it writes none.  Returns 0, 41 (no cells or 15,000 or
 * more) or 42 (a cell with more than 39 particles), as the reference, or 100
 * for a particle outside the cells (which the reference does not check). */
int orc_rf_cholesky(int ndim, int n, const double* xp, const int* type, double dr, const orc_rf_spec* s,
                    const double* zeta, int nzeta, double* out, int* ncell);

/* flspv 4: s0 the friction field (no 0 or 4), s1 the cohesion field (no 1 or
 * 5) of one phase, coe the friction-cohesion correlation; u2 holds ncell x 2
 * normals (the reference's vec_zeta_1).  out: 2 x n values (friction, then
 * cohesion).  s1 contributes its mean, sd and coe_depth only; the cells,
 * lengths, kernel and distribution type are s0's.  Codes as above. */
int orc_rf_cholesky_corr(int ndim, int n, const double* xp, const int* type, double dr, const orc_rf_spec* s0,
                         const orc_rf_spec* s1, double coe, const double* u2, int nu, double* out, int* ncell);

/* flspv 5: one correlated pair from the normals u2 for every particle of the
 * phase; out: 2 x n values. */
int orc_rv_corr(int n, const int* type, const orc_rf_spec* s0, const orc_rf_spec* s1, double coe, const double u2[2],
                double* out);

#ifdef __cplusplus
}
#endif
#endif
