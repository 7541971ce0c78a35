/*
 * kl_oracle.h -- CPU restatement of the reference's Karhunen-Loeve random
 * field generator (CPP_17-1_K-L_expansion_non.cpp, CPP_17-2_K-L_expansion_corr.cpp).
 * TEST INFRASTRUCTURE ONLY (the checker of the engine's sphgpu_kl_* path).
 */
#ifndef KL_ORACLE_H
#define KL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One field: Para_SpatialVariability (Class_spatial_variability.h:46-66) plus
 * the domain values the generator derives from Cell_Con. */
typedef struct orc_kl_spec {
    int no;                  /* 0 soil fai, 1 soil c, 2 soil cop, 3 soil ds, 4 fluid fai, 5 fluid c */
    int type;                /* 1 normal, 2 lognormal */
    double mean_value, sd_value, coe_depth;
    double rl[3];            /* correlation lengths */
    double a[3], x_trans[3]; /* half extents and centre of the field's domain */
    double soil_max, water_max;
} orc_kl_spec;

/* wi: K x 3 (row-major, column d = axis d) */
void orc_kl_solve_wi(double* wi, const double a[3], const double rl[3], int ndim, int K);
/* eigval: K; order: K x 3 */
int  orc_kl_ramdai(double* eigval, int* order, const double* wi, const double rl[3], int ndim, int K);
/* out[i] for the particles the field writes (written[i] = 1) */
int  orc_kl_field(int ndim, int n, const double* xp, const int* type, const orc_kl_spec* s, const double* wi,
                  const double* eigval, const int* order, const double* xi, int K, double* out, int* written);
/* the field domain of SpatialVariables_Generate_2D/3D (CPP_17-1:70-90, 166-186) */
void orc_kl_domain(int ndim, const double nb_min[3], const double nb_max[3], double a[3], double x_trans[3]);
/* the friction/cohesion correlation of SpatialVariables_Generate_*_corr
 * (CPP_17-2:115-168): u2 is K x 2 standard normals */
void orc_kl_correlate(const double* u2, double coefficient, double* xi_fai, double* xi_c, int K);

#ifdef __cplusplus
}
#endif
#endif
