/*
 * sph_oracle.h -- CPU restatement of the reference's per-step particle loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the GPU engine:
 * tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py may
 * load it; the engine (libsphgpu) never links or calls it.
 *
 * It restates, in plain C over structure-of-arrays state, the functions of
 * wodexinxin2015/MultiPhase-SPH-Solver that SPH_Calculation calls each step
 * (CPP_1-SPHLoops.cpp:523-753), each function citing the reference
 * file:line it follows.  It is single-threaded and deterministic.  Two
 * orders are available for the passes the reference runs in place
 * (Shepard density filter, stress/strain regularisation):
 *   ORC_INPLACE  - sequential in-place update in particle order, which is
 *                  what the reference computes when run with one thread;
 *   ORC_JACOBI   - every particle reads the values from before the pass,
 *                  which is the order the GPU engine implements.
 * The restatement is pinned against the reference itself (compiled here
 * from its own sources into oracle/_ref) by tests/test_oracle_vs_reference.py.
 */
#ifndef SPH_ORACLE_H
#define SPH_ORACLE_H

#include "../include/sphgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_JACOBI  0
#define ORC_INPLACE 1

/* Evaluation of the equation of state's pow(x, 7.0) (CPP_7-1-eos_CR.cpp:28,40):
 *   ORC_POW_LIBM - the C library's pow(), as the reference calls it;
 *   ORC_POW_CR   - x^7 correctly rounded (double-double product chain), the
 *                  value the GPU engine computes.  glibc's pow differs from
 *                  the correctly rounded value on about 0.1% of inputs near 1
 *                  by one unit in the last place. */
#define ORC_POW_LIBM 0
#define ORC_POW_CR   1

typedef struct orc_ctx orc_ctx;

orc_ctx* orc_create(const sphgpu_params* p);
void     orc_destroy(orc_ctx* c);
int      orc_set_field(orc_ctx* c, const char* name, const void* host, size_t count);
int      orc_get_field(orc_ctx* c, const char* name, void* host, size_t count);
int      orc_set_materials(orc_ctx* c, const sphgpu_fluid* fluid, const sphgpu_soil* soil, int n);
void     orc_set_mode(orc_ctx* c, int mode);
void     orc_set_pow_mode(orc_ctx* c, int pow_mode);
double   orc_pow7(double x);   /* the ORC_POW_CR evaluation */
int      orc_get_step(const orc_ctx* c);
/* parttocell + partisearching for the current step; neighbour lists copied
 * out as in Par_Cell (influ 1-based, 100 slots per particle). */
int      orc_nnps(orc_ctx* c, int* ninflu, int* influ, double* wij);
int      orc_step(orc_ctx* c, int nsteps);
/* rainfall (flr == 1): the Para_Rain record, and its nrain as the steps leave it */
int      orc_set_rain(orc_ctx* c, const sphgpu_rain* rain);
int      orc_get_rain(const orc_ctx* c, sphgpu_rain* rain);
/* the vibration table (flv 1, 2): Para_Vibra's ttime, nsteps, sttime, edtime
 * and nsteps x 3 loads; 7 for nsteps < 1, as initial_pro */
int      orc_set_vibration(orc_ctx* c, double ttime, int nsteps, double sttime, double edtime, const double* loads);

#ifdef __cplusplus
}
#endif
#endif
