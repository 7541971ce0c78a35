// sph_kernels_bulk32.cu -- the FP32-bulk form of the step's physics kernels.
//
// The same kernel source as sph_kernels.cu, built with SPH_BULK32: the pair
// arithmetic of the neighbour passes runs in FP32 with Kahan-compensated sums
// (positions, velocities, densities, stresses, time integration and the
// constitutive update stay FP64).  This file is compiled with contraction of
// multiply-adds allowed; the FP64 drop-in form is not.
#define SPH_BULK32 1
#include "sph_kernels.cu"
