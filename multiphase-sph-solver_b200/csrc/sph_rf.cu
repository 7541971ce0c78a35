// sph_rf.cu -- the correlation-matrix random fields on the device
// (clFSpatialVariability_Fun::nonstationary_random_2D / _3D,
// CPP_17-3-Nonstationary-RF.cpp:76-849, flspv 3; and
// nonstationary_correlated_random_2D / _3D,
// CPP_17-5-Nonstationary-Correlated-RF.cpp:87-735, flspv 4).
//
// The reference divides the widened non-boundary box into cells of cell_ndx
// spacings, forms the correlation matrix of the cell centres, factors it by a
// row-oriented Cholesky with the diagonal's radicand floored at 1e-6,
// multiplies the factor by standard normals and gives every particle of a
// cell the cell's value.  Here every stage runs on the GPU:
//   k_rf_cells   the cell of each particle and the per-cell counts (a cell of
//                more than 39 particles is the reference's error 42)
//   k_rf_corr    the correlation matrix, one thread per entry
//   k_rf_diag    a 64 x 64 diagonal block factored in shared memory
//   k_rf_panel   the rows below it solved against it
//   k_rf_update  the trailing lower triangle less the panel's outer product
//                (64 x 64 output tiles from shared memory)
//   k_rf_gemv    E = L zeta, one warp per row
//   k_rf_assign  each particle's value from its cell (normal or lognormal map
//                with the depth trend, as the reference writes it)
// The blocked factorisation adds its products in another order than the
// reference's row sums, so values agree to rounding, not bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#define RF_B 64
#define RF_MAXP 39

namespace {

struct RFArgs {
    int ndim, n, no, type, flag_auto;
    int depth_axis;          // the centre coordinate the depth trend reads
    int log_exp;             // lognormal map as exp(.) (1) or pow(e, .) (0)
    int nc[3], total;
    double base[3], cdx, dr;
    double mean_value, sd_value, coe_depth, rl[3], beta, beta1, soil_max, water_max;
};

__device__ __forceinline__ void centre(const RFArgs& a, int c, double x[3])
{
    const int i = c % a.nc[0], j = (c / a.nc[0]) % a.nc[1], k = c / (a.nc[0] * a.nc[1]);
    x[0] = a.base[0] + ((double)i + 0.5) * a.cdx;
    x[1] = a.base[1] + ((double)j + 0.5) * a.cdx;
    x[2] = (a.ndim == 3) ? a.base[2] + ((double)k + 0.5) * a.cdx : 0.0;
}

__global__ void k_rf_cells(RFArgs a, const double* xh, const int* type, int* cell, int* count, int* err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    cell[i] = -1;
    if (a.ndim == 2 && !(type[i] == 1 || type[i] == 2)) return;
    const double* p = xh + 4 * (size_t)i;
    int np[3] = {0, 0, 0};
    for (int d = 0; d < a.ndim; d++) np[d] = (int)(fabs(p[d] - a.base[d]) / a.cdx);
    for (int d = 0; d < a.ndim; d++)
        if (np[d] < 0 || np[d] >= a.nc[d]) { err[0] = 1; return; }
    const int c = (a.ndim == 2) ? np[1] * a.nc[0] + np[0] : np[2] * a.nc[0] * a.nc[1] + np[1] * a.nc[0] + np[0];
    if (atomicAdd(&count[c], 1) >= RF_MAXP) err[1] = 1;
    cell[i] = c;
}

// the autocorrelation of two cell centres (CPP_17-3:210-224, 600-616)
__global__ void k_rf_corr(RFArgs a, double* C)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (j >= a.total) return;
    double xk[3], xj[3];
    centre(a, k, xk);
    centre(a, j, xj);
    const double dx = fabs(xk[0] - xj[0]), dy = fabs(xk[1] - xj[1]);
    const double pi = 3.141592653;
    double acf;
    if (a.ndim == 2) {
        if (a.flag_auto == 1) acf = exp(-2.0 * (dx / a.rl[0] + dy / a.rl[1]));
        else if (a.flag_auto == 2) acf = exp(-pi * (pow(dx / a.rl[0], 2.0) + pow(dy / a.rl[1], 2.0)));
        else acf = exp(-2.0 * ((dx * cos(a.beta) + dy * sin(a.beta)) / a.rl[0] +
                               (-dx * sin(a.beta) + dy * cos(a.beta)) / a.rl[1]));
    } else {
        const double dz = fabs(xk[2] - xj[2]);
        const double t0 = dx * cos(a.beta1) + dy * sin(a.beta1);
        const double t1 = (-dx * sin(a.beta1) + dy * cos(a.beta1)) * cos(a.beta) + dz * sin(a.beta);
        const double t2 = -(-dx * sin(a.beta1) + dy * cos(a.beta1)) * sin(a.beta) + dz * cos(a.beta);
        if (a.flag_auto == 1) acf = exp(-2.0 * (dx / a.rl[0] + dy / a.rl[1] + dz / a.rl[2]));
        else if (a.flag_auto == 2)
            acf = exp(-pi * (pow(dx / a.rl[0], 2.0) + pow(dy / a.rl[1], 2.0) + pow(dz / a.rl[2], 2.0)));
        else acf = exp(-2.0 * (t0 / a.rl[0] + t1 / a.rl[1] + t2 / a.rl[2]));
    }
    C[(size_t)k * a.total + j] = acf;
}

// the diagonal block [k0, k0 + bs) factored in place (lower triangle),
// right-looking inside the block; the radicand floored at 1e-6
__global__ void __launch_bounds__(RF_B) k_rf_diag(double* A, int n, int k0, int bs)
{
    __shared__ double s[RF_B][RF_B + 1];
    const int t = threadIdx.x;
    for (int j = 0; j < bs; j++) s[t][j] = (t < bs) ? A[(size_t)(k0 + t) * n + k0 + j] : 0.0;
    __syncthreads();
    for (int k = 0; k < bs; k++) {
        if (t == k) {
            const double v = s[k][k];
            s[k][k] = sqrt(v > 1.0e-6 ? v : 1.0e-6);
        }
        __syncthreads();
        if (t > k && t < bs) s[t][k] = s[t][k] / s[k][k];
        __syncthreads();
        if (t > k && t < bs)
            for (int j = k + 1; j <= t; j++) s[t][j] = s[t][j] - s[t][k] * s[j][k];
        __syncthreads();
    }
    if (t < bs)
        for (int j = 0; j < bs; j++) A[(size_t)(k0 + t) * n + k0 + j] = (j <= t) ? s[t][j] : 0.0;
}

// rows i >= k0 + bs of the panel: L[i][k0 .. k0 + bs) from the factored
// diagonal block (forward substitution per row)
__global__ void __launch_bounds__(128) k_rf_panel(double* A, int n, int k0, int bs)
{
    __shared__ double Lk[RF_B][RF_B + 1];
    for (int e = threadIdx.x; e < bs * bs; e += blockDim.x) {
        const int r = e / bs, c = e % bs;
        Lk[r][c] = A[(size_t)(k0 + r) * n + k0 + c];
    }
    __syncthreads();
    const int i = k0 + bs + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double row[RF_B];
    for (int k = 0; k < bs; k++) row[k] = A[(size_t)i * n + k0 + k];
    for (int k = 0; k < bs; k++) {
        double v = row[k];
        for (int j = 0; j < k; j++) v = v - row[j] * Lk[k][j];
        row[k] = v / Lk[k][k];
    }
    for (int k = 0; k < bs; k++) A[(size_t)i * n + k0 + k] = row[k];
}

// the trailing lower triangle, A[i][j] -= sum_k L[i][k] L[j][k] over the
// panel's columns, for k0 + bs <= j <= i < n: 64 x 64 output tiles, the
// panel's columns staged 16 at a time (k-major, one column of padding so the
// transposing stores fall in distinct banks); each thread owns rows
// tr + 16 p and columns tc + 16 q, so the tile reads and writes are 128-byte
// runs
__global__ void __launch_bounds__(256) k_rf_update(double* A, int n, int k0, int bs)
{
    const int r0 = k0 + bs + blockIdx.y * RF_B, c0 = k0 + bs + blockIdx.x * RF_B;
    if (c0 > r0 + RF_B - 1 || r0 >= n) return;        // wholly above the diagonal
    __shared__ double As[16][RF_B + 1], Bs[16][RF_B + 1];
    const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
    double acc[4][4];
    for (int p = 0; p < 4; p++)
        for (int q = 0; q < 4; q++) acc[p][q] = 0.0;
    for (int kc = 0; kc < bs; kc += 16) {
        __syncthreads();
        for (int e = threadIdx.x; e < 16 * RF_B; e += blockDim.x) {
            const int k = e % 16, r = e / 16;
            const bool in = kc + k < bs;
            As[k][r] = (in && r0 + r < n) ? A[(size_t)(r0 + r) * n + k0 + kc + k] : 0.0;
            Bs[k][r] = (in && c0 + r < n) ? A[(size_t)(c0 + r) * n + k0 + kc + k] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; k++) {
            double a[4], b[4];
#pragma unroll
            for (int p = 0; p < 4; p++) { a[p] = As[k][tr + 16 * p]; b[p] = Bs[k][tc + 16 * p]; }
#pragma unroll
            for (int p = 0; p < 4; p++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[p][q] = fma(a[p], b[q], acc[p][q]);
        }
    }
    for (int p = 0; p < 4; p++)
        for (int q = 0; q < 4; q++) {
            const int i = r0 + tr + 16 * p, j = c0 + tc + 16 * q;
            if (i < n && j <= i) A[(size_t)i * n + j] = A[(size_t)i * n + j] - acc[p][q];
        }
}

// E = L zeta over the lower triangle, one warp per row
__global__ void k_rf_gemv(const double* L, int n, const double* zeta, double* E)
{
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= n) return;
    double t = 0.0;
    for (int j = lane; j <= row; j += 32) t = t + L[(size_t)row * n + j] * zeta[j];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) E[row] = t;
}

// each particle's value (CPP_17-3:235-450, 17-5:222-402): its cell's normal
// value with the depth trend from soil_max (soil members) or water_max (fluid
// members), or the lognormal map with the trend from soil_max for every
// member, as the reference writes them.  The depth is the centre's last
// coordinate, except for the fluid members of the correlated 3-D field, which
// read y (17-5:655-735); the correlated field maps lognormals through exp,
// the single field through pow(e, .).
__global__ void k_rf_assign(RFArgs a, const int* cell, const int* type, const double* E, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int c = cell[i];
    const bool soil = a.no <= 3;
    double v = __longlong_as_double(0x7ff8000000000000LL);
    if (c >= 0 && type[i] == (soil ? 2 : 1)) {
        double x[3];
        centre(a, c, x);
        const double depth = x[a.depth_axis];
        if (a.type == 1) {
            const double top = soil ? a.soil_max : a.water_max;
            if (top > depth) v = a.mean_value + a.coe_depth * (top - depth) + a.sd_value * E[c];
            else v = a.mean_value + a.sd_value * E[c];
        } else {
            double m = (a.soil_max > depth) ? a.mean_value + a.coe_depth * (a.soil_max - depth) : a.mean_value;
            const double sd = sqrt(log(1.0 + (a.sd_value / m) * (a.sd_value / m)));
            m = log(m) - 0.5 * sd * sd;
            v = a.log_exp ? exp(m + sd * E[c]) : pow(exp(1.0), m + sd * E[c]);
        }
    }
    out[i] = v;
}

RFArgs rf_args(const int* ip, const double* dp)
{
    RFArgs a;
    a.ndim = ip[0]; a.n = ip[1]; a.no = ip[2]; a.type = ip[3]; a.flag_auto = ip[4];
    for (int d = 0; d < 3; d++) { a.nc[d] = ip[5 + d]; a.base[d] = dp[d]; a.rl[d] = dp[3 + d]; }
    a.depth_axis = ip[8]; a.log_exp = ip[9];
    a.total = a.nc[0] * a.nc[1] * a.nc[2];
    a.cdx = dp[6]; a.dr = dp[7];
    a.mean_value = dp[8]; a.sd_value = dp[9]; a.coe_depth = dp[10];
    a.beta = dp[11]; a.beta1 = dp[12]; a.soil_max = dp[13]; a.water_max = dp[14];
    return a;
}

}  // namespace

// The host passes the field's description as two arrays:
//   ip: ndim, n, no, type, flag_auto, nc[3], depth axis, lognormal form
//   dp: base[3], rl[3], cell edge, dr, mean, sd, coe_depth, beta, beta_1
//       (radians), soil_max, water_max
// Positions are (x, y, z, h) records, 4 doubles per particle.

// Stage 1: the cell of each particle (-1 for none) and the per-cell counts
// (d_count zeroed by the caller); d_err[0] is set for a particle outside the
// cells, d_err[1] for a cell of more than 39 particles (d_err zeroed).
extern "C" int sphk_rf_cells(const int* ip, const double* dp, const double* d_xh, const int* d_type, int* d_cell,
                             int* d_count, int* d_err, cudaStream_t st)
{
    const RFArgs a = rf_args(ip, dp);
    if (a.n > 0) k_rf_cells<<<(a.n + 255) / 256, 256, 0, st>>>(a, d_xh, d_type, d_cell, d_count, d_err);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Stage 2: the correlation matrix of the cell centres into d_C (total x
// total, row-major) and its lower Cholesky factor in place (the entries above
// the diagonal are left undefined).
extern "C" int sphk_rf_factor(const int* ip, const double* dp, double* d_C, cudaStream_t st)
{
    const RFArgs a = rf_args(ip, dp);
    const int T = a.total;
    k_rf_corr<<<dim3((T + 255) / 256, T), 256, 0, st>>>(a, d_C);
    for (int k0 = 0; k0 < T; k0 += RF_B) {
        const int bs = (T - k0) < RF_B ? (T - k0) : RF_B;
        k_rf_diag<<<1, RF_B, 0, st>>>(d_C, T, k0, bs);
        const int rest = T - k0 - bs;
        if (rest > 0) {
            k_rf_panel<<<(rest + 127) / 128, 128, 0, st>>>(d_C, T, k0, bs);
            const int tiles = (rest + RF_B - 1) / RF_B;
            k_rf_update<<<dim3(tiles, tiles), 256, 0, st>>>(d_C, T, k0, bs);
        }
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Stage 3: E = L zeta and each particle's value into d_out (NaN where the
// field writes none).
extern "C" int sphk_rf_assign(const int* ip, const double* dp, const double* d_L, const double* d_zeta, double* d_E,
                              const int* d_cell, const int* d_type, double* d_out, cudaStream_t st)
{
    const RFArgs a = rf_args(ip, dp);
    const int T = a.total;
    k_rf_gemv<<<(T * 32 + 255) / 256, 256, 0, st>>>(d_L, T, d_zeta, d_E);
    if (a.n > 0) k_rf_assign<<<(a.n + 255) / 256, 256, 0, st>>>(a, d_cell, d_type, d_E, d_out);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
