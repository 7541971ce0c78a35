// sph_kl.cu -- Karhunen-Loeve random fields on the device
// (CPP_17-1_K-L_expansion_non.cpp, CPP_17-2_K-L_expansion_corr.cpp).
//
// The reference evaluates, per field, the 1-D eigenpairs of the exponential
// covariance on each axis (solve_wi: bisection roots; solve_ramdai: 1-D
// eigenvalues), keeps the K largest products of them over the 2 or 3 axes
// (a first-maximum search over K^2 or K^3 candidates, 1.6e9 comparisons in
// 3-D), and sums H(x) = sum_j sqrt(lambda_j) phi_j(x) xi_j per particle
// (solve_h_2D / solve_h_3D).  Here the roots and the per-term normalisation
// constants stay on the host in FP64 (the library's own tan / sin, a few
// hundred calls); the candidate products and their ordering, and the
// per-particle sums, run on the device:
//
//   k_kl_products   the K^ndim products lambda_m lambda_n (lambda_k), in the
//                   reference's multiplication order, keyed by their index
//   radix sort      descending by value; the sort is stable, so equal
//                   products keep ascending index order, which is the order
//                   the reference's repeated first-maximum search yields
//   k_kl_field      per particle: the K eigenfunction products, the FP64 sum
//                   in term order, the normal / lognormal map and the depth
//                   trend, written where the field applies (NaN elsewhere)
#include <cub/cub.cuh>
#include <cstdint>

#include "sph_device.cuh"

namespace {

template <int ND>
__global__ void k_kl_products(const double* __restrict__ r, int K, size_t total, double* keys, uint32_t* vals)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= total) return;
    double v;
    if (ND == 2) {
        const int m = (int)(q / K), n = (int)(q % K);
        v = r[m * 3 + 0] * r[n * 3 + 1];
    } else {
        const size_t KK = (size_t)K * K;
        const int m = (int)(q / KK), n = (int)((q / K) % K), k = (int)(q % K);
        v = r[m * 3 + 0] * r[n * 3 + 1] * r[k * 3 + 2];
    }
    keys[q] = v;
    vals[q] = (uint32_t)q;
}

// One K-L term on one axis: w, the normalisation alpha and the parity of the
// reference's 0-based term index (odd terms, (i + 1) % 2 == 1, use cos).
struct KLTerm { double w, alpha; int use_cos; int pad; };

struct KLFieldArgs {
    int n, ndim, K, no, type;
    double x_trans[3];
    double mean_value, sd_value, coe_depth, soil_max, water_max;
    const double* xh;          // (x, y, z, h) records
    const int* ptype;
    const KLTerm* terms;       // K x ndim
    const double* sqrt_eig;    // K
    const double* xi;          // K
    double* out;               // n
};

template <int ND>
__global__ void __launch_bounds__(128) k_kl_field(KLFieldArgs a)
{
    extern __shared__ unsigned char smem[];
    KLTerm* st = reinterpret_cast<KLTerm*>(smem);
    double* sc = reinterpret_cast<double*>(st + (size_t)a.K * ND);
    for (int t = threadIdx.x; t < a.K * ND; t += blockDim.x) st[t] = a.terms[t];
    for (int t = threadIdx.x; t < a.K; t += blockDim.x) {
        sc[2 * t] = a.sqrt_eig[t];
        sc[2 * t + 1] = a.xi[t];
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int t = a.ptype[i];
    const bool soil_field = a.no >= 0 && a.no <= 3;
    const bool writes = (soil_field && t == 2) || (!soil_field && t == 1);
    if (!writes) {
        a.out[i] = __longlong_as_double(0x7ff8000000000000ll);
        return;
    }
    const double2* rec = reinterpret_cast<const double2*>(a.xh) + 2 * (size_t)i;
    const double2 r0 = rec[0], r1 = rec[1];
    const double xp[3] = {r0.x, r0.y, r1.x};
    double xa[3];
    for (int d = 0; d < ND; d++) xa[d] = xp[d] - a.x_trans[d];
    double h = 0.0;
    for (int j = 0; j < a.K; j++) {
        double fd[ND];
        for (int d = 0; d < ND; d++) {
            const KLTerm q = st[j * ND + d];
            fd[d] = q.use_cos ? q.alpha * cos(q.w * xa[d]) : q.alpha * sin(q.w * xa[d]);
        }
        const double f = (ND == 2) ? fd[0] * fd[1] : fd[0] * fd[1] * fd[ND - 1];
        h = h + sc[2 * j] * f * sc[2 * j + 1];
    }
    // the depth trend reads the y coordinate in 2-D and in 3-D alike
    double mean;
    if (t == 2) mean = a.mean_value + (a.soil_max - xp[1]) * a.coe_depth;
    else mean = a.mean_value + (a.water_max - xp[1]) * a.coe_depth;
    double v;
    if (a.type == 1) {
        v = mean + h * a.sd_value;
    } else {
        const double sigma = sqrt(log(1.0 + (a.sd_value / mean) * (a.sd_value / mean)));
        const double m = log(mean) - 0.5 * sigma * sigma;
        v = exp(m + h * sigma);
    }
    a.out[i] = v;
}

}  // namespace

// Candidate eigenvalue products and their order: on return the first K entries
// of eig_sorted / idx_sorted hold the K largest products and their linear
// indices (m K + n, or (m K + n) K + k).  r is K x 3 on the device; the
// buffers hold K^ndim entries; sort_tmp of sphk_kl_sort_bytes().
extern "C" size_t sphk_kl_sort_bytes(size_t total)
{
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, (const double*)nullptr, (double*)nullptr,
                                              (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)total);
    return bytes;
}

extern "C" int sphk_kl_order(const double* d_r, int K, int ndim, double* keys_in, double* keys_out, uint32_t* vals_in,
                             uint32_t* vals_out, void* sort_tmp, size_t sort_bytes, cudaStream_t st)
{
    const size_t total = (ndim == 2) ? (size_t)K * K : (size_t)K * K * K;
    const unsigned blocks = (unsigned)((total + 255) / 256);
    if (ndim == 2) k_kl_products<2><<<blocks, 256, 0, st>>>(d_r, K, total, keys_in, vals_in);
    else k_kl_products<3><<<blocks, 256, 0, st>>>(d_r, K, total, keys_in, vals_in);
    size_t bytes = sort_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairsDescending(sort_tmp, bytes, keys_in, keys_out, vals_in, vals_out,
                                                             (int)total, 0, 64, st);
    return e == cudaSuccess ? 0 : 1;
}

extern "C" int sphk_kl_field(int n, int ndim, int K, int no, int type, const double* x_trans, double mean_value,
                             double sd_value, double coe_depth, double soil_max, double water_max, const double* d_xh,
                             const int* d_type, const void* d_terms, const double* d_sqrt_eig, const double* d_xi,
                             double* d_out, cudaStream_t st)
{
    KLFieldArgs a;
    a.n = n; a.ndim = ndim; a.K = K; a.no = no; a.type = type;
    for (int d = 0; d < 3; d++) a.x_trans[d] = x_trans[d];
    a.mean_value = mean_value; a.sd_value = sd_value; a.coe_depth = coe_depth;
    a.soil_max = soil_max; a.water_max = water_max;
    a.xh = d_xh; a.ptype = d_type; a.terms = (const KLTerm*)d_terms; a.sqrt_eig = d_sqrt_eig; a.xi = d_xi;
    a.out = d_out;
    const size_t smem = sizeof(KLTerm) * (size_t)K * ndim + sizeof(double) * 2 * (size_t)K;
    const unsigned blocks = (unsigned)((n + 127) / 128);
    if (ndim == 2) {
        cudaFuncSetAttribute(k_kl_field<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_kl_field<2><<<blocks, 128, smem, st>>>(a);
    } else {
        cudaFuncSetAttribute(k_kl_field<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_kl_field<3><<<blocks, 128, smem, st>>>(a);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

extern "C" size_t sphk_kl_term_bytes(void) { return sizeof(KLTerm); }
