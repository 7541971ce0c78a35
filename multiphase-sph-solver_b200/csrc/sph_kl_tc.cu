// sph_kl_tc.cu -- batched K-L random field synthesis on the tensor cores
// (tcgen05, sm_100a).
//
// For R realisations of one field on one geometry the reference's sum
// (solve_h_2D / solve_h_3D, CPP_17-1_K-L_expansion_non.cpp:486-700)
//     H[r][i] = sum_j sqrt(lambda_j) phi_j(x_i) xi[r][j]
// is the product of the eigenfunction matrix Phi (n x K) with the
// coefficient matrix C (K x R), C[j][r] = sqrt(lambda_j) xi[r][j].  One CTA
// takes 128 particles: its threads evaluate their Phi rows into shared memory
// K_TILE terms at a time, one thread issues tcgen05.mma (kind::tf32, M = 128,
// N = R, K = 8 per instruction) on that tile and the matching C tile, and the
// FP32 accumulator lives in tensor memory (R columns).  TF32 keeps 10 mantissa
// bits, so each operand is split into a TF32-exact high part and the FP32
// remainder, and three products are accumulated:
//     Phi C ~= Phi_hi C_hi + Phi_hi C_lo + Phi_lo C_hi
// (the dropped Phi_lo C_lo is below 2^-20 of each term).  The epilogue reads
// the accumulator with tcgen05.ld and applies the normal / lognormal map and
// the depth trend of the reference, writing out[r * n + i] in FP32.
//
// The eigenfunction arguments w x are formed and reduced modulo 2 pi in FP64
// before the FP32 cos / sin, so the phase error stays at FP32 rounding for
// the large arguments of high-order terms.
//
// Every wait on the MMA completion barrier is bounded (about one second of
// SM clock); on expiry the kernel records SPHGPU_KL_TIMEOUT in *err, waits
// once more (bounded) for its MMAs, releases its tensor memory and returns.
#include <cuda_runtime.h>
#include <cstdint>

#define KL_TILE_M 128
#define KL_K_TILE 40                   // terms per shared-memory tile (5 MMA K-steps of 8)
#define KL_CORE_BYTES 128              // a core matrix: 8 rows x 16 bytes
#define KL_TIMEOUT_CODE 105

namespace {

struct KLTCTerm { double w; float alpha; int use_cos; };

struct KLTCArgs {
    int n, ndim, K, R, no, type;
    double x_trans[3];
    double mean_value, sd_value, coe_depth, soil_max, water_max;
    const double* xh;          // (x, y, z, h) records
    const int* ptype;
    const KLTCTerm* terms;     // K x ndim
    const float* c_hi;         // R x K, K contiguous (K-major B operand)
    const float* c_lo;
    float* out;                // R x n
    int* err;
    long long budget;          // SM clocks one completion wait may take
    int probe;                 // 1: the wait self-test (below), no synthesis
    // the separable form: the distinct 1-D eigenfunctions of each axis
    // (nmode[d] of them, from modes + moff[d]) and, per term and axis, the
    // index of its factor among them (tidx, K x ndim); null: each term's
    // factors are evaluated in the tile loop
    const KLTCTerm* modes;
    int nmode[3], moff[3];
    const unsigned short* tidx;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (row, k) in a K-major, unswizzled canonical layout
// of K_TILE columns: 8-row x 4-element core matrices, adjacent along K at
// LBO = 128 bytes, adjacent along rows at SBO = K_TILE / 4 * 128 bytes
__device__ __forceinline__ uint32_t kmajor_off(int row, int k)
{
    return (uint32_t)((row >> 3) * (KL_K_TILE / 4) * KL_CORE_BYTES + (k >> 2) * KL_CORE_BYTES + (row & 7) * 16 +
                      (k & 3) * 4);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr)
{
    const uint64_t lbo = KL_CORE_BYTES, sbo = (KL_K_TILE / 4) * KL_CORE_BYTES;
    return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | (1ull << 46);   // version 1, no swizzle
}

// x rounded to TF32 (10 explicit mantissa bits, nearest-even), exact in FP32
__device__ __forceinline__ float tf32_hi(float x)
{
    uint32_t u = __float_as_uint(x);
    if ((u & 0x7f800000u) == 0x7f800000u) return x;
    u += 0xfffu + ((u >> 13) & 1u);
    u &= 0xffffe000u;
    return __uint_as_float(u);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long budget)
{
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
        if (clock64() - t0 > budget) return false;
    }
}

__global__ void __launch_bounds__(KL_TILE_M, 1) k_kl_synth(KLTCArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    // layout: A_hi | A_lo | B_hi | B_lo | barrier | tmem base
    const int R = a.R;
    const uint32_t a_bytes = KL_TILE_M * KL_K_TILE * 4;
    const uint32_t b_bytes = (uint32_t)R * KL_K_TILE * 4;
    unsigned char* A_hi = smem;
    unsigned char* A_lo = A_hi + a_bytes;
    unsigned char* B_hi = A_lo + a_bytes;
    unsigned char* B_lo = B_hi + b_bytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(B_lo + b_bytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
    // separable form: each particle's values of the distinct 1-D factors,
    // table[m * 128 + thread], then the factor indices of the K terms
    float* table = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(bar) + 16);
    const int nmodes = a.modes ? a.nmode[0] + a.nmode[1] + a.nmode[2] : 0;
    unsigned short* tix = reinterpret_cast<unsigned short*>(table + (size_t)nmodes * KL_TILE_M);

    const int t = threadIdx.x, warp = t >> 5;
    int ncols = 32;
    while (ncols < R) ncols <<= 1;

    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    const int i = blockIdx.x * KL_TILE_M + t;
    const bool live = i < a.n;
    double xa[3] = {0.0, 0.0, 0.0};
    double yp = 0.0;
    if (live) {
        const double2* rec = reinterpret_cast<const double2*>(a.xh) + 2 * (size_t)i;
        const double2 r0 = rec[0], r1 = rec[1];
        xa[0] = r0.x - a.x_trans[0];
        xa[1] = r0.y - a.x_trans[1];
        xa[2] = r1.x - a.x_trans[2];
        yp = r0.y;
    }
    if (a.modes && !a.probe) {
        // each distinct factor once per particle and axis: alpha cos / sin of
        // w x reduced modulo 2 pi in FP64, the values the tile loop below
        // multiplies (the same operations as the direct form, so the same
        // floats)
        const double two_pi_ = 6.283185307179586, inv_two_pi_ = 0.15915494309189535;
        for (int d = 0; d < a.ndim; d++)
            for (int m = 0; m < a.nmode[d]; m++) {
                float v = 0.f;
                if (live) {
                    const KLTCTerm q = a.modes[a.moff[d] + m];
                    const double arg = q.w * xa[d];
                    const float red = (float)(arg - rint(arg * inv_two_pi_) * two_pi_);
                    v = q.alpha * (q.use_cos ? cosf(red) : sinf(red));
                }
                table[(size_t)(a.moff[d] + m) * KL_TILE_M + t] = v;
            }
        for (int e = t; e < a.K * a.ndim; e += KL_TILE_M) tix[e] = a.tidx[e];
        __syncthreads();
    }
    // instruction descriptor: D F32, A and B TF32, both K-major, N = R, M = 128
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(R >> 3) << 17) |
                           ((uint32_t)(KL_TILE_M >> 4) << 24);
    const double two_pi = 6.283185307179586, inv_two_pi = 0.15915494309189535;
    uint32_t phase = 0;
    bool ok = true;
    const long long budget = a.budget;
    if (a.probe) {
        // the failure path on demand: a wait on the completion barrier before
        // any MMA has been issued, which nothing will signal, must expire
        // within the budget, record the code and leave through the normal
        // teardown (tensor memory released, nothing in flight)
        const bool got = mbar_wait(smem_u32(bar), phase, budget);
        if (__syncthreads_or(!got)) {
            ok = false;
            if (t == 0) atomicCAS(a.err, 0, KL_TIMEOUT_CODE);
        }
    }
    for (int k0 = 0; k0 < a.K && ok && !a.probe; k0 += KL_K_TILE) {
        const int kt = min(KL_K_TILE, a.K - k0);
        // this thread's Phi row for terms k0 .. k0 + kt
        for (int k = 0; k < KL_K_TILE; k++) {
            float phi = 0.f;
            if (live && k < kt) {
                phi = 1.f;
                if (a.modes) {
                    for (int d = 0; d < a.ndim; d++)
                        phi *= table[(size_t)(a.moff[d] + tix[(k0 + k) * a.ndim + d]) * KL_TILE_M + t];
                } else {
                    for (int d = 0; d < a.ndim; d++) {
                        const KLTCTerm q = a.terms[(size_t)(k0 + k) * a.ndim + d];
                        const double arg = q.w * xa[d];
                        const float red = (float)(arg - rint(arg * inv_two_pi) * two_pi);
                        phi *= q.alpha * (q.use_cos ? cosf(red) : sinf(red));
                    }
                }
            }
            const float hi = tf32_hi(phi);
            *reinterpret_cast<float*>(A_hi + kmajor_off(t, k)) = hi;
            *reinterpret_cast<float*>(A_lo + kmajor_off(t, k)) = phi - hi;
        }
        // the coefficient tile: R rows (realisations) x kt terms
        for (int e = t; e < R * KL_K_TILE; e += KL_TILE_M) {
            const int r = e / KL_K_TILE, k = e % KL_K_TILE;
            float hi = 0.f, lo = 0.f;
            if (k < kt) {
                hi = a.c_hi[(size_t)r * a.K + k0 + k];
                lo = a.c_lo[(size_t)r * a.K + k0 + k];
            }
            *reinterpret_cast<float*>(B_hi + kmajor_off(r, k)) = hi;
            *reinterpret_cast<float*>(B_lo + kmajor_off(r, k)) = lo;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t ah = smem_u32(A_hi), al = smem_u32(A_lo), bh = smem_u32(B_hi), bl = smem_u32(B_lo);
            const int nks = (kt + 7) / 8;
            for (int s = 0; s < nks; s++) {
                const uint32_t off = (uint32_t)s * 2 * KL_CORE_BYTES;   // 8 terms = 2 core matrices along K
                const uint64_t d_ah = smem_desc(ah + off), d_al = smem_desc(al + off);
                const uint64_t d_bh = smem_desc(bh + off), d_bl = smem_desc(bl + off);
                const uint32_t acc0 = (k0 == 0 && s == 0) ? 0u : 1u;
                asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                             ::"r"(tmem), "l"(d_ah), "l"(d_bh), "r"(idesc), "r"(acc0));
                asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                             ::"r"(tmem), "l"(d_ah), "l"(d_bl), "r"(idesc), "r"(1u));
                asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                             ::"r"(tmem), "l"(d_al), "l"(d_bh), "r"(idesc), "r"(1u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(bar)) : "memory");
        }
        // the tile's MMAs must finish before its shared memory is refilled;
        // the outcome is made uniform over the CTA (the epilogue's TMEM loads
        // are warp-collective)
        const bool got = mbar_wait(smem_u32(bar), phase, budget);
        if (__syncthreads_or(!got)) {
            ok = false;
            if (t == 0) atomicCAS(a.err, 0, KL_TIMEOUT_CODE);
            if (!got) mbar_wait(smem_u32(bar), phase, budget);
            __syncthreads();
        }
        phase ^= 1u;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok && !a.probe) {
        // epilogue: warp w holds accumulator lanes 32 w .. 32 w + 31 (particle t)
        const int ptype = live ? a.ptype[i] : -1;
        const bool soil_field = a.no >= 0 && a.no <= 3;
        const bool writes = live && ((soil_field && ptype == 2) || (!soil_field && ptype == 1));
        double mean = 0.0, sigma = 0.0;
        if (writes) {
            mean = a.mean_value + ((ptype == 2 ? a.soil_max : a.water_max) - yp) * a.coe_depth;
            if (a.type == 1) {
                sigma = a.sd_value;
            } else {
                sigma = sqrt(log(1.0 + (a.sd_value / mean) * (a.sd_value / mean)));
                mean = log(mean) - 0.5 * sigma * sigma;
            }
        }
        for (int c0 = 0; c0 < R; c0 += 8) {
            uint32_t v[8];
            const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7])
                         : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (live) {
                for (int q = 0; q < 8 && c0 + q < R; q++) {
                    const double h = (double)__uint_as_float(v[q]);
                    float o = __int_as_float(0x7fc00000);
                    if (writes) o = (float)((a.type == 1) ? mean + h * sigma : exp(mean + h * sigma));
                    a.out[(size_t)(c0 + q) * a.n + i] = o;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// C = sqrt(lambda) xi split into TF32-exact high and FP32 remainder parts
__global__ void k_kl_coef(int K, int R, const double* sqrt_eig, const double* xi, float* c_hi, float* c_lo)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= K * R) return;
    const int j = e % K;
    const float c = (float)(sqrt_eig[j] * xi[e]);
    const float hi = tf32_hi(c);
    c_hi[e] = hi;
    c_lo[e] = c - hi;
}

}  // namespace

extern "C" size_t sphk_kl_tc_smem_bytes(int R)
{
    return (size_t)2 * KL_TILE_M * KL_K_TILE * 4 + (size_t)2 * R * KL_K_TILE * 4 + 16;
}

// shared memory of the separable form: the above, the factor table of
// nmodes factors per particle and the K x ndim factor indices
static size_t kl_tc_smem_table(int R, int nmodes, int K, int ndim)
{
    return sphk_kl_tc_smem_bytes(R) + (size_t)nmodes * KL_TILE_M * 4 + ((size_t)K * ndim * 2 + 15) / 16 * 16;
}

// the largest dynamic shared memory a CTA of this kernel may take
#define KL_SMEM_MAX (227 * 1024)

extern "C" size_t sphk_kl_tc_term_bytes(void) { return sizeof(KLTCTerm); }

// R: multiple of 16 in [16, 256]; K: multiple of 8.  d_terms K x ndim
// KLTCTerm, d_sqrt_eig K, d_xi R x K (FP64), scratch c_hi / c_lo R x K floats.
extern "C" int sphk_kl_synthesize(int n, int ndim, int K, int R, int no, int type, const double* x_trans,
                                  double mean_value, double sd_value, double coe_depth, double soil_max,
                                  double water_max, const double* d_xh, const int* d_type, const void* d_terms,
                                  const double* d_sqrt_eig, const double* d_xi, float* c_hi, float* c_lo,
                                  float* d_out, int* d_err, cudaStream_t st, const void* d_modes,
                                  const int* nmode, const unsigned short* d_tidx)
{
    if (R < 16 || R > 256 || R % 16 != 0 || K < 8 || K % 8 != 0) return 1;
    k_kl_coef<<<(K * R + 255) / 256, 256, 0, st>>>(K, R, d_sqrt_eig, d_xi, c_hi, c_lo);
    KLTCArgs a;
    a.n = n; a.ndim = ndim; a.K = K; a.R = R; a.no = no; a.type = type;
    for (int d = 0; d < 3; d++) a.x_trans[d] = x_trans[d];
    a.mean_value = mean_value; a.sd_value = sd_value; a.coe_depth = coe_depth;
    a.soil_max = soil_max; a.water_max = water_max;
    a.xh = d_xh; a.ptype = d_type; a.terms = (const KLTCTerm*)d_terms; a.c_hi = c_hi; a.c_lo = c_lo;
    a.out = d_out; a.err = d_err;
    a.budget = 2000000000ll;     // SM clocks, about one second
    a.probe = 0;
    a.modes = nullptr;
    a.tidx = nullptr;
    a.nmode[0] = a.nmode[1] = a.nmode[2] = 0;
    a.moff[0] = a.moff[1] = a.moff[2] = 0;
    size_t smem = sphk_kl_tc_smem_bytes(R);
    if (d_modes && d_tidx && nmode) {
        const int total = nmode[0] + nmode[1] + nmode[2];
        const size_t with = kl_tc_smem_table(R, total, K, ndim);
        if (with <= KL_SMEM_MAX) {       // else the factors are evaluated per term
            a.modes = (const KLTCTerm*)d_modes;
            a.tidx = d_tidx;
            for (int d = 0; d < 3; d++) a.nmode[d] = nmode[d];
            a.moff[1] = nmode[0];
            a.moff[2] = nmode[0] + nmode[1];
            smem = with;
        }
    }
    if (cudaFuncSetAttribute(k_kl_synth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 1;
    k_kl_synth<<<(n + KL_TILE_M - 1) / KL_TILE_M, KL_TILE_M, smem, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// One CTA of the synthesis kernel in its wait self-test: it allocates its
// tensor memory, waits `budget` SM clocks on a completion barrier nothing
// signals, records the timeout code in *d_err and releases the memory.
extern "C" int sphk_kl_wait_probe(long long budget, int* d_err, cudaStream_t st)
{
    KLTCArgs a = {};
    a.n = 0; a.ndim = 2; a.K = 8; a.R = 16;
    a.modes = nullptr;
    a.tidx = nullptr;
    a.err = d_err;
    a.budget = budget;
    a.probe = 1;
    const size_t smem = sphk_kl_tc_smem_bytes(a.R);
    if (cudaFuncSetAttribute(k_kl_synth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 1;
    k_kl_synth<<<1, KL_TILE_M, smem, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
