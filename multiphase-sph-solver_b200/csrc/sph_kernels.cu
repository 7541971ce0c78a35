// sph_kernels.cu -- the per-step particle loop of the multi-phase SPH solver
// as sm_100a kernels (FP64 drop-in form).
//
// One time step (the body of SPH_Calculation's main loop,
// CPP_1-SPHLoops.cpp:523-753), one kernel per level of the neighbour-data
// dependency chain:
//
//   k_cellkey      parttocell: cell key per particle            (CPP_3-NNPS.cpp:175-257)
//   radix sort     Binary_Sort's order: cell ascending, index descending
//   k_cellreset    cell_info reset                              (CPP_3-NNPS.cpp:196-201)
//   k_cellrange    cell_info start/end (:621-629) + the cell-sorted copy of positions
//   k_nnps         partisearching: stencil scan in cell-sorted order, FP32 prefilter
//   k_nnps_resolve FP64 decisions of the undecided candidates, neighbour list, slot masks
//   k_density      fluid porosity + continuity                  (CPP_6-density.cpp:25-165)
//   k_shepard_eos  Shepard filter (Jacobi) + local EOS          (CPP_6-density.cpp:168-188, CPP_7-1-eos_CR.cpp:22-43)
//   k_strain       velocity gradient, strain rate and spin, gathered pore pressures and
//                  wall stresses, free-surface colour          (CPP_7-1-strain.cpp:20-220, CPP_7-1-eos_CR.cpp:46-177)
//   k_stress       permeability, constitutive update, free-surface correction,
//                  principal stresses (per particle)           (CPP_7-2-constitutive.cpp, CPP_8-1-consfactor.cpp)
//   k_accel        momentum (fluid / soil / structure), artificial viscosity,
//                  wall stress, Darcy drag, geostatic damping, velocity update
//   k_xsph_update  XSPH, wall velocity correction, domain check, position update
//
// Every pair sum is gathered by the particle that owns it, in the reference's
// neighbour order, with no atomics: results are deterministic and, with
// -fmad=false, equal to the reference's FP64 arithmetic.  Kernel values are
// computed once per pair by the neighbour search and stored with the list,
// as partisearching stores Par_Cell::wij.
// All kernels return immediately once an error code is set, so a failing step
// leaves the state as the reference leaves it when it returns the code.
//
// The file is compiled twice.  Built plainly it is the FP64 drop-in form:
// -fmad=false, every pair sum in the reference's FP64 order.  Built with
// SPH_BULK32 defined (sph_kernels_bulk32.cu) it is the FP32-bulk form: the
// pair arithmetic of the neighbour passes (kernel values and gradients, pair
// terms, their sums) runs in FP32 with Kahan-compensated sums, while
// positions, velocities, densities, stresses, their time integration and the
// constitutive update stay FP64; pair differences of positions and velocities
// are taken in FP64 before they are rounded.  The neighbour search is shared
// by both forms and lives in the FP64 build only.
#include <cub/cub.cuh>
#include <climits>
#include "sph_device.cuh"
#include "sph_constitutive.cuh"

#ifdef SPH_BULK32
typedef float real;            // pair arithmetic of the neighbour passes
#define SPH_NS sph_bulk32
#define SPHK_ENTRY(name) name##_bulk32
#else
typedef double real;
#define SPH_NS sph_fp64
#define SPHK_ENTRY(name) name
#endif

#define IDX (blockIdx.x * blockDim.x + threadIdx.x)

namespace SPH_NS {

// minimum resident 128-thread blocks per SM requested from the register
// allocator for the neighbour-loop kernels (an occupancy / spill trade-off)
// (4 measured fastest on B200 for the 3-D soil column: 49.9 ms vs 55.0 ms per
// step at 1, 2 or 3)
#ifndef SPH_MINB
#define SPH_MINB 4
#endif
// the constitutive pass keeps a dense 6x6 tangent per thread: 2 blocks of
// 128 threads per SM leave it 222 registers and no spills
#ifndef SPH_MINB_STRESS
#define SPH_MINB_STRESS 2
#endif
// the momentum pass: its neighbour loops (k_accel_b) at 7 blocks per SM
// (72 registers, a few spills: faster than 8, 6 or 5), its per-particle tail
// (k_accel_b_tail) at 6 (faster than 5 and 4)
#ifndef SPH_MINB_ACCB
#define SPH_MINB_ACCB 6
#endif
#ifndef SPH_MINB_ACCB1
#define SPH_MINB_ACCB1 7
#endif
#ifndef SPH_MINB_ACCB2
#define SPH_MINB_ACCB2 7
#endif
#ifndef SPH_MINB_PAIRW
#define SPH_MINB_PAIRW SPH_MINB
#endif
// the same trade for the strain pass (6 blocks: 80 registers, a few spills),
// the density pass (6: 72, none; 7 no faster) and XSPH (8: 64); the
// stress-divergence pass ran slower at 5 blocks (2.2 -> 2.5 ms) and keeps 4
#ifndef SPH_MINB_STRAIN
#define SPH_MINB_STRAIN 6
#endif
#ifndef SPH_MINB_ACCA
#define SPH_MINB_ACCA 4
#endif
#ifndef SPH_MINB_DENS
#define SPH_MINB_DENS 6
#endif
#ifndef SPH_MINB_XSPH
#define SPH_MINB_XSPH 8
#endif

__device__ __forceinline__ void raise_err(int* err, int code) { atomicCAS(err, 0, code); }

__device__ __forceinline__ bool same_bits(double a, double b)
{
    return __double_as_longlong(a) == __double_as_longlong(b);
}

// x86-64 cvttsd2si semantics for the reference's (int) casts of FP64 cell
// coordinates: NaN and out-of-range values become INT_MIN.
__device__ __forceinline__ int to_int_x86(double v)
{
    return (v >= -2147483648.0 && v < 2147483648.0) ? (int)v : INT_MIN;
}

// cell_link slot p of cell c (celllist_ini2, CPP_3-NNPS.cpp:124-171) on the
// grid g, in the context's cell ids (0: no cell)
template <int ND>
__device__ __forceinline__ int cell_link(const CellGrid& g, int c, int slot)
{
    int v;
    const int lc = c - g.base;
    if (ND == 2) {
        int ky = slot / 3 + 1, kx = slot % 3 + 1;
        v = (kx - 2) * g.cym + ky - 2 + lc;
    } else {
        int kz = slot / 9 + 1, kx = (slot / 3) % 3 + 1, ky = slot % 3 + 1;
        v = (ky - 2) * g.cxm * g.czm + (kx - 2) * g.czm + kz - 2 + lc;
    }
    return (v <= 0 || v > g.ctotal) ? 0 : v + g.base;
}

__device__ __forceinline__ int nbr_count(const Dev& d, int i)
{
    int c = d.s.nnb[i];
    return c > SPH_NB_CAP ? SPH_NB_CAP : c;
}

// The slot mask of particles of type t in particle i's list (word 0: slots
// 0-63, word 1: slots 64-98); types 0-4 only (type 7 has none)
struct SlotMask {
    unsigned long long lo, hi;
    __device__ __forceinline__ SlotMask operator|(const SlotMask& o) const { return SlotMask{lo | o.lo, hi | o.hi}; }
    __device__ __forceinline__ bool any() const { return (lo | hi) != 0ull; }
    __device__ __forceinline__ bool has(int s) const { return ((s < 64 ? lo >> s : hi >> (s - 64)) & 1ull) != 0; }
};
__device__ __forceinline__ SlotMask type_mask(const Dev& d, int i, int t)
{
    if (t < 0 || t > 4) return SlotMask{0ull, 0ull};
    const size_t N = (size_t)d.p.N;
    return SlotMask{d.s.nbm[(2 * t) * N + i], d.s.nbm[(2 * t + 1) * N + i]};
}

// The slots of particle i's list whose bits are set in a mask (from nbm:
// one type's slots or a union), in slot order, with the next slot's particle index
// loaded one slot ahead.  Lanes of a warp then take their k-th slot of the
// class together, whatever the slots of other classes between them, so the
// pass body runs with its lanes in step instead of idling on other classes.
struct MaskIter {
    const int* nbr;
    size_t N;
    int i, jn, sn;
    unsigned long long m0, m1;
    __device__ __forceinline__ int pop()
    {
        if (m0) { const int s = __ffsll(m0) - 1; m0 &= m0 - 1; return s; }
        if (m1) { const int s = 63 + __ffsll(m1); m1 &= m1 - 1; return s; }
        return -1;
    }
    __device__ __forceinline__ MaskIter(const Dev& d, int i_, SlotMask m)
        : nbr(d.s.nbr), N((size_t)d.p.N), i(i_), m0(m.lo), m1(m.hi)
    {
        sn = pop();
        jn = (sn >= 0) ? nbr[(size_t)sn * N + i] : 0;
    }
    // the next slot s and its particle j; false when the mask is exhausted
    __device__ __forceinline__ bool next(int& s, int& j)
    {
        if (sn < 0) return false;
        s = sn;
        j = jn;
        sn = pop();
        if (sn >= 0) jn = nbr[(size_t)sn * N + i];
        return true;
    }
};

// The list slots of particle i in order, each slot's particle index loaded
// two slots ahead and its type one slot ahead.  A neighbour pass is a chain of
// dependent loads per slot (list -> type -> the neighbour's fields); issuing
// the first two for later slots while the current slot's gathers are in
// flight leaves one load latency per slot instead of three.
struct NbrIter {
    const int* nbr;
    const int* type;
    size_t N;
    int i, nn, s, j1, j2, t1;
    __device__ __forceinline__ NbrIter(const Dev& d, int i_, int nn_)
        : nbr(d.s.nbr), type(d.s.type), N((size_t)d.p.N), i(i_), nn(nn_), s(0)
    {
        j1 = (nn > 0) ? nbr[i] : 0;
        j2 = (nn > 1) ? nbr[N + i] : 0;
        t1 = (nn > 0) ? type[j1] : 0;
    }
    // slot s's particle and type; issues the loads of the slots after it
    __device__ __forceinline__ void next(int& j, int& tj)
    {
        j = j1;
        tj = t1;
        j1 = j2;
        t1 = (s + 1 < nn) ? type[j1] : 0;
        j2 = (s + 2 < nn) ? nbr[(size_t)(s + 2) * N + i] : 0;
        s++;
    }
};

// ---------------------------------------------------------------------------
#ifndef SPH_BULK32
template <int ND>
__global__ void k_cellkey(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    const Pos q = load_pos(d.s.xh, i);
    const double xp[3] = {q.x, q.y, q.z};
    const CellGrid g = cell_grid(d, i);
    const double xmin[3] = {g.xmin, g.ymin, g.zmin};
    const double dr = 2.0 * d.p.dr;
    int nx_t[3] = {0, 0, 0};
    for (int j = 0; j < ND; j++) {
        double nx = fabs(xp[j] - xmin[j]) / dr + 2.0;
        nx_t[j] = to_int_x86(nx);
        if (nx_t[j] < 2) nx_t[j] = 2;
    }
    unsigned key;
    if (ND == 2)
        key = (unsigned)g.cym * (unsigned)(nx_t[0] - 1) + (unsigned)nx_t[1];
    else
        key = (unsigned)g.cxm * (unsigned)g.czm * (unsigned)(nx_t[1] - 1) +
              (unsigned)g.czm * (unsigned)(nx_t[0] - 1) + (unsigned)nx_t[2];
    int c = (int)key;
    if (!(c > 0 && c <= g.ctotal)) {
        raise_err(d.s.err, SPH_ERR_CELL);
        c = 0;
    }
    c += g.base;
    d.s.cell[i] = c;
    // placed by the particle's index in the caller's order, reversed: the
    // stable radix sort then keeps equal keys in descending caller's index,
    // the order Binary_Sort's merge produces, in whatever order the state is
    // held
    const int o = d.s.i2o[i];
    d.s.key_in[N - 1 - o] = (uint32_t)c;
    d.s.val_in[N - 1 - o] = i;
}

// rainpro (CPP_15-1-rain.cpp:43-85), at the top of the steps with
// (l - inip) > 0 and (l - inip) % lp == 0: the next row of waiting rain
// particles -- from index N - nrain on (in the caller's order, mapped to
// where the state holds them) while each next particle's vertical
// coordinate stays within 0.1 dr of the one before it -- becomes water:
// lowered to 0.95 of its height, falling at vrain, with its density, mass and
// pressure set as the reference sets them.  One block: the row's end is the
// first break found over windows of the block's width, then each thread
// releases its share of the row.
template <int ND>
__global__ void __launch_bounds__(256) k_rain(Dev d)
{
    if (*d.s.err) return;
    const int rel = *d.s.step - d.p.inip;
    if (!(rel > 0 && d.p.rain_lp > 0 && rel % d.p.rain_lp == 0)) return;
    const int nrain = *d.s.nrain;
    if (nrain <= 0) return;
    const int N = d.p.N, k0 = N - nrain;
    const double dr = d.p.dr;
    __shared__ int s_end;
    if (threadIdx.x == 0) s_end = N - 1;
    __syncthreads();
    for (int base = k0; base < N - 1; base += blockDim.x) {
        const int e = base + threadIdx.x;
        if (e < N - 1) {
            const Pos a = load_pos(d.s.xh, d.s.o2i[e]), b = load_pos(d.s.xh, d.s.o2i[e + 1]);
            const double za = (ND == 2) ? a.y : a.z, zb = (ND == 2) ? b.y : b.z;
            if (!(fabs(zb - za) < 0.1 * dr)) atomicMin(&s_end, e);
        }
        __syncthreads();
        const bool found = s_end < N - 1 && s_end < base + (int)blockDim.x;
        __syncthreads();
        if (found) break;
    }
    const int end = s_end;
    const double g = (ND == 2) ? d.p.gy : d.p.gz;
    for (int ko = k0 + threadIdx.x; ko <= end; ko += blockDim.x) {
        const int k = d.s.o2i[ko];
        Pos p = load_pos(d.s.xh, k);
        if (ND == 2) p.y = 0.95 * p.y;
        else p.z = 0.95 * p.z;
        p.h = dr;
        store_pos(d.s.xh, k, p);
        d.s.type[k] = 1;
        d.s.matype[k] = 0;
        d.s.etype[k] = 7;
        const double rhop = d.s.f_por[k] * d.s.f_dens[k];
        d.s.rhop[k] = rhop;
        d.s.mass[k] = (ND == 2) ? rhop * p.h * p.h : rhop * p.h * p.h * p.h;
        for (int c = 0; c < 3; c++) {
            d.s.vxp[c * N + k] = 0.0;
            d.s.vx[c * N + k] = 0.0;
        }
        d.s.vxp[(ND - 1) * N + k] = d.p.rain_vrain;
        d.s.prep[k] = rhop * dr * (-g) * d.p.rain_press;
        d.s.satu[k] = 0.99;
    }
    if (threadIdx.x == 0) *d.s.nrain = nrain - (end - k0 + 1);
}

__global__ void k_cellreset(Dev d)
{
    const int c = IDX;
    if (c >= d.p.ctotal || *d.s.err) return;
    if (d.p.ninst > 0) {
        // each instance's own cell ctotal keeps its range, as in one system
        int lo = 0, hi = d.p.ninst - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (d.s.inst[mid].cell_base <= c) lo = mid;
            else hi = mid - 1;
        }
        if (c - d.s.inst[lo].cell_base == d.s.inst[lo].ctotal) return;
    }
    d.s.cstart[c] = 10000000;
    d.s.cend[c] = -10000000;
}

// cell_info start/end, and the positions in cell-sorted order.  Cell ctotal
// is never reset by the reference (its reset loop stops at ctotal - 1), so its
// range accumulates across steps.
__global__ void k_cellrange(Dev d)
{
    const int q = IDX, N = d.p.N;
    if (q >= N || *d.s.err) return;
    const uint32_t c = d.s.key_out[q];
    const bool first = (q == 0) || d.s.key_out[q - 1] != c;
    const bool last = (q == N - 1) || d.s.key_out[q + 1] != c;
    const int pid = d.s.pid_sorted[q];
    const CellGrid g = cell_grid(d, pid);
    if ((int)c - g.base == g.ctotal) {
        if (first) atomicMin(&d.s.cstart[c], q);
        if (last) atomicMax(&d.s.cend[c], q);
    } else {
        if (first) d.s.cstart[c] = q;
        if (last) d.s.cend[c] = q;
    }
    d.s.sortpos[pid] = q;
    const int t = d.s.type[pid];
    d.s.pts[q] = (pid << 3) | ((t >= 0 && t <= 4) ? t : 7);
    const Pos r = load_pos(d.s.xh, pid);
    store_pos(d.s.xs, q, r);
    reinterpret_cast<float4*>(d.s.xsf)[q] =
        make_float4((float)(r.x - g.xmin), (float)(r.y - g.ymin), (float)(r.z - g.zmin), (float)r.h);
}

// partisearching (CPP_3-NNPS.cpp:265-374): neighbours of i in stencil order,
// descending index inside each cell; inclusion dst <= h_i + h_j decided as the
// reference decides it (sqrt of the FP64 sum of squares).
//
// Each candidate is first tested in FP32 on the (x - xmin, y - ymin, z - zmin,
// h) records, against a margin M that bounds every rounding between the FP32
// squared distance d2f and the exact one: the coordinates' rounding to FP32
// (at most 2^-24 |coordinate|, and |x_j - xmin| <= |x_i - xmin| + |x_i - x_j|),
// the subtraction, squares and sum, and the rounding of T = h_i + h_j and T^2.
// With F_i the particle's largest |coordinate - min| and e = 2.2 u (F_i + 2 T),
// u = 2^-24, every candidate with d2f <= 4 T^2 has |d2f - d2| <= nd e (4 T + e)
// + 12.4 u T^2; M adds 32 u T^2 on top of that.  Candidates with d2f > 4 T^2
// are outside whenever h_i > 10 u F_i (the error then grows more slowly than
// d2f - T^2); the test requires h_i > 64 u F_i and otherwise sends every
// candidate to the FP64 path.  Only candidates within M of T^2 take the FP64
// path, where the sqrt is evaluated only within 1e-10 of the squared radius,
// so the decisions are those of the reference.
// The per-type slot masks of one particle's list (nbm), built as the list
// is written: bit s of word (t, s / 64) set when slot s holds type t (0-4)
struct TypeMasks {
    unsigned long long m[5][2];
    __device__ __forceinline__ TypeMasks()
    {
#pragma unroll
        for (int t = 0; t < 5; t++) m[t][0] = m[t][1] = 0ull;
    }
    __device__ __forceinline__ void add(int t, int s)
    {
        const unsigned long long lo = (s < 64) ? (1ull << s) : 0ull, hi = (s < 64) ? 0ull : (1ull << (s - 64));
#pragma unroll
        for (int k = 0; k < 5; k++)
            if (t == k) {
                m[k][0] |= lo;
                m[k][1] |= hi;
            }
    }
    __device__ __forceinline__ void store(const Dev& d, int i) const
    {
        const size_t N = (size_t)d.p.N;
#pragma unroll
        for (int k = 0; k < 5; k++) {
            d.s.nbm[(2 * k) * N + i] = m[k][0];
            d.s.nbm[(2 * k + 1) * N + i] = m[k][1];
        }
    }
};

// The FP64 inclusion test of one candidate, as partisearching decides it:
// sqrt of the FP64 sum of squares against h_i + h_j, the sqrt evaluated only
// within 1e-10 of the squared radius (outside that band the comparison of the
// squares gives the same answer).
template <int ND>
__device__ __forceinline__ bool nnps_in_fp64(const double xi[3], double hi, const Pos& pj)
{
    const double xj[3] = {pj.x, pj.y, pj.z};
    double d2 = 0.0;
    for (int k = 0; k < ND; k++) d2 = d2 + (xi[k] - xj[k]) * (xi[k] - xj[k]);
    const double ra = (hi + pj.h) / 2;
    const double T = 2 * ra, T2 = T * T;
    if (d2 < T2 * (1.0 - 1.0e-10)) return true;
    if (d2 > T2 * (1.0 + 1.0e-10)) return false;
    return sqrt(d2) <= T;
}

// FP32 prefilter of the candidates of one particle: its (x - xmin, y - ymin,
// z - zmin, h) in FP32, the margin terms, and the decision bounds lo / hi of a
// candidate with the same h (the usual case), so that such a candidate costs
// its squared distance and two comparisons.  The squared distance is summed
// with fused multiply-adds: one rounding per term instead of two, inside the
// margin derived for separate roundings.
struct Prefilter {
    float fx, fy, fz, fh, ce, ct, lo0, hi0;
};

template <int ND>
__device__ __forceinline__ void prefilter_bounds(const Prefilter& P, float hj, float* lo, float* hi)
{
    constexpr float U = 5.9604645e-8f;     // 2^-24
    const float Tf = P.fh + hj, T2f = Tf * Tf;
    const float e = P.ce + 4.4f * U * Tf;
    const float M = ND * e * (4.f * Tf + e) + P.ct * T2f;
    *lo = T2f - M;
    *hi = T2f + M;
}

template <int ND>
__device__ __forceinline__ Prefilter make_prefilter(float fx, float fy, float fz, float fh, float ce, float ct)
{
    Prefilter P{fx, fy, fz, fh, ce, ct, 0.f, 0.f};
    prefilter_bounds<ND>(P, fh, &P.lo0, &P.hi0);
    return P;
}

// verdict of one candidate: 1 inside, 0 outside, -1 undecided (within the
// rounding margin of the radius).  A candidate beyond twice the radius is
// outside; hi < 4 T^2, so the bounds test covers that case too.
template <int ND>
__device__ __forceinline__ int nnps_prefilter(const Prefilter& P, float4 fj)
{
    float t = P.fx - fj.x;
    float d2f = t * t;
    t = P.fy - fj.y;
    d2f = __fmaf_rn(t, t, d2f);
    if (ND == 3) {
        t = P.fz - fj.z;
        d2f = __fmaf_rn(t, t, d2f);
    }
    float lo = P.lo0, hi = P.hi0;
    if (fj.w != P.fh) {
        const float Tf = P.fh + fj.w;
        if (d2f > 4.f * (Tf * Tf)) return 0;
        prefilter_bounds<ND>(P, fj.w, &lo, &hi);
    }
    if (d2f < lo) return 1;
    if (d2f > hi) return 0;
    return -1;
}

// partisearching with every candidate decided in FP64 as soon as it is met
// (used when the FP32 prefilter does not apply to the particle, or when its
// provisional list below overflows); returns the neighbour count
template <int ND>
__device__ __forceinline__ int nnps_direct(const Dev& d, int i, int nc, const Pos& pi, bool fast, const Prefilter& P)
{
    const int N = d.p.N;
    constexpr int nst = (ND == 2) ? 9 : 27;
    const double xi[3] = {pi.x, pi.y, pi.z};
    const float4* xsf = reinterpret_cast<const float4*>(d.s.xsf);
    const CellGrid g = cell_grid(d, i);
    int cnt = 0;
    for (int nj = 0; nj < nst; nj++) {
        const int nl = cell_link<ND>(g, nc, nj);
        if (nl <= 0) continue;
        const int start = d.s.cstart[nl], end = d.s.cend[nl];
        for (int q = start; q <= end; q++) {
            int v = fast ? nnps_prefilter<ND>(P, xsf[q]) : -1;
            if (v < 0) v = nnps_in_fp64<ND>(xi, pi.h, load_pos(d.s.xs, q)) ? 1 : 0;
            if (v) {
                const int j = d.s.pid_sorted[q];
                if (i != j) {
                    cnt++;
                    if (cnt <= SPH_NB_CAP) d.s.nbr[(size_t)(cnt - 1) * N + i] = j;
                    else raise_err(d.s.err, SPH_ERR_NEIGH);
                }
            }
        }
    }
    return cnt;
}

// partisearching (CPP_3-NNPS.cpp:265-374): neighbours of i in stencil order,
// descending index inside each cell; inclusion dst <= h_i + h_j decided as the
// reference decides it (sqrt of the FP64 sum of squares).
//
// Each candidate is first tested in FP32 on the (x - xmin, y - ymin, z - zmin,
// h) records, against a margin M that bounds every rounding between the FP32
// squared distance d2f and the exact one: the coordinates' rounding to FP32
// (at most 2^-24 |coordinate|, and |x_j - xmin| <= |x_i - xmin| + |x_i - x_j|),
// the subtraction, squares and sum, and the rounding of T = h_i + h_j and T^2.
// With F_i the particle's largest |coordinate - min| and e = 2.2 u (F_i + 2 T),
// u = 2^-24, every candidate with d2f <= 4 T^2 has |d2f - d2| <= nd e (4 T + e)
// + 12.4 u T^2; M adds 32 u T^2 on top of that.  Candidates with d2f > 4 T^2
// are outside whenever h_i > 10 u F_i (the error then grows more slowly than
// d2f - T^2); the test requires h_i > 64 u F_i and otherwise takes every
// candidate to the FP64 test.
//
// Two passes.  The scan (k_nnps) runs one thread per cell-sorted position,
// so the lanes of a warp belong to one or two cells, walk the same stencil
// cells and load the same candidate records (one broadcast per load instead
// of a line per lane).  It stores, in candidate order, the index-and-type
// word w of each candidate inside (w) or undecided (~w) into the provisional
// list of its own sorted position, nbrs[s * N + q], which the lanes of a warp
// fill row by row.  The resolve pass (k_nnps_resolve) runs one thread per
// particle in the caller's order: it reads its provisional list, decides the
// undecided candidates in FP64, and writes the list nbr[s * N + i] and the
// per-type slot masks.  The order, and so the
// list, is the one a single pass in candidate order gives.  A provisional list
// longer than the capacity (possible only when undecided candidates or the
// particle itself push it over), and a particle the FP32 test does not apply
// to, are searched again by the direct form, which also raises the
// reference's error for a true overflow.
template <int ND>
__global__ void __launch_bounds__(128, SPH_MINB) k_nnps(Dev d)
{
    const int q = IDX, N = d.p.N;
    if (q >= N || *d.s.err) return;
    int np = 0;   // provisional entries
    const int pid = d.s.pid_sorted[q];
    if (d.s.type[pid] != 7) {
        constexpr int nst = (ND == 2) ? 9 : 27;
        constexpr float U = 5.9604645e-8f;     // 2^-24
        const float4* xsf = reinterpret_cast<const float4*>(d.s.xsf);
        const int nc = (int)d.s.key_out[q];
        const float4 fi = xsf[q];              // the particle's own FP32 record
        const float fz = (ND == 3) ? fi.z : 0.f;
        float Fi = fmaxf(fabsf(fi.x), fabsf(fi.y));
        if (ND == 3) Fi = fmaxf(Fi, fabsf(fz));
        if (!(fi.w > 64.f * U * Fi)) {
            np = -1;
        } else {
            const Prefilter P = make_prefilter<ND>(fi.x, fi.y, fz, fi.w, 2.2f * U * Fi, 32.f * U);
            const CellGrid g = cell_grid(d, pid);
            int* row = d.s.nbrs + q;
            for (int nj = 0; nj < nst; nj++) {
                const int nl = cell_link<ND>(g, nc, nj);
                if (nl <= 0) continue;
                const int start = d.s.cstart[nl], end = d.s.cend[nl];
                for (int c = start; c <= end; c++) {
                    const float4 fc = xsf[c];
                    const int w = d.s.pts[c];
                    const int v = nnps_prefilter<ND>(P, fc);
                    if (v != 0) {
                        if (np < SPH_NB_CAP) row[(size_t)np * N] = (v > 0) ? w : ~w;
                        np++;
                    }
                }
            }
        }
    }
    d.s.nps[q] = np;
}

// The resolve pass of the search (see k_nnps), one thread per particle, with
// the per-type slot masks of the list written beside it.
template <int ND>
__global__ void __launch_bounds__(128, SPH_MINB) k_nnps_resolve(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    int cnt = 0;
    TypeMasks tm;
    if (d.s.type[i] != 7) {
        const int q0 = d.s.sortpos[i];
        const int np = d.s.nps[q0];
        const Pos pi = load_pos(d.s.xh, i);
        if (np < 0 || np > SPH_NB_CAP) {
            constexpr float U = 5.9604645e-8f;     // 2^-24
            const float4 fi = reinterpret_cast<const float4*>(d.s.xsf)[q0];
            const float fz = (ND == 3) ? fi.z : 0.f;
            float Fi = fmaxf(fabsf(fi.x), fabsf(fi.y));
            if (ND == 3) Fi = fmaxf(Fi, fabsf(fz));
            const Prefilter P = make_prefilter<ND>(fi.x, fi.y, fz, fi.w, 2.2f * U * Fi, 32.f * U);
            cnt = nnps_direct<ND>(d, i, d.s.cell[i], pi, np >= 0, P);
            const int nn = cnt < SPH_NB_CAP ? cnt : SPH_NB_CAP;
            for (int s = 0; s < nn; s++) tm.add(d.s.type[d.s.nbr[(size_t)s * N + i]], s);
        } else {
            const double xi[3] = {pi.x, pi.y, pi.z};
            const int* row = d.s.nbrs + q0;
            // provisional entries two slots ahead
            int v1 = (np > 0) ? row[0] : 0, v2 = (np > 1) ? row[N] : 0;
            for (int s = 0; s < np; s++) {
                const int v = v1;
                v1 = v2;
                if (s + 2 < np) v2 = row[(size_t)(s + 2) * N];
                const int w = (v < 0) ? ~v : v, j = w >> 3;
                const bool in = (v >= 0) || nnps_in_fp64<ND>(xi, pi.h, load_pos(d.s.xh, j));
                if (in && j != i) {
                    d.s.nbr[(size_t)cnt * N + i] = j;
                    tm.add(w & 7, cnt);
                    cnt++;
                }
            }
        }
    }
    d.s.nnb[i] = cnt;
    tm.store(d, i);
}

// The pair records of every list slot, as partisearching stores wij with the
// list (CPP_3-NNPS.cpp:339-345): weight() / weight2() of the pair in FP64, or
// in FP32 from the FP64 position differences in the bulk form.  One thread per
// particle walks its list, so for each slot a warp writes consecutive records.
template <int ND, typename R>
__device__ __forceinline__ void pairw_particle(const Dev& d, int i)
{
    const int N = d.p.N, nn = nbr_count(d, i);
    const PairI<R> I = pair_i<ND, R>(d, i);
    const R rra = R(1.0) / I.h;     // RN(1 / h_i), the reciprocal of ra when h_j = h_i
    // the next slot's index and position are loaded one slot ahead
    int jn = (nn > 1) ? d.s.nbr[(size_t)N + i] : 0;
    Pos pn = load_pos(d.s.xh, (nn > 0) ? d.s.nbr[i] : i);
    for (int s = 0; s < nn; s++) {
        const Pos pj = pn;
        if (s + 1 < nn) pn = load_pos(d.s.xh, jn);
        if (s + 2 < nn) jn = d.s.nbr[(size_t)(s + 2) * N + i];
        R w[4];
        pair_w_raw<ND, R>(d, I, rra, pj, w);
        store_w(d, s, i, w);
    }
}

template <int ND>
__global__ void __launch_bounds__(128, SPH_MINB_PAIRW) k_pairw(Dev d)
{
    const int i = IDX;
    if (i >= d.p.N || *d.s.err) return;
    {
        // k_density's record of the porosity gathers: mass, porosity, rho of
        // the last step and its reciprocal (for the divisions by rho_j)
        const double r = d.s.rho[i];
        double2* q = reinterpret_cast<double2*>(d.s.rrho) + 2 * (size_t)i;
        q[0] = make_double2(d.s.mass[i], d.s.porosity[i]);
        q[1] = make_double2(r, 1.0 / r);
    }
    {
        // the neighbour record of this step (vxp and mass change only between steps)
        const int N = d.p.N;
        double2* q = reinterpret_cast<double2*>(d.s.nv) + 2 * (size_t)i;
        q[0] = make_double2(d.s.vxp[i], d.s.vxp[N + i]);
        q[1] = make_double2(d.s.vxp[2 * N + i], d.s.mass[i]);
    }
    if (d.p.bulk) pairw_particle<ND, float>(d, i);
    else pairw_particle<ND, double>(d, i);
}
#endif  // !SPH_BULK32

// ---------------------------------------------------------------------------
// density(): fluid porosity (:25-54) and continuity (:57-165) -> rho_c.  The
// porosity loop needs only the kernel values and recomputes them from the
// neighbours' positions (pair_value); the continuity loop reads the gradients
// from the pair records.
template <int ND>
__global__ void __launch_bounds__(128, SPH_MINB_DENS) k_density(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    constexpr int nd = ND;
    const int ti = d.s.type[i], nn = nbr_count(d, i);
    const int l = *d.s.step;
    const Pos P = load_pos(d.s.xh, i);
    const double xi[3] = {P.x, P.y, P.z};
    double por = d.s.porosity[i];
    double pcop = d.s.poro_cop[i];
    if (ti == 1) {
        Sum<real> sup, sdown;
        const PairI<real> I = pair_i<ND, real>(d, i);
        const real rra = real(1.0) / I.h;
        MaskIter it(d, i, type_mask(d, i, 2));
        int s, j;
        while (it.next(s, j)) {
            real w[4];
            pair_value<ND, real>(d, I, rra, j, s, i, w);
            const NV pj = load_nv(d.s.rrho, j);     // (mass, porosity, rho, 1 / rho)
            const real mj = (real)pj.vx, rj = (real)pj.vz;
            const double rrj = pj.m;
            sup.add(div_rho(mj * (real)pj.vy, rj, rrj) * w[3]);
            sdown.add(div_rho(mj, rj, rrj) * w[3]);
        }
        const double up = sup.v(), down = sdown.v();
        if (fabs(down) > 1.0e-7) {
            pcop = por;
            por = up / down;
            if (l == 1) pcop = por;
        } else {
            pcop = por;
        }
        d.s.porosity[i] = por;
        d.s.poro_cop[i] = pcop;
    }
    double rnew = d.s.rho[i];
    if (ti != 7) {
        Sum<real> sup[3], sdown[3];
        double vi[3];
        for (int k = 0; k < 3; k++) vi[k] = d.s.vxp[k * N + i];
        const bool solid = (ti == 2 || ti == 4), fluid = (ti == 1 || ti == 3);
        const bool moving = (ti >= 1 && ti <= 4);
        // slots of i's own type (not for walls) and, for moving i, wall slots
        const SlotMask wallm = moving ? type_mask(d, i, 0) : SlotMask{0ull, 0ull};
        MaskIter it(d, i, (ti != 0 ? type_mask(d, i, ti) : SlotMask{0ull, 0ull}) | wallm);
        int s, j;
        while (it.next(s, j)) {
            double vxj[3];
            const NV nj = load_nv(d.s.nv, j);
            if (!wallm.has(s)) {
                vxj[0] = nj.vx; vxj[1] = nj.vy; vxj[2] = nj.vz;
            } else if (moving) {
                // virtual wall velocity (:89-121)
                for (int k = 0; k < 3; k++) vxj[k] = wall_vel(d, ti, j, vi, k);
            } else {
                continue;
            }
            real w[4];
            load_w(d, s, i, w);
            const real mj = (real)nj.m;
            if (solid) {
                const Pos pj = load_pos(d.s.xh, j);
                const double xj[3] = {pj.x, pj.y, pj.z};
                for (int k = 0; k < nd; k++) {
                    sup[k].add(mj * (real)(vi[k] - vxj[k]) * w[k]);
                    sdown[k].add(mj * (real)(xi[k] - xj[k]) * w[k]);
                }
            }
            if (fluid) {
                for (int k = 0; k < nd; k++) sup[k].add(mj * (real)(vi[k] - vxj[k]) * w[k]);
            }
        }
        double up[3], down[3];
        for (int k = 0; k < 3; k++) { up[k] = sup[k].v(); down[k] = sdown[k].v(); }
        double drhot = 0.0;
        if (solid) {
            for (int k = 0; k < nd; k++) {
                if (fabs(down[k]) > 1.0e-7) drhot -= up[k] / down[k];
                else drhot += up[k];
            }
        }
        if (fluid)
            for (int k = 0; k < nd; k++) drhot += up[k];
        const double rhop = d.s.rhop[i], dt = step_dt(d);
        if (ti == 1 && fabs(por) > 0.0001)
            rnew = rhop + drhot * dt + rhop * (por - pcop) / (1.0 - pcop);
        else
            rnew = rhop + drhot * dt;
    }
    // the continuity density with the mass, one record for the Shepard gathers
    reinterpret_cast<double2*>(d.s.rho_c)[i] = make_double2(rnew, d.s.mass[i]);
}

// Shepard filter (:168-188) reading every neighbour's continuity density
// (Jacobi order), then the local equation of state (CPP_7-1-eos_CR.cpp:22-43).
// The pass needs only the kernel values, which it recomputes from the
// neighbours' positions (pair_value) instead of streaming the 32-byte pair
// records for them.
template <int ND>
__global__ void __launch_bounds__(128, SPH_MINB) k_shepard_eos(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    const int ti = d.s.type[i], nn = nbr_count(d, i);
    Sum<real> sup, sdown;
    const PairI<real> I = pair_i<ND, real>(d, i);
    const real rra = real(1.0) / I.h;
    MaskIter it(d, i, type_mask(d, i, ti));
    int s, j;
    while (it.next(s, j)) {
        real w[4];
        pair_value<ND, real>(d, I, rra, j, s, i, w);
        const double2 cm = reinterpret_cast<const double2*>(d.s.rho_c)[j];
        const real mj = (real)cm.y;
        sup.add(mj * w[3]);
        sdown.add(mj / (real)cm.x * w[3]);
    }
    const double up = sup.v(), down = sdown.v();
    double r = reinterpret_cast<const double2*>(d.s.rho_c)[i].x;
    if (ti != 7 && fabs(down) > 1.0e-7) r = up / down;
    d.s.rho[i] = r;
    {
        // the strain loop's neighbour record: vxp and mass / rho of this step
        double2* q = reinterpret_cast<double2*>(d.s.svr) + 2 * (size_t)i;
        q[0] = make_double2(d.s.vxp[i], d.s.vxp[N + i]);
        q[1] = make_double2(d.s.vxp[2 * N + i], d.s.mass[i] / r);
    }
    const double prep = d.s.prep[i];
    if (ti == 1) {
        double pr = prep * (pow7(r / d.s.f_dens[i] / d.s.f_por[i]) - 1.0);
        d.s.pre[i] = pr + prep;
    } else if (ti == 3) {
        // the reference's comma expression evaluates to -1.0 (:34)
        double pr = 1.403 * prep * (-1.0);
        d.s.pre[i] = pr + prep;
    } else if (ti == 0 && d.s.matype[i] == 1) {
        double pr = prep * (pow7(r / d.s.rhop[i]) - 1.0);
        d.s.pre[i] = pr + prep;
    }
    {
        // the pressure gathers' record: mass, rho and pressure of this step
        double2* q = reinterpret_cast<double2*>(d.s.pmr) + 2 * (size_t)i;
        q[0] = make_double2(d.s.mass[i], r);
        q[1] = make_double2(d.s.pre[i], 0.0);
    }
}

// ---------------------------------------------------------------------------
// strain_noreg (CPP_7-1-strain.cpp:20-220), the gathered pore pressures and
// wall stresses of eos (CPP_7-1-eos_CR.cpp:46-177) and the colour sum of
// free_surface_check (CPP_7-2-constitutive.cpp:462-480): a loop over the
// slots of the particle's own type and the walls, then one over the fluid
// (and, for walls, soil) slots, each sum in list order.  Writes de, we,
// color, prew, prea,
// and the walls' gathered stress into sig_next (reads the soil stresses of
// the previous step from sig).
template <int ND>
__global__ void __launch_bounds__(128, SPH_MINB_STRAIN) k_strain(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    constexpr int nd = ND;
    const int ti = d.s.type[i], nn = nbr_count(d, i);
    const Pos P = load_pos(d.s.xh, i);
    double vi[3];
    for (int k = 0; k < 3; k++) vi[k] = d.s.vxp[k * N + i];
    const bool solid = (ti == 2 || ti == 4);
    const bool moving = (ti >= 1 && ti <= 4);
    Sum<real> sup[9], sdown[3];
    Sum<real> scolor;
    // the velocity-gradient and colour sums over i's own type (not walls,
    // not type 7) and, for moving i, the walls
    const SlotMask wallm = moving ? type_mask(d, i, 0) : SlotMask{0ull, 0ull};
    MaskIter it(d, i, ((ti != 0 && ti != 7) ? type_mask(d, i, ti) : SlotMask{0ull, 0ull}) | wallm);
    int q, j;
    while (it.next(q, j)) {
        const bool same = !wallm.has(q);
        real w[4];
        load_w(d, q, i, w);
        // vxp and m_j / rho_j (the quotient the reference forms per pair,
        // formed once per particle by k_shepard_eos: the same value in FP64;
        // the FP32-bulk form divides its FP32 operands per pair)
        NV nj;
        real mr;
        if constexpr (sizeof(real) == 8) {
            nj = load_nv(d.s.svr, j);
            mr = (real)nj.m;
        } else {
            nj = load_nv(d.s.nv, j);
            mr = (real)nj.m / (real)d.s.rho[j];
        }
        {
            real dvx[3];
            const double vjs[3] = {nj.vx, nj.vy, nj.vz};
            for (int k = 0; k < 3; k++) {
                double vj = same ? vjs[k] : wall_vel(d, ti, j, vi, k);
                dvx[k] = (real)(vi[k] - vj);
            }
            sup[0].add(mr * dvx[0] * w[0]);
            sup[1].add(mr * dvx[0] * w[1]);
            sup[2].add(mr * dvx[0] * w[2]);
            sup[3].add(mr * dvx[1] * w[0]);
            sup[4].add(mr * dvx[1] * w[1]);
            sup[5].add(mr * dvx[1] * w[2]);
            sup[6].add(mr * dvx[2] * w[0]);
            sup[7].add(mr * dvx[2] * w[1]);
            sup[8].add(mr * dvx[2] * w[2]);
            if (solid) {
                const Pos pj = load_pos(d.s.xh, j);
                sdown[0].add(mr * (real)(P.x - pj.x) * w[0]);
                sdown[1].add(mr * (real)(P.y - pj.y) * w[1]);
                sdown[2].add(mr * (real)(P.z - pj.z) * w[2]);
            }
            scolor.add(mr * real(1.0) * w[3]);
        }
    }
    // velocity gradient (:148-181), strain rate and spin (:183-218), written
    // before the gathers below so that their sums are not held across them
    {
        double up[9], down[3];
        for (int k = 0; k < 9; k++) up[k] = sup[k].v();
        for (int k = 0; k < 3; k++) down[k] = sdown[k].v();
        double dv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (ti == 1 || ti == 3) {
            for (int k = 0; k < 9; k++) dv[k] = up[k];
        } else {
            if (fabs(down[0]) > 1.0e-7) { dv[0] = up[0] / down[0]; dv[3] = up[3] / down[0]; dv[6] = up[6] / down[0]; }
            if (fabs(down[1]) > 1.0e-7) { dv[1] = up[1] / down[1]; dv[4] = up[4] / down[1]; dv[7] = up[7] / down[1]; }
            if (fabs(down[2]) > 1.0e-7) { dv[2] = up[2] / down[2]; dv[5] = up[5] / down[2]; dv[8] = up[8] / down[2]; }
        }
        double de[6] = {dv[0], dv[4], dv[8], dv[1] + dv[3], dv[5] + dv[7], dv[6] + dv[2]};
        double we[6] = {0.5 * (dv[1] - dv[3]), 0.5 * (dv[2] - dv[6]), 0.5 * (dv[3] - dv[1]),
                        0.5 * (dv[5] - dv[7]), 0.5 * (dv[6] - dv[2]), 0.5 * (dv[7] - dv[5])};
        if (nd == 2) {
            de[2] = 0.0; de[4] = 0.0; de[5] = 0.0;
            we[1] = 0.0; we[3] = 0.0; we[4] = 0.0; we[5] = 0.0;
        }
        for (int k = 0; k < 6; k++) {
            d.s.de[k * N + i] = de[k];
            d.s.we[k * N + i] = we[k];
        }
        d.s.color[i] = scolor.v();
    }
    // the pressure (and, for walls, stress) gathers of eos from the fluids
    // (and, for walls, the soil), in a loop of their own over those slots:
    // per particle the water (type 1) and air (type 3) pressure sums u1 / d1
    // and u2 / d2, which the reference keeps in separate variables for soil
    // and structure particles (only one of which a particle is)
    if (ti == 2 || ti == 4 || ti == 0) {
        Sum<real> su1, su2, sd1, sd2;
        Sum<real> sus[6], sdsw;
        const SlotMask m1 = type_mask(d, i, 1), m3 = type_mask(d, i, 3);
        MaskIter itg(d, i, m1 | m3 | (ti == 0 ? type_mask(d, i, 2) : SlotMask{0ull, 0ull}));
        while (itg.next(q, j)) {
            const int tj = m1.has(q) ? 1 : m3.has(q) ? 3 : 2;
            real w[4];
            load_w(d, q, i, w);
            const NV pm = load_nv(d.s.pmr, j);      // (mass, rho, pre, -)
            const real mj = (real)pm.vx, rj = (real)pm.vy;
            const real w3 = w[3];
            const real pj_ = (ti == 0 && tj == 2) ? real(0) : (real)pm.vz;
            if (tj == 1) { su1.add(mj * pj_ * w3 / rj); sd1.add(mj * w3 / rj); }
            if (tj == 3) { su2.add(mj * pj_ * w3 / rj); sd2.add(mj * w3 / rj); }
            if (ti == 0 && tj == 2) {
                for (int k = 0; k < 6; k++) sus[k].add(mj * (real)d.s.sig[k * N + j] * w3 / rj);
                sdsw.add(mj * w3 / rj);
            }
        }
        // gathered pressures (eos :122-176)
        const double u1 = su1.v(), u2 = su2.v(), d1 = sd1.v(), d2 = sd2.v();
        d.s.prew[i] = (d1 != 0.0) ? u1 / d1 : u1;
        d.s.prea[i] = (d2 != 0.0) ? u2 / d2 : u2;
        if (ti == 0) {
            const double dsw = sdsw.v();
            for (int k = 0; k < 6; k++) {
                const double us = sus[k].v();
                d.s.sig_next[k * N + i] = (dsw != 0.0) ? us / dsw : us;
            }
        }
    }
}

// saturation (flagum == 1, CPP_7-1-strain.cpp:222-281): each soil particle's
// degree of saturation from the Shepard ratio of its water neighbours, its
// change dsatu (a decrease is undone), the clamp to [sitar, sitas] and the
// suction of moisturesuct.  Reads only the particle's own satu, so the
// in-place and Jacobi orders agree.
__global__ void __launch_bounds__(128, SPH_MINB) k_saturation(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err || d.s.type[i] != 2) return;
    const double sitas = d.s.s_sitas[i], sitar = d.s.s_sitar[i], cof = sitas - sitar;
    const int nn = nbr_count(d, i);
    Sum<real> up, down;
    for (int s = 0; s < nn; s++) {
        const int j = d.s.nbr[(size_t)s * N + i];
        if (d.s.type[j] != 1) continue;
        real w[4];
        load_w(d, s, i, w);
        const double mr = d.s.mass[j] / d.s.rho[j];
        up.add((real)(mr * cof) * w[3]);
        down.add((real)mr * w[3]);
    }
    const double tempup = up.v(), tempdown = down.v();
    const double psatu = d.s.satu[i];
    double satu = (tempdown != 0.0) ? tempup / tempdown + sitar : tempup + sitar;
    double dsatu = satu - psatu;
    if (dsatu < 0) {
        satu = satu - dsatu;
        dsatu = 0.0;
    }
    if (satu > sitas) satu = sitas;
    else if (satu < sitar) satu = sitar;
    d.s.satu[i] = satu;
    d.s.dsatu[i] = dsatu;
    d.s.suct[i] = moisture_suction(satu, dsatu, sitas, sitar, d.s.s_ext + i, N);
}

// cal_permeability (CPP_7-2-constitutive.cpp:355-382), strain_to_stress
// (:13-321), free_surface_check's correction (:482-504) and Stress_eigValue
// (CPP_7-1-strain.cpp:283-332), per particle.  Also evaluates the particle's
// own stress / rho^2 and pore-pressure / rho^2 terms the momentum pass uses.
// PHASE 0 does all of it.  Where stress_regu can run (step_regu within the
// run), PHASE 1 stops after the constitutive update (writing sig_next), the
// smoothing pass runs, and PHASE 2 continues from the smoothed stresses.
template <int ND, int PHASE>
__global__ void __launch_bounds__(128, SPH_MINB_STRESS) k_stress(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    const int ti = d.s.type[i], l = *d.s.step;
    const double dt = step_dt(d);
    double s[6], ep[6], de[6], we9[9];
    for (int k = 0; k < 6; k++) {
        if (PHASE == 2) s[k] = d.s.sig_tmp[k * N + i];
        else s[k] = (ti == 0) ? d.s.sig_next[k * N + i] : d.s.sig[k * N + i];
        ep[k] = (PHASE == 2) ? d.s.eps[k * N + i] : d.s.eps_in[k * N + i];
        de[k] = d.s.de[k * N + i];
    }
    if (PHASE != 2 && l == d.p.inip)
        for (int k = 0; k < 6; k++) ep[k] = 0.0;
    double vsig = 0, veps = 0, divq = 0, divr = 0, meps = 0;
    bool have_deq = false;
    if (PHASE != 2) {
    {
        double w6[6];
        for (int k = 0; k < 6; k++) w6[k] = d.s.we[k * N + i];
        we9[0] = 0.0; we9[1] = w6[0]; we9[2] = w6[1];
        we9[3] = w6[2]; we9[4] = 0.0; we9[5] = w6[3];
        we9[6] = w6[4]; we9[7] = w6[5]; we9[8] = 0.0;
    }
    if (d.p.fli == 1 && ti == 2) {
        double cop = d.s.cop[i];
        const int pt = d.p.permtype;
        if (pt == 0) cop = d.s.s_cop[i];
        else if (pt == 1) cop = d.p.pers;
        else if (pt == 2) {
            double sitas = d.s.s_sitas[i], sitar = d.s.s_sitar[i], sat = d.s.satu[i];
            if (sat < sitar) cop = d.p.pers;
            else if (sat > sitas) cop = d.p.perl;
            else cop = (d.p.perl - d.p.pers) * sat / (sitas - sitar) + d.p.pers;
        } else if (pt == 3) {
            const int pm = d.s.permtype[i];
            if (pm == 1) cop = d.p.pers;
            if (pm == 2) cop = d.p.perm;
            if (pm == 3) cop = d.p.perl;
        }
        d.s.cop[i] = cop;
    }
    if (ti == 1 || ti == 3) {
        double viscos1 = d.s.f_vis[i];
        if (ti == 1) {
            const double smin = d.s.f_smin[i];
            double depsmax = (de[0] + de[1] + de[2]) / 3.0;
            ep[0] = de[0] - depsmax;
            ep[1] = de[1] - depsmax;
            ep[2] = de[2] - depsmax;
            depsmax = 0.666666666666667 * (ep[0] * ep[0] + ep[1] * ep[1]
                + ep[2] * ep[2] + de[3] * de[3] * 0.25 +
                de[4] * de[4] * 0.25 + de[5] * de[5] * 0.25);
            depsmax = sqrt(depsmax);
            if (d.s.f_bhtype[i] == 1) {
                double tao = d.s.pre[i] * d.s.f_tanfai[i] + d.s.f_c[i];
                if (depsmax < smin) viscos1 = d.s.f_vis[i] + tao / smin;
                else viscos1 = d.s.f_vis[i] + tao / depsmax;
            }
        }
        double dd_[6];
        dd_[0] = 2.0 * de[0] - 2.0 * (de[0] + de[1] + de[2]) / 3.0;
        dd_[1] = 2.0 * de[1] - 2.0 * (de[0] + de[1] + de[2]) / 3.0;
        dd_[2] = 2.0 * de[2] - 2.0 * (de[0] + de[1] + de[2]) / 3.0;
        dd_[3] = de[3]; dd_[4] = de[4]; dd_[5] = de[5];
        const double pr = d.s.pre[i];
        for (int a = 0; a < 6; a++) s[a] = (a < 3) ? -pr - viscos1 * dd_[a] : -viscos1 * dd_[a];
    } else if (ti == 2 || ti == 4) {
        double D[6][6], adps[6] = {0, 0, 0, 0, 0, 0}, ds[6] = {0, 0, 0, 0, 0, 0};
        double erfs[6] = {0, 0, 0, 0, 0, 0};
        double dlam, dmu, sm;
        const int m = d.s.matype[i], mt = m % 10;
        const bool plastic = (ti == 2) && !(l < d.p.inip);
        const bool dp = plastic && (mt == 2 || mt == 5);
        // TSSMP step 1 (CPP_7-2-constitutive.cpp:99-101): the model and the
        // Jaumann terms see the transformed stress
        const bool ts = (ti == 2) && d.p.flts >= 1;
        double ts_s[6], qc = 0.0;
        if (ts) {
            const double sp[3] = {d.s.strep[i], d.s.strep[N + i], d.s.strep[2 * N + i]};
            qc = tssmp_before(s, ts_s, sp, d.s.vsig[i], d.s.divq[i], d.p.alphats);
        }
        if (ti == 2) {
            // elastic_plastic (M-C, matype 9) and sub_camunsatu (3) take their
            // mean stress with 0.333333333
            elastic_consts(s, d.s.s_e[i], d.s.s_poi[i], d.s.s_eps0[i], d.s.s_kapa[i], &dlam, &dmu, &sm,
                           (plastic && (mt == 9 || mt == 3)) ? 0.333333333 : 0.3333333333);
        } else {
            const double e0 = d.p.st_e, poi = d.p.st_poi;
            dlam = e0 * poi / (1.0 + poi) / (1.0 - 2.0 * poi);
            dmu = e0 * 0.5 / (1.0 + poi);
            sm = 0.0;
        }
        // sub_camanisotropy (matype 4, CPP_8-2-consfactor-amcc.cpp:17-99) has
        // its body commented out: its dept stays zero
        fill_elastic(D, (plastic && mt == 4) ? 0.0 : dlam, (plastic && mt == 4) ? 0.0 : dmu);
        if (dp) dp_tangent(D, adps, s, de, dlam, dmu, sm, d.s.s_yalf[i], d.s.s_ykap[i], (mt == 5) ? d.s.s_yalf_dil[i] : 0.0);
        if (plastic && mt == 9) dp_tangent<true>(D, adps, s, de, dlam, dmu, sm, d.s.s_yalf[i], d.s.s_ykap[i], 0.0);
        if (plastic && mt == 1)
            subcam_tangent(D, adps, s, de, dlam, dmu, sm, d.s.s_ann[i], d.s.s_zmf[i], d.s.s_ramda[i], d.s.s_kapa[i],
                           d.s.s_eps0[i], d.s.s_sme0[i], d.s.s_fs[i]);
        // the two rarely used models run out of line on copies in local
        // memory, so that D, s and de of the other models stay in registers
        if (plastic && mt == 3) {
            double Dl[6][6], sl[6], dl[6], al[6], el[6];
            for (int a = 0; a < 6; a++) {
                sl[a] = s[a]; dl[a] = de[a]; al[a] = 0.0; el[a] = 0.0;
                for (int b = 0; b < 6; b++) Dl[a][b] = D[a][b];
            }
            unsat_tangent(Dl, al, el, sl, dl, dlam, dmu, sm, d.s.satu[i], d.s.dsatu[i], d.s.s_zmf[i], d.s.s_fs[i],
                          d.s.s_ramda[i], d.s.s_kapa[i], d.s.s_eps0[i], d.s.s_sme0[i], d.s.s_ann[i],
                          d.s.s_sitas[i], d.s.s_sitar[i], d.s.s_ext + i, N);
            for (int a = 0; a < 6; a++) {
                adps[a] = al[a]; erfs[a] = el[a];
                for (int b = 0; b < 6; b++) D[a][b] = Dl[a][b];
            }
        }
        // fractional-order Cam-clay (matype 8): D and the elastic compliance C
        double C[6][6];
        const bool fo_plastic = (ti == 2) && (m == 8 || m == 18 || m == 28);
        if (fo_plastic || (plastic && mt == 8))
            for (int a = 0; a < 6; a++)
                for (int b = 0; b < 6; b++) C[a][b] = 0.0;
        if (plastic && mt == 8) {
            double Dl[6][6], sl[6], dl[6];
            for (int a = 0; a < 6; a++) { sl[a] = s[a]; dl[a] = de[a]; }
            focc_tangent(Dl, C, sl, dl, d.s.e[i], d.s.s_poi[i], d.s.s_zmf[i], d.s.s_ramda[i], d.s.s_ann[i],
                         d.s.s_ext + i, N);
            for (int a = 0; a < 6; a++)
                for (int b = 0; b < 6; b++) D[a][b] = Dl[a][b];
        }
        // StiffMat::depp0 = dept (CPP_7-2-constitutive.cpp:112-229, 292), which
        // the vibration damping reads through its largest diagonal entry; the
        // viscous-elastic model (matype % 10 == 7) leaves it as it was
        if (d.s.stiff && (ti == 4 || !plastic || mt != 7)) {
            double st = fmax(0.0, D[0][0]);
            st = fmax(st, D[1][1]);
            st = fmax(st, D[2][2]);
            d.s.stiff[i] = st;
        }
        if (plastic && mt == 7) {
            double smv;
            const double e0 = elastic_e0(s, d.s.s_e[i], d.s.s_poi[i], d.s.s_eps0[i], d.s.s_kapa[i], &smv);
            visco_elastic(ds, de, e0, d.s.s_poi[i], d.s.s_c[i]);
        } else
            add_dense(ds, D, de);
        if (dp) dp_check(s, ds, d.s.s_yalf[i], d.s.s_ykap[i], dt);
        jaumann(ds, s, we9);
        // fractional_plastic for matype 8, 18, 28 (:255-258).  In elastic steps
        // (l < inip) the reference reads its compliance uninitialised there;
        // only the output-only adps depends on it, and a zero compliance is
        // taken.
        if (fo_plastic) fractional_plastic(ds, de, adps, C);
        if (ts) {
            // TSSMP step 2 (:261-262): the rate back to the real stress space
            tssmp_after(ds, s, ts_s, d.s.divq[i], qc);
            for (int a = 0; a < 6; a++) d.s.tssig[a * N + i] = ts_s[a];
            d.s.tsqc[i] = qc;
        }
        if (ti == 2) {
            for (int a = 0; a < 6; a++) {
                double ad = d.s.adps[a * N + i];
                d.s.adps[a * N + i] = ad + adps[a] * dt;
                ep[a] = ep[a] + de[a] * dt;
                s[a] = s[a] + ds[a] * dt + erfs[a];
            }
        } else {
            for (int a = 0; a < 6; a++) {
                ep[a] = ep[a] + de[a] * dt;
                s[a] = s[a] + ds[a] * dt;
            }
        }
        deq(s, ep, &vsig, &veps, &divq, &divr);
        meps = shearstrain(ep, veps);
        have_deq = true;
        // poro_cal (Class_particle.cpp:194-203)
        double e = d.s.e[i];
        double dE = (1 + e) * (de[0] + de[1] + de[2]) * dt;
        double et = e + dE;
        if (et < 0.0) et = 0.0;
        d.s.porosity[i] = et / (1 + et);
        d.s.e[i] = et;
    }
    }   // PHASE != 2
    if (PHASE == 1) {
        // stresses before stress_regu, and the invariants of the last deq
        for (int k = 0; k < 6; k++) {
            d.s.sig_next[k * N + i] = s[k];
            d.s.eps[k * N + i] = ep[k];
        }
        if (have_deq) {
            d.s.vsig[i] = vsig; d.s.veps[i] = veps; d.s.divq[i] = divq; d.s.divr[i] = divr;
            d.s.meps[i] = meps;
        }
        return;
    }
    if (PHASE == 2 && (ti == 2 || ti == 4)) {
        vsig = d.s.vsig[i]; veps = d.s.veps[i]; divq = d.s.divq[i]; divr = d.s.divr[i];
        meps = d.s.meps[i];
        have_deq = true;
    }
    // free_surface_check correction (:482-504)
    const double color = d.s.color[i];
    const double tmax = d.p.thr_max, tmin = d.p.thr_min, incline = tmax - tmin;
    if (ti == 1) {
        if (color < tmin / 2.0) {
            s[0] = s[1] = s[2] = -1.0;
            s[3] = s[4] = s[5] = 0.0;
        } else if (color >= tmin / 2.0 && color < tmax / 2.0) {
            double xishu = (2.0 * color - tmin) / incline;
            for (int k = 0; k < 6; k++) s[k] = xishu * s[k];
        }
    } else if (ti == 2) {
        if (color < tmin) {
            s[0] = s[1] = s[2] = -1.0;
            s[3] = s[4] = s[5] = 0.0;
        } else if (color >= tmin && color < tmax) {
            double xishu = (color - tmin) / incline * 1.0;
            for (int k = 0; k < 6; k++) s[k] = xishu * s[k];
        }
        // Particle::stress_adjust (Class_particle.cpp:205-215) on the vsig of the last deq
        if (vsig > 0.0) {
            double temp = -vsig;
            s[0] = s[0] + temp; s[1] = s[1] + temp; s[2] = s[2] + temp;
            s[3] = 0.0; s[4] = 0.0; s[5] = 0.0;
        }
        deq(s, ep, &vsig, &veps, &divq, &divr);
    }
    if (have_deq || ti == 2) {
        d.s.vsig[i] = vsig; d.s.veps[i] = veps; d.s.divq[i] = divq; d.s.divr[i] = divr;
        d.s.meps[i] = meps;
    }
    double sp[3];
    eig3(s, sp);
    for (int k = 0; k < 3; k++) d.s.strep[k * N + i] = sp[k];
    // own halves of the momentum pair terms (CPP_9-4-derivation_stress.cpp):
    // fluids use porosity * sigma / rho / rho, soil and structure sigma / rho / rho
    const double r = d.s.rho[i];
    const double pf = (ti == 1 || ti == 3) ? d.s.f_por[i] : 0.0;
    double srk[6];
    for (int k = 0; k < 6; k++) {
        d.s.sig_next[k * N + i] = s[k];
        d.s.eps[k * N + i] = ep[k];
        srk[k] = (ti == 1 || ti == 3) ? pf * s[k] / r / r : s[k] / r / r;
    }
    double pp = 0.0;
    if (ti == 2) {
        const double satu = d.s.satu[i], por = d.s.s_por[i];
        pp = (1 - por) * (-satu * d.s.prew[i] + (1 - satu) * d.s.prea[i]) / r / r;
    } else if (ti == 4) {
        const double satu = d.s.satu[i];
        pp = (-satu * d.s.prew[i] + (1 - satu) * d.s.prea[i]) / r / r;
    }
    store_sr(d.s.sr, i, srk, pp, d.s.mass[i]);
    {
        // the drag loop's record: rho, saturation, porosity, and the soil's
        // permeability or the fluid's density
        double2* q = reinterpret_cast<double2*>(d.s.dr4) + 2 * (size_t)i;
        q[0] = make_double2(r, d.s.satu[i]);
        q[1] = make_double2(d.s.porosity[i], (ti == 2) ? d.s.cop[i] : d.s.f_dens[i]);
    }
}

// The per-particle tensor R_i of artificial_stress_2d / artificial_stress_3d
// (CPP_9-5-artificialstress.cpp:50-86, 180-234) for soil particles, from the
// stresses k_stress finished with: in 2-D from the in-plane principal
// direction, in 3-D R_i = beta^-1 diag(r) beta_ts^-1 with beta = v^T and
// beta_ts = v the eigenvectors of Stress_eigValue (CPP_7-1-strain.cpp:311-330)
// and r_k = -coe sigma_k / rho^2 for the tensile principal stresses.
// Only run when art_stre_coe > 0.
template <int ND>
__global__ void __launch_bounds__(128) k_art_rij(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    if (d.s.type[i] != 2) return;
    double s[6];
    for (int k = 0; k < 6; k++) s[k] = d.s.sig_next[k * N + i];
    const double xishu = d.p.art_stre_coe, r = d.s.rho[i];
    if (ND == 3) {
        double sp[3], v[9], bt[9], bi[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, bti[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        eig3v(s, sp, v);
        double st[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, tmp[9], R[9];
        for (int k = 0; k < 3; k++) st[k * 4] = (sp[k] > 0.0) ? -xishu * sp[k] / r / r : 0.0;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) bt[a * 3 + b] = v[b * 3 + a];
        inv3_or_keep(bt, bi);
        inv3_or_keep(v, bti);
        mul3(bi, st, tmp);
        mul3(tmp, bti, R);
        for (int k = 0; k < 9; k++) d.s.rij[k * N + i] = R[k];
    } else {
        const double pi_ = 3.141592653;   // Header_Parameters.h:10
        double sita;
        if (fabs(s[0] - s[1]) < 1.0e-6) {
            if (s[3] > 0.0) sita = -pi_ * 0.78539816325;
            else if (s[3] < 0.0) sita = pi_ * 0.78539816325;
            else sita = 0.0;
        } else
            sita = 0.5 * atan(2.0 * s[3] / (s[0] - s[1]));
        const double cs = cos(sita), sn = sin(sita);
        const double sxx = cs * cs * s[0] + 2.0 * sn * cs * s[3] + sn * sn * s[1];
        const double syy = sn * sn * s[0] - 2.0 * sn * cs * s[3] + cs * cs * s[1];
        const double rxx = (sxx > 0.0) ? -xishu * sxx / r / r : 0.0;
        const double ryy = (syy > 0.0) ? -xishu * syy / r / r : 0.0;
        const double r01 = (rxx - ryy) * sn * cs;
        d.s.rij[0 * N + i] = rxx * cs * cs + ryy * sn * sn;
        d.s.rij[1 * N + i] = r01;
        d.s.rij[3 * N + i] = r01;
        d.s.rij[4 * N + i] = rxx * sn * sn + ryy * cs * cs;
    }
}

// ---------------------------------------------------------------------------
// fluid_acceleration_water/air (+ minor forms), soil_acceleration_noreg and
// structure_acceleration_noreg (CPP_9-4-derivation_stress.cpp:12-505): the
// stress-divergence sums, whose per-pair stress / rho^2 halves were evaluated
// once per particle by k_stress.  Writes ax = g + sums for particle types 1-4;
// k_accel_b continues from this value in the reference's order.
template <int ND>
__global__ void __launch_bounds__(128, SPH_MINB_ACCA) k_accel_a(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    const int ti = d.s.type[i];
    const bool fluid = (ti == 1 || ti == 3);
    const bool solid = (ti == 2 || ti == 4);
    if (!fluid && !solid) return;
    const int nn = nbr_count(d, i);
    const double ri = d.s.rho[i];
    const int other = (ti == 1) ? 3 : 1;
    const bool minor = (ti == 1) ? d.p.water_minor : d.p.air_minor;
    real sri[6];
    {
        const SR own = load_sr(d.s.sr, i);
        for (int k = 0; k < 6; k++) sri[k] = (real)own.s[k];
    }
    Sum<real> tf[3][3];
    const double satu_i = d.s.satu[i];
    const double prew_i = solid ? d.s.prew[i] : 0.0, prea_i = solid ? d.s.prea[i] : 0.0;
    const double poro_f = fluid ? d.s.f_por[i] : 0.0;
    const double poro_s = (ti == 2) ? d.s.s_por[i] : 0.0;
    const double dens_s = (ti == 2) ? d.s.s_dens[i] : 1.0;
    // own pore term with the particle's own saturation (used when the
    // neighbour's saturation is the same)
    double pi_own = 0.0;
    if (ti == 2) pi_own = (1 - poro_s) * (-satu_i * prew_i + (1 - satu_i) * prea_i) / dens_s / dens_s;
    if (ti == 4) pi_own = (-satu_i * prew_i + (1 - satu_i) * prea_i) / ri / ri;
    // fluid: its own and the other fluid's slots; solid: its own type's
    MaskIter it(d, i, fluid ? (type_mask(d, i, ti) | type_mask(d, i, other)) : type_mask(d, i, ti));
    int q, j;
    while (it.next(q, j)) {
        const bool f_pair = fluid;
        const bool s_pair = solid;
        real w[4];
        load_w(d, q, i, w);
        const SR rj_ = load_sr(d.s.sr, j);
        const real mj = (real)rj_.m;
        real srj[6];
        if (s_pair || same_bits(d.s.f_por[j], poro_f)) {
            for (int k = 0; k < 6; k++) srj[k] = (real)rj_.s[k];
        } else {
            const double rj = d.s.rho[j];
            for (int k = 0; k < 6; k++) srj[k] = (real)(poro_f * d.s.sig_next[k * N + j] / rj / rj);
        }
        if (f_pair && minor) {
            tf[0][0].add(mj * (srj[0] - sri[0]) * w[0]);
            tf[0][1].add(mj * (srj[3] - sri[3]) * w[1]);
            tf[0][2].add(mj * (srj[5] - sri[5]) * w[2]);
            tf[1][0].add(mj * (srj[3] - sri[3]) * w[0]);
            tf[1][1].add(mj * (srj[1] - sri[1]) * w[1]);
            tf[1][2].add(mj * (srj[4] - sri[4]) * w[2]);
            tf[2][0].add(mj * (srj[5] - sri[5]) * w[0]);
            tf[2][1].add(mj * (srj[4] - sri[4]) * w[1]);
            tf[2][2].add(mj * (srj[2] - sri[2]) * w[2]);
        } else {
            tf[0][0].add(mj * (srj[0] + sri[0]) * w[0]);
            tf[0][1].add(mj * (srj[3] + sri[3]) * w[1]);
            tf[0][2].add(mj * (srj[5] + sri[5]) * w[2]);
            tf[1][0].add(mj * (srj[3] + sri[3]) * w[0]);
            tf[1][1].add(mj * (srj[1] + sri[1]) * w[1]);
            tf[1][2].add(mj * (srj[4] + sri[4]) * w[2]);
            tf[2][0].add(mj * (srj[5] + sri[5]) * w[0]);
            tf[2][1].add(mj * (srj[4] + sri[4]) * w[1]);
            tf[2][2].add(mj * (srj[2] + sri[2]) * w[2]);
        }
        if (s_pair) {
            const double satu = d.s.satu[j];
            if (ti == 2) {
                double pj_, pi_;
                if (same_bits(d.s.s_por[j], poro_s)) {
                    pj_ = rj_.p;
                } else {
                    const double rj = d.s.rho[j];
                    pj_ = (1 - poro_s) * (-satu * d.s.prew[j] + (1 - satu) * d.s.prea[j]) / rj / rj;
                }
                pi_ = same_bits(satu, satu_i) ? pi_own
                    : (1 - poro_s) * (-satu * prew_i + (1 - satu) * prea_i) / dens_s / dens_s;
                const real pq = (real)(pj_ + pi_);
                tf[0][0].add(mj * pq * w[0]);
                tf[1][1].add(mj * pq * w[1]);
                tf[2][2].add(mj * pq * w[2]);
            } else {
                const double pj_ = rj_.p;
                const double pi_ = same_bits(satu, satu_i) ? pi_own
                    : (-satu * prew_i + (1 - satu) * prea_i) / ri / ri;
                const real pq = (real)(pj_ - pi_);
                tf[0][0].add(mj * pq * w[0]);
                tf[1][1].add(mj * pq * w[1]);
                tf[2][2].add(mj * pq * w[2]);
            }
        }
    }
    const double g[3] = {d.p.gx, d.p.gy, d.p.gz};
    double ax[3];
    for (int k = 0; k < 3; k++) ax[k] = g[k];
    ax[0] += tf[0][0].v() + tf[0][1].v() + tf[0][2].v();
    ax[1] += tf[1][0].v() + tf[1][1].v() + tf[1][2].v();
    ax[2] += tf[2][0].v() + tf[2][1].v() + tf[2][2].v();
    for (int k = 0; k < 3; k++) d.s.ax[k * N + i] = ax[k];
}

// Soil-water drag coefficient of interact2 (Tsuji / Shi, form 2,
// CPP_10-interact1.cpp:154-176) and interact3 (Peng, form 3, :294-306) for
// a soil particle of porosity por and grain diameter ds in water of density
// dens and viscosity vis, at relative speed mag_v; rho_w is the density the
// reference reads there.  Out of line: only fli 2/3 call it, and its pow calls
// would otherwise widen the register budget of every run.
__device__ __noinline__ double drag_beta(int form, double por, double ds, double dens, double vis, double mag_v,
                                         double rho_w)
{
    double re, cd, beta;
    if (form == 2) {
        re = mag_v * dens * por * ds / vis;
        if (re > 1000.0) cd = 0.43;
        else if (fabs(re) > 0.0001) cd = 24.0 * (1.0 + 0.15 * pow(re, 0.687)) / re;
        else cd = 0.0;
        if (por <= 0.8) {
            beta = 150.0 * (1.0 - por) * (1.0 - por) / por / por / ds / ds * vis;
            beta = beta + 1.75 * (1.0 - por) / ds / por * dens * mag_v;
        } else
            beta = 0.75 * cd * mag_v * dens * (1.0 - por) / ds * pow(por, -2.7);
    } else {
        re = mag_v * dens * ds / vis;
        cd = por * por * por * ds * ds * 0.0066666667 / (1.0 - por) / (1.0 - por);
        if (re > 60.0) beta = vis / cd + 1.75 / sqrt(150.0) * rho_w * mag_v / sqrt(cd) / pow(por, 1.5);
        else beta = vis / cd;
    }
    return beta;
}

// The wall-stress sums of one moving particle (boundary_moving_stress_effect,
// CPP_9-4-derivation_stress.cpp:631-721; boundary_stress_effect_tran,
// :725-846; boundary_effect_free_struct, :900-990) over the wall particles of
// its list, in list order: the rows (t_k0 + t_k1) + t_k2 that are added to the
// acceleration.  Out of line, so that its nine sums and the particle's
// stress operands hold registers only for particles next to a wall.
template <int ND>
__device__ __noinline__ void wall_stress_rows(int i, int N, unsigned long long wlo, unsigned long long whi, int ti,
                                              bool fluid, bool tran, bool free_struct,
                                              double ri, double satu_i, const int* nbr,
                                              const double* nbw, const double* mass, const double* rho,
                                              const double* sb, const double* sig_next, const double* prew,
                                              const double* prea, double rows[3])
{
    Sum<real> tb[3][3];
    real ab[6], abr[6];
    double si[6];
    for (int k = 0; k < 6; k++) si[k] = sig_next[k * N + i];
    double abd[6];
    if (fluid || (tran && ti == 4)) {
        for (int k = 0; k < 6; k++) abd[k] = si[k];
    } else {
        const double prew_i = prew[i], prea_i = prea[i];
        abd[0] = si[0] - satu_i * prew_i + (1 - satu_i) * prea_i;
        abd[1] = si[1] - satu_i * prew_i + (1 - satu_i) * prea_i;
        abd[2] = si[2] - satu_i * prew_i + (1 - satu_i) * prea_i;
        abd[3] = si[3]; abd[4] = si[4]; abd[5] = si[5];
    }
    for (int k = 0; k < 6; k++) {
        ab[k] = (real)abd[k];
        abr[k] = (real)(abd[k] / ri / ri);
    }
    // the wall slots (type 0) of the list, in slot order
    for (int wd = 0; wd < 2; wd++) {
      unsigned long long m = wd ? whi : wlo;
      while (m) {
        const int q = wd * 64 + __ffsll((long long)m) - 1;
        m &= m - 1;
        const int j = nbr[(size_t)q * N + i];
        real w[4];
        load_w_raw(nbw, N, q, i, w);
        const real mj = (real)mass[j], rj = (real)rho[j];
        real abj[6];
        if (free_struct && fluid)
            for (int k = 0; k < 6; k++) abj[k] = ((k < 3) ? ab[k] : -ab[k]) / rj / rj;
        else if (tran)
            for (int k = 0; k < 6; k++)
                abj[k] = (real)(sb[(size_t)((ti - 1) * 6 + k) * N + j] / rho[j] / rho[j]);
        else
            for (int k = 0; k < 6; k++) abj[k] = ab[k] / rj / rj;
        tb[0][0].add(mj * (abj[0] + abr[0]) * w[0]);
        tb[0][1].add(mj * (abj[3] + abr[3]) * w[1]);
        tb[0][2].add(mj * (abj[5] + abr[5]) * w[2]);
        tb[1][0].add(mj * (abj[3] + abr[3]) * w[0]);
        tb[1][1].add(mj * (abj[1] + abr[1]) * w[1]);
        tb[1][2].add(mj * (abj[4] + abr[4]) * w[2]);
        tb[2][0].add(mj * (abj[5] + abr[5]) * w[0]);
        tb[2][1].add(mj * (abj[4] + abr[4]) * w[1]);
        tb[2][2].add(mj * (abj[2] + abr[2]) * w[2]);
      }
    }
    for (int k = 0; k < 3; k++) rows[k] = tb[k][0].v() + tb[k][1].v() + tb[k][2].v();
}

// ff_stress_2d_solid / ff_stress_3d_solid (CPP_19-FreeFieldParticles.cpp:21-76,
// the same in CPP_19-FreeFieldParticles_soil.cpp:21-68): the viscous stress a
// free-field particle of elastic constants (e, poi), density dens and wave
// direction `type` (its permtype) puts between velocities va and vb
template <int ND>
__device__ __forceinline__ void ff_stress(double sg[3], const double va[3], const double vb[3], double e, double poi,
                                          double dens, int type)
{
    const double g = e * 0.5 / (1 + poi);
    const double k = e * 0.333333333333333 / (1 - 2.0 * poi);
    const double c_p = sqrt((k + 4.0 * g * 0.333333333333333) / dens);
    const double c_s = sqrt(g / dens);
    sg[0] = 0.0; sg[1] = 0.0; sg[2] = 0.0;
    if (ND == 2) {
        if (type == 1) {
            sg[0] = -c_p * dens * (va[0] - vb[0]);
            sg[1] = -c_s * dens * (va[1] - vb[1]);
        } else if (type == 2) {
            sg[0] = -c_s * dens * (va[0] - vb[0]);
            sg[1] = -c_p * dens * (va[1] - vb[1]);
        }
    } else {
        const double c0 = (type == 1) ? c_p : c_s, c1 = (type == 2) ? c_p : c_s, c2 = (type == 3) ? c_p : c_s;
        if (type >= 1 && type <= 3) {
            sg[0] = -c0 * dens * (va[0] - vb[0]);
            sg[1] = -c1 * dens * (va[1] - vb[1]);
            sg[2] = -c2 * dens * (va[2] - vb[2]);
        }
    }
}

// artificial_viscosity (CPP_9-3-artificialvis.cpp:12-99), the pair sum of
// artificial_stress_2d/_3d (CPP_9-5-artificialstress.cpp, ART = 1),
// boundary_moving_stress_effect (CPP_9-4-derivation_stress.cpp:631-721),
// interact1/2/3 (CPP_10-interact1.cpp:15-405), soil_damping_geostress
// (CPP_9-4:849-896) and veocity_update (CPP_11-xsph.cpp:11-142): one loop
// per group of sums over the list slots that group takes (its own type; the
// types the drag pairs; walls; soil), each sum over its pairs in list order,
// combined with the stress-divergence result of k_accel_a in the reference's
// call order.
// Writes ax, interf, interfss and the updated velocity into vx_next (the
// reference's vx before XSPH).  DRAG = 1 carries the interact2/3 drag
// coefficient (fli 2, 3), whose out-of-line call the Darcy form does without.
// VIB = 1 (flv != 0) adds the vibration damping and free-field sums to the
// first loop; runs without vibration take the variant without them.
template <int ND, int DRAG = 0, int LOOP = 0, int VIB = 0>
__global__ void __launch_bounds__(128, LOOP ? SPH_MINB_ACCB2 : SPH_MINB_ACCB1) k_accel_b(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    constexpr int nd = ND;
    const int ti = d.s.type[i], nn = nbr_count(d, i);
    const PairI<real> I = pair_i<ND, real>(d, i);
    const double ri = d.s.rho[i];
    const real riR = (real)ri;
    double vi[3];
    for (int k = 0; k < 3; k++) vi[k] = d.s.vxp[k * N + i];
    const bool solid = (ti == 2 || ti == 4);
    Sum<real> tav[3], tin[3], tdm[3];
    const bool damping = (*d.s.step <= d.p.inip) && solid;
    const real cdi = damping ? (real)d.s.cd[i] : real(0);
    // artificial viscosity coefficients of particle i
    real ca = 0, aa = 0, bb = 0;
    if (ti == 1) { ca = (real)d.s.f_vpu[i]; aa = (real)d.p.av[0][0]; bb = (real)d.p.av[0][1]; }
    if (ti == 2) { ca = (real)d.s.s_vpu[i]; aa = (real)d.p.av[1][0]; bb = (real)d.p.av[1][1]; }
    if (ti == 3) { ca = (real)d.s.f_vpu[i]; aa = (real)d.p.av[2][0]; bb = (real)d.p.av[2][1]; }
    const double satu_i = d.s.satu[i];
    // vibration (flv != 0): the free-field sums of free_field_solid over the
    // walls of matype 5 (CPP_19-FreeFieldParticles.cpp:79-141) and of its soil
    // form between free-field soil (matype >= 50) and the rest
    // (CPP_19-FreeFieldParticles_soil.cpp:71-175), for soil particles; the
    // sums of soil_damping_vibration (CPP_9-1-acceleration_vibration.cpp:
    // 171-224) for soil and structure particles (flv > 0)
    const bool ffree = LOOP == 0 && VIB && d.p.flv != 0 && ti == 2;
    const bool vdamp = LOOP == 0 && VIB && d.p.flv > 0 && solid;
    Sum<real> tfw[3], tfs[3], tdv[3], tdn;
    real cdv = 0;
    double vnow_i[3] = {0.0, 0.0, 0.0};
    const int mti = d.s.matype[i];
    if (vdamp) {
        const double hl = d.s.xh[4 * (size_t)i + 3];
        cdv = (real)(d.s.s_ext[(size_t)SX_DAMP1 * N + i] +
                     d.s.s_ext[(size_t)SX_DAMP2 * N + i] * sqrt(d.s.stiff[i] / d.s.rhop[i] / hl / hl));
    }
    if (ffree) {
        for (int k = 0; k < 3; k++) vnow_i[k] = d.s.vx[k * N + i];
        MaskIter itw(d, i, type_mask(d, i, 0));
        int q, j;
        while (itw.next(q, j)) {
            if (d.s.matype[j] != 5) continue;
            real w[4];
            load_w(d, q, i, w);
            double vj[3], sg[3];
            for (int k = 0; k < 3; k++) vj[k] = d.s.interfss[k * N + j];
            const double rj = d.s.rho[j];
            ff_stress<ND>(sg, vnow_i, vj, d.p.ff_e, d.p.ff_poi, rj, d.s.permtype[j]);
            const real mr = (real)(d.s.mass[j] / rj);
            for (int k = 0; k < nd; k++) tfw[k].add(mr * (real)sg[k] / riR * w[k]);
        }
    }
    // artificial viscosity and geostatic damping over i's own type's slots,
    // then the soil-water (soil-air) drag of interact1/2/3 over the slots of
    // the types it pairs (the reference visits every other pair of different
    // types too, but adds nothing for them); each sum in list order
    if (LOOP == 0) {
        MaskIter it(d, i, (ti != 7) ? type_mask(d, i, ti) : SlotMask{0ull, 0ull});
        int q, j;
        while (it.next(q, j)) {
            const bool dm_pair = damping;
            const Pos pj = load_pos(d.s.xh, j);
            real w[4];
            load_w(d, q, i, w);
            const NV nj = load_nv(d.s.nv, j);
            const real mj = (real)nj.m, rj = (real)d.s.rho[j];
            const double xj[3] = {pj.x, pj.y, pj.z};
            const double vjs[3] = {nj.vx, nj.vy, nj.vz};
            real inprod = 0, dst = 0, dx[3], dvx[3];
            for (int k = 0; k < nd; k++) {
                dvx[k] = (real)(vi[k] - vjs[k]);
                dx[k] = (real)(I.x[k] - xj[k]);
                dst = dst + dx[k] * dx[k];
                inprod = inprod + dvx[k] * dx[k];
            }
            const real hl = ((real)pj.h + I.h) * real(0.5);
            const real rou = (rj + riR) * real(0.5);
            real paix;
            if (inprod < real(0)) {
                dst = sqrt(dst);
                real myu = hl * inprod / (dst * dst + real(0.01) * hl * hl);
                paix = (-aa * ca * myu + bb * myu * myu) / rou;
            } else
                paix = 0;
            for (int k = 0; k < nd; k++) tav[k].add(mj * paix * w[k]);
            if (dm_pair)
                for (int k = 0; k < nd; k++) tdm[k].add(mj / rj * cdi * dvx[k] * w[3]);
            if (vdamp) {
                for (int k = 0; k < nd; k++) tdv[k].add(mj / rj * cdv * dvx[k] * w[3]);
                tdn.add(mj / rj * w[3]);
            }
            if (ffree) {
                const int mtj = d.s.matype[j];
                if ((mti < 50) != (mtj < 50)) {
                    double vj[3], sg[3];
                    for (int k = 0; k < 3; k++) vj[k] = d.s.vx[k * N + j];
                    if (mti < 50)
                        ff_stress<ND>(sg, vnow_i, vj, d.s.s_e[j], d.s.s_poi[j], d.s.rho[j], d.s.permtype[j]);
                    else
                        ff_stress<ND>(sg, vj, vnow_i, d.s.s_e[i], d.s.s_poi[i], ri, d.s.permtype[i]);
                    for (int k = 0; k < nd; k++) tfs[k].add(mj / rj * (real)sg[k] / riR * w[k]);
                }
            }
        }
    }
    if (LOOP == 1 && d.p.fli >= 1 && (ti == 1 || ti == 2 || ti == 3)) {
        const SlotMask m1 = type_mask(d, i, 1);
        MaskIter it(d, i, (ti == 2) ? (m1 | type_mask(d, i, 3)) : type_mask(d, i, 2));
        int q, j;
        while (it.next(q, j)) {
            const int tj = (ti != 2) ? 2 : m1.has(q) ? 1 : 3;
            const Pos pj = load_pos(d.s.xh, j);
            real w[4];
            load_w(d, q, i, w);
            const NV nj = load_nv(d.s.nv, j);
            const NV dj = load_nv(d.s.dr4, j);      // (rho, satu, porosity, cop | f_dens)
            const real mj = (real)nj.m, rj = (real)dj.vx;
            const double xj[3] = {pj.x, pj.y, pj.z};
            const double vjs[3] = {nj.vx, nj.vy, nj.vz};
            real inprod = 0, dvx[3];
            for (int k = 0; k < nd; k++) {
                dvx[k] = (real)(vi[k] - vjs[k]);
                const real dxk = (real)(I.x[k] - xj[k]);
                inprod = inprod + dvx[k] * dxk;
            }
            if (inprod < 0) {
                const real w3 = w[3], ga = (real)d.p.g_acc;
                if (DRAG && d.p.fli > 1 && ((ti == 2 && tj == 1) || (ti == 1 && tj == 2))) {
                    // interact2/3 soil-water drag, m_j / rho_j W beta (v_i - v_j)
                    double mv = 0.0;
                    for (int k = 0; k < nd; k++) mv = mv + (double)dvx[k] * (double)dvx[k];
                    mv = sqrt(mv);
                    const int so = (ti == 2) ? i : j, wa = (ti == 2) ? j : i;
                    const real beta = (real)drag_beta(d.p.fli, d.s.porosity[so], d.s.s_ds[so], d.s.f_dens[wa],
                                                      d.s.f_vis[wa], mv, (ti == 2) ? dj.vx : ri);
                    for (int k = 0; k < nd; k++) tin[k].add(mj / rj * w3 * beta * dvx[k]);
                } else if (ti == 2 && tj == 1) {
                    const real sa = (real)satu_i, po = (real)d.s.porosity[i], cp = (real)d.s.cop[i],
                               fd = (real)dj.m;
                    for (int k = 0; k < nd; k++)
                        tin[k].add(sa * sa * po * po * fd * ga * dvx[k] / cp * mj / rj * w3);
                } else if (ti == 1 && tj == 2) {
                    const real sa = (real)dj.vy, po = (real)dj.vz, cp = (real)dj.m,
                               fd = (real)d.s.f_dens[i];
                    for (int k = 0; k < nd; k++)
                        tin[k].add(sa * sa * po * po * fd * ga * dvx[k] / cp * mj / rj * w3);
                } else if (ti == 2 && tj == 3) {
                    const real sa = (real)satu_i, po = (real)d.s.porosity[i], fd = (real)dj.m;
                    for (int k = 0; k < nd; k++)
                        tin[k].add((1 - sa) * (1 - sa) * po * po * fd * ga * dvx[k] * 2000 * mj / rj * w3);
                } else if (ti == 3 && tj == 2) {
                    const real sa = (real)dj.vy, po = (real)dj.vz, fd = (real)d.s.f_dens[i];
                    for (int k = 0; k < nd; k++)
                        tin[k].add((1 - sa) * (1 - sa) * po * po * fd * ga * dvx[k] * 2000 * mj / rj * w3);
                }
            }
        }
    }
    if (LOOP == 0 && VIB && d.p.flv != 0) {
        for (int k = 0; k < 3; k++) {
            d.s.accb[(size_t)(9 + k) * N + i] = (double)tfw[k].v();
            d.s.accb[(size_t)(12 + k) * N + i] = (double)tfs[k].v();
            d.s.accb[(size_t)(15 + k) * N + i] = (double)tdv[k].v();
        }
        d.s.accb[(size_t)18 * N + i] = (double)tdn.v();
    }
    for (int k = 0; k < 3; k++) {
        if (LOOP == 0) {
            d.s.accb[(size_t)k * N + i] = (double)tav[k].v();
            d.s.accb[(size_t)(6 + k) * N + i] = (double)tdm[k].v();
        } else {
            d.s.accb[(size_t)(3 + k) * N + i] = (double)tin[k].v();
        }
    }
}

// The vibration load of the step at time t (vibration_acceleration and
// vibration_velocity, CPP_9-1-acceleration_vibration.cpp:10-160): 0 outside
// [sttime, edtime]; else the entry of Para_Vibra::loads the elapsed time
// selects in v, and 1 when its largest magnitude is under 1000, 2 when not.
__device__ __forceinline__ int vib_load(const Dev& d, double t, double v[3])
{
    const double time1 = t - d.p.vib_st, time2 = t - d.p.vib_ed;
    if (!(time1 >= 0.0 && time2 <= 0.0)) return 0;
    const int ns = d.p.vib_nsteps;
    // (int)(time1 / ttime * nsteps), capped at nsteps - 1 (the cap taken
    // before the conversion, which would overflow past it)
    const double q = time1 / d.p.vib_ttime * (double)ns;
    const int step = (q >= (double)(ns - 1)) ? ns - 1 : (int)q;
    for (int k = 0; k < 3; k++) v[k] = d.s.vib_loads[(size_t)step * 3 + k];
    double m = fmax(0.0, fabs(v[0]));
    m = fmax(m, fabs(v[1]));
    m = fmax(m, fabs(v[2]));
    return (m < 1000.0) ? 1 : 2;
}

// The rest of the momentum pass, per particle: the wall stress and the
// artificial-stress sums (each over the list in order), then the combination
// with the sums of k_accel_b (accb) and k_accel_a in the reference's call
// order, the velocity update and the writes of ax, interf, interfss and the
// velocity before XSPH (vx_next).  In a kernel of its own so that the loops of
// k_accel_b run under a smaller register budget than this straight-line code.
template <int ND, int ART = 0, int VIB = 0>
__global__ void __launch_bounds__(128, SPH_MINB_ACCB) k_accel_b_tail(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    constexpr int nd = ND;
    const int ti = d.s.type[i], nn = nbr_count(d, i);
    const PairI<real> I = pair_i<ND, real>(d, i);
    const double ri = d.s.rho[i];
    double vi[3];
    for (int k = 0; k < 3; k++) vi[k] = d.s.vxp[k * N + i];
    const bool fluid = (ti == 1 || ti == 3);
    const bool solid = (ti == 2 || ti == 4);
    const bool moving = (ti >= 1 && ti <= 4);
    const bool damping = (*d.s.step <= d.p.inip) && solid;
    const bool art = ART && ti == 2;   // artificial stress (art_stre_coe > 0)
    // wall-stress operand of particle i (:668-700) and its own half
    const double satu_i = d.s.satu[i];
    // flbndy 3/4/13/14: boundary_stress_effect_tran (CPP_9-4:725-846) takes the
    // wall's stress for i's phase, and a structure particle's own stress
    // without the pore terms
    const bool tran = d.p.flbndy == 3 || d.p.flbndy == 4 || d.p.flbndy == 13 || d.p.flbndy == 14;
    // boundary_effect_free_struct (CPP_9-4:900-990) for the other flbndy
    // values: a fluid's mirrored stress has its shear components negated
    const bool free_struct = !(tran || d.p.flbndy == 1 || d.p.flbndy == 2);
    const SlotMask wallm = type_mask(d, i, 0);
    // the artificial-viscosity, drag and damping sums of k_accel_b
    double tav[3], tin[3], tdm[3];
    for (int k = 0; k < 3; k++) {
        tav[k] = d.s.accb[(size_t)k * N + i];
        tin[k] = d.s.accb[(size_t)(3 + k) * N + i];
        tdm[k] = d.s.accb[(size_t)(6 + k) * N + i];
    }
    // the wall stress of moving particles with a wall in their list, out of
    // line (its nine sums take registers only there); each sum still runs
    // over the list in order
    double tbrow[3] = {0.0, 0.0, 0.0};
    if (moving && wallm.any())
        wall_stress_rows<ND>(i, N, wallm.lo, wallm.hi, ti, fluid, tran, free_struct, ri, satu_i, d.s.nbr, d.s.nbw,
                             d.s.mass, d.s.rho, d.s.sb, d.s.sig_next, d.s.prew, d.s.prea, tbrow);
    // the artificial-stress pair sum (ART), likewise in a loop of its own
    Sum<real> tu[3];
    if (art) {
        MaskIter ita(d, i, type_mask(d, i, 2));
        int q, j;
        while (ita.next(q, j)) {
            const Pos pj = load_pos(d.s.xh, j);
            real w[4];
            load_w(d, q, i, w);
            const real mj = (real)d.s.mass[j];
            const double xj[3] = {pj.x, pj.y, pj.z};
            // artificial_stress_2d/_3d pair sum (CPP_9-5-artificialstress.cpp:
            // 100-140, 248-290): f_ij = (W(q) / W(dr))^2.55 of the cubic
            // spline, m_j f_ij (R_i + R_j) grad W_ij
            real dst = 0;
            for (int k = 0; k < 3; k++) {
                const real t = (real)(I.x[k] - xj[k]);
                dst = dst + t * t;
            }
            dst = sqrt(dst);
            const real hl = (I.h + (real)pj.h) * real(0.5);
            const real qd = dst / hl;
            real f;
            if (qd >= real(0) && qd < real(1))
                f = pow((real(0.666666666666667) - qd * qd + real(0.5) * qd * qd * qd) * real(3.82300884955752), real(2.55));
            else if (qd >= real(1) && qd < real(2))
                f = pow((real(2.0) - qd) * (real(2.0) - qd) * (real(2.0) - qd) * real(0.629737609329447), real(2.55));
            else f = 0;
            for (int a = 0; a < nd; a++) {
                Sum<real> acc = tu[a];
                for (int b = 0; b < nd; b++) {
                    const int c = a * 3 + b;
                    acc.add(mj * f * (real)(d.s.rij[(size_t)c * N + i] + d.s.rij[(size_t)c * N + j]) * w[b]);
                }
                tu[a] = acc;
            }
        }
    }
    double ax[3];
    for (int k = 0; k < 3; k++) ax[k] = d.s.ax[k * N + i];   // g + stress divergence (k_accel_a) or the old value
    if (ti != 7)
        for (int k = 0; k < nd; k++) ax[k] = ax[k] - tav[k];
    if (art)
        for (int k = 0; k < nd; k++) ax[k] = ax[k] + tu[k].v();
    if (moving)
        for (int k = 0; k < 3; k++) ax[k] += tbrow[k];
    if (VIB && d.p.flv != 0 && ti == 2) {
        // free_field_solid: the walls' sum, then the soil form's
        for (int k = 0; k < nd; k++) ax[k] = ax[k] + d.s.accb[(size_t)(9 + k) * N + i];
        for (int k = 0; k < nd; k++) ax[k] = ax[k] + d.s.accb[(size_t)(12 + k) * N + i];
    }
    if (d.p.ss_coupled && (ti == 1 || ti == 2 || ti == 4))
        for (int k = 0; k < 3; k++) ax[k] += d.s.cpl[(size_t)k * N + i];
    const double dt = step_dt(d);
    double axp[3];
    for (int k = 0; k < 3; k++) axp[k] = d.s.axp[k * N + i];
    if (d.p.fli >= 1 && moving) {
        const double xishu = d.p.interc;
        for (int k = 0; k < nd; k++) {
            double itf = tin[k];
            double vx1 = vi[k] + 0.5 * (axp[k] + ax[k]) * dt;
            double vx2 = vi[k] + 0.5 * (axp[k] + ax[k] - itf * xishu / ri) * dt;
            if (vx1 * vx2 <= 0.0) {
                itf = 0.0;
                ax[k] = -2.0 * vi[k] / dt - axp[k];
            } else
                ax[k] -= itf * xishu / ri;
            d.s.interf[k * N + i] = itf;
        }
    }
    if (d.p.ss_type >= 1 && (ti == 1 || ti == 2 || ti == 4)) {
        // the contact forces into interfss and the acceleration
        // (CPP_10-1-interact_ss.cpp:1008-1034 and the same sums of the rigid
        // and deformable forms, which scale them by zeta)
        const bool own = (ti != 4) && d.s.ss_id[i] >= 0;
        double fn[3] = {0, 0, 0}, ft[3] = {0, 0, 0};
        if (ti == 4) {
            for (int k = 0; k < 3; k++) { fn[k] = d.s.ss_fs[(size_t)k * N + i]; ft[k] = d.s.ss_fs[(size_t)(3 + k) * N + i]; }
        } else if (own) {
            for (int k = 0; k < 3; k++) { fn[k] = d.s.ss_own[(size_t)k * N + i]; ft[k] = d.s.ss_own[(size_t)(3 + k) * N + i]; }
        }
        const double mi = d.s.mass[i];
        for (int k = 0; k < 3; k++) {
            double f = 0.0;
            if (d.p.ss_type != 3) f += d.p.ss_zeta * (ft[k] + fn[k]);
            else f += ft[k] + fn[k];
            d.s.interfss[k * N + i] = f;
            ax[k] += f / mi;
        }
    }
    if (damping) {
        for (int k = 0; k < nd; k++) {
            double vx1 = vi[k] + 0.5 * (axp[k] + ax[k]) * dt;
            double vx2 = vi[k] + 0.5 * (axp[k] + ax[k] - tdm[k]) * dt;
            if (vx1 * vx2 <= 0.0) ax[k] = -2.0 * vi[k] / dt - axp[k];
            else ax[k] -= tdm[k];
        }
    }
    if (VIB && d.p.flv > 0 && solid) {
        // soil_damping_vibration (CPP_9-1-acceleration_vibration.cpp:171-224)
        double td = d.s.accb[(size_t)18 * N + i];
        for (int k = 0; k < nd; k++) {
            if (fabs(td) < 1.0e-7) td = 1.0e-7;
            const double dm = d.s.accb[(size_t)(15 + k) * N + i];
            double vx1 = vi[k] + 0.5 * (axp[k] + ax[k]) * dt;
            double vx2 = vi[k] + 0.5 * (axp[k] + ax[k] - dm / td) * dt;
            if (vx1 * vx2 <= 0.0) ax[k] = -2.0 * vi[k] / dt - axp[k];
            else ax[k] -= dm / td;
        }
    }
    if (d.p.flbndy == 5 && d.s.fsol_on[i]) {
        // boundary_free_solid (CPP_13-boundary.cpp:1239-1516), after the damping
        const double mi = d.s.mass[i];
        for (int k = 0; k < 3; k++) ax[k] += d.s.fsol[(size_t)k * N + i] / mi;
    }
    // veocity_update, if_move 0 and 1
    double vout[3];
    for (int k = 0; k < 3; k++) vout[k] = d.s.vx[k * N + i];
    const int mt = d.s.matype[i];
    if (VIB && d.p.flv == 1 && ti == 0 && (mt == 3 || mt == 5)) {
        // vibration_acceleration: the load into the wall's interf (a load of
        // 1000 or more, or a time outside the window, zeroes interf and
        // interfss)
        double v[3];
        const int ld = vib_load(d, *d.s.tsim + dt, v);
        for (int k = 0; k < nd; k++) {
            if (ld == 1) d.s.interf[k * N + i] = v[k];
            else { d.s.interf[k * N + i] = 0.0; d.s.interfss[k * N + i] = 0.0; }
        }
    }
    if (d.p.if_move == 0) {
        if (ti == 0 && mt < 2) {
            for (int k = 0; k < nd; k++) {
                d.s.interf[k * N + i] = 0.0;
                double ath = (0.0 + 0.0) * 0.5;
                d.s.interfss[k * N + i] = d.s.interfss[k * N + i] + ath * dt;
            }
        } else if (ti == 0 && (mt == 3 || (mt == 5 && d.p.flv == 1))) {
            for (int k = 0; k < nd; k++) {
                double itf = d.s.interf[k * N + i];
                double ath = (itf + itf) * 0.5;
                d.s.interfss[k * N + i] = d.s.interfss[k * N + i] + ath * dt;
            }
        } else if (ti != 0) {
            for (int k = 0; k < nd; k++) {
                double ath = (axp[k] + ax[k]) * 0.5;
                vout[k] = vi[k] + ath * dt;
            }
        }
    } else if (d.p.if_move == 1) {
        if (ti == 0 && mt == 2 && *d.s.step > d.p.inip) {
            for (int k = 0; k < nd; k++) d.s.interfss[k * N + i] = d.p.move_vx[k];
        } else if (ti == 0) {
            for (int k = 0; k < nd; k++) d.s.interfss[k * N + i] = 0.0;
        } else {
            for (int k = 0; k < nd; k++) {
                double ath = (axp[k] + ax[k]) * 0.5;
                vout[k] = vi[k] + ath * dt;
            }
        }
    } else {
        // if_move 2 (soil) / 3 (structure) with etype 5 driven at move_vx after
        // inip (CPP_11-xsph.cpp:92-141); every particle then takes
        // v = vxp + (axp + ax) dt / 2, walls included
        const int tmove = (d.p.if_move == 2) ? 2 : 4;
        double vp[3] = {vi[0], vi[1], vi[2]};
        if (ti == tmove && d.s.etype[i] == 5 && *d.s.step > d.p.inip) {
            for (int k = 0; k < nd; k++) {
                axp[k] = 0.0;
                vp[k] = d.p.move_vx[k];
                vout[k] = d.p.move_vx[k];
                ax[k] = 0.0;
            }
        }
        for (int k = 0; k < nd; k++) {
            double ath = (axp[k] + ax[k]) * 0.5;
            vout[k] = vp[k] + ath * dt;
        }
    }
    if (VIB && d.p.flv == 2 && ti == 0 && (mt == 4 || mt == 5)) {
        // vibration_velocity, after the velocity update: the load is the
        // wall's velocity interfss
        double v[3];
        const int ld = vib_load(d, *d.s.tsim + dt, v);
        for (int k = 0; k < nd; k++) {
            if (ld == 1) d.s.interfss[k * N + i] = v[k];
            else { d.s.interf[k * N + i] = 0.0; d.s.interfss[k * N + i] = 0.0; }
        }
    }
    for (int k = 0; k < 3; k++) d.s.ax[k * N + i] = ax[k];
    // the velocity before XSPH, with the mass, as one record for XSPH's gathers
    double2* vq = reinterpret_cast<double2*>(d.s.vx_next) + 2 * (size_t)i;
    vq[0] = make_double2(vout[0], vout[1]);
    vq[1] = make_double2(vout[2], d.s.mass[i]);
}

// xsph (CPP_11-xsph.cpp:145-256, Jacobi by construction: reads the velocities
// before XSPH), tmboundary (CPP_13-boundary.cpp:125-177), check_domain
// (CPP_13-boundary.cpp:20-68) and update (CPP_12-1-update.cpp:11-55).
// Reads xh / vx_next, writes xh_next / vx.
template <int ND>
__global__ void __launch_bounds__(128, SPH_MINB_XSPH) k_xsph_update(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    constexpr int nd = ND;
    const int ti = d.s.type[i], nn = nbr_count(d, i);
    const double dt = step_dt(d);
    const PairI<real> I = pair_i<ND, real>(d, i);
    double vm[3];
    {
        const NV own = load_nv(d.s.vx_next, i);
        vm[0] = own.vx; vm[1] = own.vy; vm[2] = own.vz;
    }
    const bool moving = (ti >= 1 && ti <= 4);
    double vn[3] = {vm[0], vm[1], vm[2]};
    const SlotMask wallm = type_mask(d, i, 0);
    const bool any_wall = wallm.any();
    if (d.p.if_move != 2 && moving) {
        const real xs_same = (real)((ti == 1) ? d.p.xsph0 : (ti == 3) ? d.p.xsph2 : d.p.xsph1);
        const real xs_wall = (real)((ti == 1 || ti == 3) ? 0.006 : d.p.xsph1 / 5.0);
        Sum<real> stu[3], sdown;
        // same-type and wall slots in list order (disjoint for moving i)
        MaskIter it(d, i, type_mask(d, i, ti) | wallm);
        int q, j;
        while (it.next(q, j)) {
            const real xishu = wallm.has(q) ? xs_wall : xs_same;
            real w[4];
            load_w(d, q, i, w);
            const NV nj = load_nv(d.s.vx_next, j);
            const real mj = (real)nj.m, rj = (real)d.s.rho[j];
            const double vjs[3] = {nj.vx, nj.vy, nj.vz};
            for (int k = 0; k < nd; k++)
                stu[k].add(xishu * mj * (real)(vjs[k] - vm[k]) * w[3] / rj);
            sdown.add(mj * w[3] / rj);
        }
        double tu[3];
        for (int k = 0; k < 3; k++) tu[k] = stu[k].v();
        const double down = sdown.v();
        if (fabs(down) > 1.0e-7 && (ti == 2 || ti == 4))
            for (int k = 0; k < nd; k++) vn[k] = vm[k] + tu[k] / down;
        else
            for (int k = 0; k < nd; k++) vn[k] = vm[k] + tu[k];
    }
    // tmboundary (flbndy 1, moving particles, a = b = 0.3) or
    // velocity_set_domain (flbndy 2, fluid particles, a = b = coe_bndy,
    // CPP_13-boundary.cpp:71-122): the same correction
    const bool vsd = d.p.flbndy == 2 || d.p.flbndy == 13 || d.p.flbndy == 14;
    const bool vcorr = (d.p.flbndy == 1 && moving) || (vsd && (ti == 1 || ti == 3));
    if (vcorr && any_wall) {
        const double a = (d.p.flbndy == 1) ? 0.30 : d.p.coe_bndy, b = a, dr = d.p.dr;
        double tb[3] = {0, 0, 0};
        MaskIter itw(d, i, wallm);
        int q, j;
        while (itw.next(q, j)) {
            const Pos pj = load_pos(d.s.xh, j);
            const double xj[3] = {pj.x, pj.y, pj.z};
            double inprod = 0.0, dst = 0.0;
            for (int k = 0; k < nd; k++) {
                inprod = inprod + (vn[k] - d.s.interfss[k * N + j]) * (I.x[k] - xj[k]);
                dst = dst + (I.x[k] - xj[k]) * (I.x[k] - xj[k]);
            }
            if (inprod < 0.0) {
                dst = sqrt(dst);
                const double db = a * dr;
                double beta = 1 + db / (dst - b * dr);
                beta = fmin(1.5, beta);
                for (int k = 0; k < nd; k++)
                    tb[k] = tb[k] + (1 - beta) * (I.x[k] - xj[k]) * inprod / dst / dst;
            }
        }
        for (int k = 0; k < nd; k++) vn[k] = vn[k] + tb[k];
    }
    else if (vcorr) {
        // no wall in the list: the correction adds zeros (kept, for -0.0)
        for (int k = 0; k < nd; k++) vn[k] = vn[k] + 0.0;
    }
    if (d.p.flbndy != 1 && d.p.flbndy != 5 && moving)
        for (int k = 0; k < 3; k++) d.s.vx_vb[k * N + i] = vn[k];
    if (ti != 0 && ti != 7) {
        const double dr = d.p.dr;
        const CellGrid g = cell_grid(d, i);
        const double bmax[3] = {g.xmax, g.ymax, g.zmax}, bmin[3] = {g.xmin, g.ymin, g.zmin};
        bool hit = false;
        if (I.x[0] - bmax[0] >= -0.5 * dr) hit = true;
        if (I.x[0] - bmin[0] <= 0.5 * dr) hit = true;
        if (I.x[1] - bmax[1] >= -0.5 * dr) hit = true;
        if (I.x[1] - bmin[1] <= 0.5 * dr) hit = true;
        if (I.x[2] - bmax[2] >= -0.5 * dr && nd == 3) hit = true;
        if (I.x[2] - bmin[2] <= 0.5 * dr && nd == 3) hit = true;
        if (hit) {
            // w0 and the comparison in the caller's order
            const int w0 = g.w0;
            const bool after = d.s.i2o[i] > w0;
            const int wi = after ? d.s.o2i[w0] : 0;
            for (int k = 0; k < 3; k++) vn[k] = after ? d.s.interfss[k * N + wi] : 0.0;
        }
    }
    // update (vxp is move_vx for the particles if_move 2 / 3 drives)
    const int loop = *d.s.step - d.p.inip;
    double xn[3] = {I.x[0], I.x[1], I.x[2]};
    const bool driven = d.p.if_move >= 2 && ti == ((d.p.if_move == 2) ? 2 : 4) && d.s.etype[i] == 5 &&
                        *d.s.step > d.p.inip;
    if (ti != 0) {
        for (int k = 0; k < nd; k++) {
            const double vp = driven ? d.p.move_vx[k] : d.s.vxp[k * N + i];
            xn[k] = I.x[k] + (vn[k] + vp) * dt * 0.5;
            double u = d.s.ux[k * N + i];
            u = (loop == 0) ? 0.0 : u + (vn[k] + vp) * dt * 0.5;
            d.s.ux[k * N + i] = u;
            d.s.vxp[k * N + i] = vn[k];
            d.s.axp[k * N + i] = d.s.ax[k * N + i];
        }
        if (nd > 0) d.s.rhop[i] = d.s.rho[i];
    } else {
        const int mt = d.s.matype[i];
        if (mt == 2 || mt == 3 || mt == 4 || mt == 5) {
            for (int k = 0; k < nd; k++) {
                const double its = d.s.interfss[k * N + i];
                xn[k] = I.x[k] + (its + its) * dt * 0.5;
                d.s.ux[k * N + i] = d.s.ux[k * N + i] + (its + its) * dt * 0.5;
            }
            d.s.rhop[i] = d.s.rho[i];
            d.s.prep[i] = d.s.pre[i];
        }
    }
    store_pos(d.s.xh_next, i, Pos{xn[0], xn[1], xn[2], load_pos(d.s.xh, i).h});
    for (int k = 0; k < 3; k++) d.s.vx[k * N + i] = vn[k];
}

// tm_boundary_2d / tm_boundary_3d, first pass (CPP_13-boundary.cpp:200-297,
// 410-508): for each moving particle the wall particles of its list with
// their distances, sorted as clParti_Pair::dist_sorting does (four passes
// swapping ids, not distances, Class_particle.cpp:343-359); the line through
// the two nearest (2-D, with clLine's C = 1 that cal_line leaves) or the plane
// through the three nearest (3-D; plane_two_points when they are collinear,
// D = 1 from clPlane() unless plane_two_points sets it), the particle's
// distance to it, and vel_bndy = (1 - beta) v + beta v_wall, v_wall the
// interfss of the last wall of matype > 2 in the list (particle 0 if none;
// in a batched context the instance's first particle).
template <int ND>
__global__ void __launch_bounds__(128) k_tm_vb(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    const int ti = d.s.type[i];
    if (ti == 0 || ti == 7) return;
    const int nn = nbr_count(d, i);
    int ids[SPH_NB_CAP];
    double dsts[SPH_NB_CAP];
    // without such a wall the reference reads particle 0 (of the instance)
    int total = 0, id = d.s.o2i[(d.p.ninst > 0) ? d.s.inst[d.s.pinst[i]].first : 0];
    const Pos P = load_pos(d.s.xh, i);
    for (int q = 0; q < nn; q++) {
        const int j = d.s.nbr[(size_t)q * N + i];
        if (d.s.type[j] != 0) continue;
        const Pos pj = load_pos(d.s.xh, j);
        const double d2 = (P.x - pj.x) * (P.x - pj.x) + (P.y - pj.y) * (P.y - pj.y) + (P.z - pj.z) * (P.z - pj.z);
        ids[total] = j;
        dsts[total] = sqrt(d2);
        total++;
        if (d.s.matype[j] > 2) id = j;
    }
    for (int a = 0; a < 4; a++)
        for (int b = a + 1; b < total; b++)
            if (dsts[a] > dsts[b]) { const int t = ids[a]; ids[a] = ids[b]; ids[b] = t; }
    double vi[3], vb[3];
    for (int k = 0; k < 3; k++) vi[k] = d.s.vx_vb[k * N + i];
    const double dr = d.p.dr;
    if (total >= (ND == 2 ? 2 : 3)) {
        const Pos q1 = load_pos(d.s.xh, ids[0]), q2 = load_pos(d.s.xh, ids[1]);
        const double p4[3] = {P.x, P.y, P.z}, p1[3] = {q1.x, q1.y, q1.z}, p2[3] = {q2.x, q2.y, q2.z};
        double dst;
        if (ND == 2) {
            // cal_line (:645-650), cal_dpline (:617-628)
            const double den = p2[1] * p1[0] - p1[1] * p2[0];
            const double A = (p1[1] - p2[1]) / den, B = (p2[0] - p1[0]) / den, C = 1.0;
            const double num = fabs(A * p4[0] + B * p4[1] + C);
            const double tmp = sqrt(A * A + B * B);
            dst = (tmp > 1.0e-3) ? num / tmp : 0.0;
        } else {
            const Pos q3 = load_pos(d.s.xh, ids[2]);
            const double p3[3] = {q3.x, q3.y, q3.z};
            double pc1[3], pc2[3], A, B, C, D = 1.0;
            // cal_plane (:653-666) of (p1, p2, p4) and (p1, p3, p4)
            const double den1 = -p1[0] * (p2[1] * p4[2] - p4[1] * p2[2]) - p2[0] * (p4[1] * p1[2] - p1[1] * p4[2]) -
                                p4[0] * (p1[1] * p2[2] - p2[1] * p1[2]);
            pc1[0] = p1[1] * (p2[2] - p4[2]) + p2[1] * (p4[2] - p1[2]) + p4[1] * (p1[2] - p2[2]);
            pc1[1] = p1[2] * (p2[0] - p4[0]) + p2[2] * (p4[0] - p1[0]) + p4[2] * (p1[0] - p2[0]);
            pc1[2] = p1[0] * (p2[1] - p4[1]) + p2[0] * (p4[1] - p1[1]) + p4[0] * (p1[1] - p2[1]);
            pc1[0] = pc1[0] / den1; pc1[1] = pc1[1] / den1; pc1[2] = pc1[2] / den1;
            const double den2 = -p1[0] * (p3[1] * p4[2] - p4[1] * p3[2]) - p3[0] * (p4[1] * p1[2] - p1[1] * p4[2]) -
                                p4[0] * (p1[1] * p3[2] - p3[1] * p1[2]);
            pc2[0] = p1[1] * (p3[2] - p4[2]) + p3[1] * (p4[2] - p1[2]) + p4[1] * (p1[2] - p3[2]);
            pc2[1] = p1[2] * (p3[0] - p4[0]) + p3[2] * (p4[0] - p1[0]) + p4[2] * (p1[0] - p3[0]);
            pc2[2] = p1[0] * (p3[1] - p4[1]) + p3[0] * (p4[1] - p1[1]) + p4[0] * (p1[1] - p3[1]);
            pc2[0] = pc2[0] / den2; pc2[1] = pc2[1] / den2; pc2[2] = pc2[2] / den2;
            double cs = pc1[0] * pc2[0] + pc1[1] * pc2[1] + pc1[2] * pc2[2];
            cs = cs / sqrt(pc1[0] * pc1[0] + pc1[1] * pc1[1] + pc1[2] * pc1[2]) /
                 sqrt(pc2[0] * pc2[0] + pc2[1] * pc2[1] + pc2[2] * pc2[2]);
            if (fabs(cs) > 0.999999) {
                // plane_two_points(p4, p1) (:684-708)
                const double a = p4[0] - p1[0], b = p4[1] - p1[1], c = p4[2] - p1[2];
                const double tmp = -a * p1[0] - b * p1[1] - c * p1[2];
                if (fabs(tmp) > 1.0e-6) { A = a / tmp; B = b / tmp; C = c / tmp; D = 1.0; }
                else { A = a; B = b; C = c; D = 0.0; }
            } else {
                const double den = -p1[0] * (p2[1] * p3[2] - p3[1] * p2[2]) - p2[0] * (p3[1] * p1[2] - p1[1] * p3[2]) -
                                   p3[0] * (p1[1] * p2[2] - p2[1] * p1[2]);
                A = p1[1] * (p2[2] - p3[2]) + p2[1] * (p3[2] - p1[2]) + p3[1] * (p1[2] - p2[2]);
                B = p1[2] * (p2[0] - p3[0]) + p2[2] * (p3[0] - p1[0]) + p3[2] * (p1[0] - p2[0]);
                C = p1[0] * (p2[1] - p3[1]) + p2[0] * (p3[1] - p1[1]) + p3[0] * (p1[1] - p2[1]);
                A = A / den; B = B / den; C = C / den;
            }
            // cal_dpplane (:631-642)
            const double num = fabs(A * p4[0] + B * p4[1] + C * p4[2] + D);
            const double tmp = sqrt(A * A + B * B + C * C);
            dst = (tmp > 1.0e-3) ? num / tmp : 0.0;
        }
        const double da = (dst > 0.6 * dr) ? dst - 0.5 * dr : 0.1 * dr;
        const double db = 0.5 * dr;
        double beta;
        if (fabs(da) > 1.0e-6) { beta = 1.0 + db / da; beta = fmin(1.5, beta); }
        else beta = 1.5;
        for (int k = 0; k < 2; k++) vb[k] = (1.0 - beta) * vi[k] + beta * d.s.interfss[(size_t)k * N + id];
        vb[2] = (ND == 2) ? 0.0 : (1.0 - beta) * vi[2] + beta * d.s.interfss[(size_t)2 * N + id];
    } else {
        for (int k = 0; k < 3; k++) vb[k] = vi[k];
    }
    for (int k = 0; k < 3; k++) d.s.vel_bndy[k * N + i] = vb[k];
}

// tm_boundary second pass (CPP_13-boundary.cpp:298-386, 509-614): each wall
// particle's Shepard sums of the moving neighbours' vel_bndy per phase, with
// the reference's [0][0] operand in components 1 and 2.
__global__ void __launch_bounds__(128) k_tm_wall(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    if (d.s.type[i] != 0) return;
    const int nn = nbr_count(d, i);
    double up[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, down[4] = {0, 0, 0, 0};
    for (int q = 0; q < nn; q++) {
        const int j = d.s.nbr[(size_t)q * N + i];
        const int tj = d.s.type[j];
        if (tj < 1 || tj > 4) continue;
        const int p = tj - 1;
        real w[4];
        load_w(d, q, i, w);
        const double w3 = w[3], mj = d.s.mass[j], rj = d.s.rho[j];
        up[p][0] = up[p][0] + mj * d.s.vel_bndy[j] * w3 / rj;
        up[p][1] = up[p][0] + mj * d.s.vel_bndy[(size_t)N + j] * w3 / rj;
        up[p][2] = up[p][0] + mj * d.s.vel_bndy[(size_t)2 * N + j] * w3 / rj;
        down[p] = down[p] + mj * w3 / rj;
    }
    for (int p = 0; p < 4; p++)
        for (int k = 0; k < 3; k++)
            d.s.vb[(size_t)(p * 3 + k) * N + i] = (fabs(down[p]) > 1.0e-6) ? up[p][k] / down[p] : 0.0;
}

// ---------------------------------------------------------------------------
// Soil-structure contact: interaction_ss_rigid / _deformable / _penalty
// (CPP_10-1-interact_ss.cpp:17-1036, geometry helpers :1039-1369).  The
// reference scatters each contact's reaction onto the two (2-D) or three
// (3-D) structure particles it touches, accumulating per thread; here each
// water / soil particle records its contact (k_ss_pair) and each structure
// particle gathers its reactions in ascending particle order (k_ss_struct),
// the order one reference thread applies them in.

struct SSPt { double x, y, z; };

__device__ __forceinline__ SSPt ss_pt(const Dev& d, int i)
{
    const Pos p = load_pos(d.s.xh, i);
    return SSPt{p.x, p.y, p.z};
}

// linear_interpolate (:1187-1202)
__device__ __forceinline__ void ss_interp(SSPt P1, SSPt P2, SSPt r, double m1, double m2, const double v1[3],
                                          const double v2[3], double* m, double v[3])
{
    const double xk1 = 0.0;
    const double xk2 = sqrt((P2.x - P1.x) * (P2.x - P1.x) + (P2.y - P1.y) * (P2.y - P1.y) + (P2.z - P1.z) * (P2.z - P1.z));
    const double xp = sqrt((r.x - P1.x) * (r.x - P1.x) + (r.y - P1.y) * (r.y - P1.y) + (r.z - P1.z) * (r.z - P1.z));
    *m = (m1 * fabs(xp - xk2) + m2 * fabs(xp - xk1)) / fabs(xk2 - xk1);
    for (int k = 0; k < 3; k++) v[k] = (v1[k] * fabs(xp - xk2) + v2[k] * fabs(xp - xk1)) / fabs(xk2 - xk1);
}

// linear_interpolate_force (:1204-1222)
__device__ __forceinline__ void ss_interp_force(SSPt P1, SSPt P2, SSPt r, const double f[3], double f1[3], double f2[3])
{
    const double xk1 = 0.0;
    const double xk2 = sqrt((P2.x - P1.x) * (P2.x - P1.x) + (P2.y - P1.y) * (P2.y - P1.y) + (P2.z - P1.z) * (P2.z - P1.z));
    const double xp = sqrt((r.x - P1.x) * (r.x - P1.x) + (r.y - P1.y) * (r.y - P1.y) + (r.z - P1.z) * (r.z - P1.z));
    for (int k = 0; k < 3; k++) f1[k] = -fabs(xp - xk2) / fabs(xk1 - xk2) * f[k];
    for (int k = 0; k < 3; k++) f2[k] = -fabs(xp - xk1) / fabs(xk1 - xk2) * f[k];
}

template <int ND>
__global__ void __launch_bounds__(128) k_ss_pair(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    for (int q = 0; q < 3; q++) d.s.ss_id[(size_t)q * N + i] = -1;
    const int ti = d.s.type[i];
    if (!(ti == 1 || ti == 2)) return;
    const int form = d.p.ss_type, nn = nbr_count(d, i);
    const double dt = step_dt(d), dr = d.p.dr, myu = d.p.ss_myu, zeta = d.p.ss_zeta;
    const double reach = (form == 1) ? 0.5 * dr : dr;
    int ids[SPH_NB_CAP];
    double dsts[SPH_NB_CAP];
    int total = 0;
    const SSPt p4 = ss_pt(d, i);
    for (int q = 0; q < nn; q++) {
        const int j = d.s.nbr[(size_t)q * N + i];
        if (d.s.type[j] != 4) continue;
        const SSPt pj = ss_pt(d, j);
        const double dd = (p4.x - pj.x) * (p4.x - pj.x) + (p4.y - pj.y) * (p4.y - pj.y) + (p4.z - pj.z) * (p4.z - pj.z);
        ids[total] = j;
        dsts[total] = sqrt(dd);
        total++;
    }
    for (int a = 0; a < 4; a++)   // clParti_Pair::dist_sorting
        for (int b = a + 1; b < total; b++)
            if (dsts[a] > dsts[b]) { const int t = ids[a]; ids[a] = ids[b]; ids[b] = t; }
    if (total < ND) return;
    const double mi = d.s.mass[i];
    double vpi[3];
    for (int k = 0; k < 3; k++) vpi[k] = d.s.vxp[(size_t)k * N + i];
    const int id1 = ids[0], id2 = ids[1];
    const SSPt p1 = ss_pt(d, id1), p2 = ss_pt(d, id2);
    double v1[3], v2[3];
    for (int k = 0; k < 3; k++) { v1[k] = d.s.vxp[(size_t)k * N + id1]; v2[k] = d.s.vxp[(size_t)k * N + id2]; }
    double fn[3] = {0, 0, 0}, ft[3] = {0, 0, 0};
    double con[3][6];                // reactions per slot: normal (3), tangential (3)
    int sid[3] = {-1, -1, -1};
    if (ND == 2) {
        // cal_line (:1055-1060) with clLine()'s C = 1, cal_dpline, cal_mappoint_line (:1094-1125)
        const double den = p2.y * p1.x - p1.y * p2.x;
        const double A = (p1.y - p2.y) / den, B = (p2.x - p1.x) / den, C = 1.0;
        const double tmp0 = sqrt(A * A + B * B);
        const double dp = (tmp0 > 1.0e-3) ? fabs(A * p4.x + B * p4.y + C) / tmp0 : 0.0;
        const double tmp = sqrt(A * A + B * B);
        const SSPt P1 = {p4.x + dp * A / tmp, p4.y + dp * B / tmp, 0.0}, P2 = {p4.x - dp * A / tmp, p4.y - dp * B / tmp, 0.0};
        const double dp1 = (tmp0 > 1.0e-3) ? fabs(A * P1.x + B * P1.y + C) / tmp0 : 0.0;
        SSPt outp = (dp1 < 1.0e-3) ? P1 : P2;
        outp.z = 0.0;
        // check_ifinside_line (:1290-1305) with the mapped point's z = 0
        const double v0x = p2.x - p1.x, v0y = p2.y - p1.y, v0z = p2.z - p1.z;
        const double w1x = outp.x - p1.x, w1y = outp.y - p1.y, w1z = 0.0 - p1.z;
        const double dot00 = v0x * v0x + v0y * v0y + v0z * v0z, dot01 = v0x * w1x + v0y * w1y + v0z * w1z;
        const double u = 1.0 / dot00 * dot01;
        if ((u < 0 || u > 1) || !(dp < reach)) return;
        // clLine::set_normal, check_ifoutward2D (:1252-1270)
        double nx = 0.0, ny = 0.0;
        const double tot = sqrt(A * A + B * B);
        if (tot > 1.0e-10) { nx = A / tot; ny = B / tot; }
        const double dot = (outp.x - p4.x) * nx + (outp.y - p4.y) * ny + 0.0 * 0.0;
        if (!(dot <= 0.0)) { nx = -nx; ny = -ny; }
        double ms, vs[3];
        ss_interp(p1, p2, outp, d.s.mass[id1], d.s.mass[id2], v1, v2, &ms, vs);
        vs[0] -= vpi[0];
        vs[1] -= vpi[1];
        if (form != 1) {
            vs[0] *= ms / (ms + mi);
            vs[1] *= ms / (ms + mi);
        }
        const double v = vs[0] * nx + vs[1] * ny;   // decomposition_velocity2D (:1346-1356)
        double vt[2] = {vs[0] - v * nx, vs[1] - v * ny};
        const double vn[2] = {v * nx, v * ny};
        if (form == 3) {
            const double mag = (1.0 - zeta) * 2.0 * mi * (dr - dp) / dt / dt;
            fn[0] = mag * nx; fn[1] = mag * ny;
        } else {
            fn[0] = mi * vn[0] / dt; fn[1] = mi * vn[1] / dt;
        }
        ft[0] = mi * vt[0] / dt; ft[1] = mi * vt[1] / dt;
        const double mag_fn = sqrt(fn[0] * fn[0] + fn[1] * fn[1]);
        const double mag_ft = sqrt(ft[0] * ft[0] + ft[1] * ft[1]);
        if (mag_ft > (mag_fn * myu)) {
            vt[0] = vt[0] * myu * mag_fn / mag_ft;
            vt[1] = vt[1] * myu * mag_fn / mag_ft;
            ft[0] = mi * vt[0] / dt; ft[1] = mi * vt[1] / dt;
        }
        double f1n[3], f2n[3], f1t[3], f2t[3];
        ss_interp_force(p1, p2, outp, fn, f1n, f2n);
        ss_interp_force(p1, p2, outp, ft, f1t, f2t);
        sid[0] = id1; sid[1] = id2;
        for (int k = 0; k < 3; k++) {
            con[0][k] = f1n[k]; con[0][3 + k] = f1t[k];
            con[1][k] = f2n[k]; con[1][3 + k] = f2t[k];
        }
    } else {
        const int id3 = ids[2];
        const SSPt p3 = ss_pt(d, id3);
        // cal_plane (:1063-1076) with clPlane()'s D = 1
        const double den = -p1.x * (p2.y * p3.z - p3.y * p2.z) - p2.x * (p3.y * p1.z - p1.y * p3.z) -
                           p3.x * (p1.y * p2.z - p2.y * p1.z);
        double A = p1.y * (p2.z - p3.z) + p2.y * (p3.z - p1.z) + p3.y * (p1.z - p2.z);
        double B = p1.z * (p2.x - p3.x) + p2.z * (p3.x - p1.x) + p3.z * (p1.x - p2.x);
        double C = p1.x * (p2.y - p3.y) + p2.x * (p3.y - p1.y) + p3.x * (p1.y - p2.y);
        A = A / den; B = B / den; C = C / den;
        const double D = 1.0;
        const double tmp0 = sqrt(A * A + B * B + C * C);
        const double dp = (tmp0 > 1.0e-3) ? fabs(A * p4.x + B * p4.y + C * p4.z + D) / tmp0 : 0.0;
        // cal_mappoint_plane (:1127-1160)
        const double tmp = sqrt(A * A + B * B + C * C);
        const SSPt P1 = {p4.x + dp * A / tmp, p4.y + dp * B / tmp, p4.z + dp * C / tmp};
        const SSPt P2 = {p4.x - dp * A / tmp, p4.y - dp * B / tmp, p4.z - dp * C / tmp};
        const double dp1 = (tmp0 > 1.0e-3) ? fabs(A * P1.x + B * P1.y + C * P1.z + D) / tmp0 : 0.0;
        const SSPt outp = (dp1 < 1.0e-3) ? P1 : P2;
        // check_ifinside_triangle (:1307-1344)
        const double a0[3] = {p3.x - p1.x, p3.y - p1.y, p3.z - p1.z};
        const double a1[3] = {p2.x - p1.x, p2.y - p1.y, p2.z - p1.z};
        const double a2[3] = {outp.x - p1.x, outp.y - p1.y, outp.z - p1.z};
        const double dot00 = a0[0] * a0[0] + a0[1] * a0[1] + a0[2] * a0[2];
        const double dot01 = a0[0] * a1[0] + a0[1] * a1[1] + a0[2] * a1[2];
        const double dot02 = a0[0] * a2[0] + a0[1] * a2[1] + a0[2] * a2[2];
        const double dot11 = a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2];
        const double dot12 = a1[0] * a2[0] + a1[1] * a2[1] + a1[2] * a2[2];
        const double inv = 1 / (dot00 * dot11 - dot01 * dot01);
        const double u = (dot11 * dot02 - dot01 * dot12) * inv;
        bool inside;
        if (u < 0 || u > 1) inside = false;
        else {
            const double v = (dot00 * dot12 - dot01 * dot02) * inv;
            inside = (v < 0 || v > 1) ? false : (u + v <= 1);
        }
        if (!(inside && dp < reach)) return;
        // clPlane::set_normal, check_ifoutward3D (:1272-1288)
        double nx = 0.0, ny = 0.0, nz = 0.0;
        const double tot = sqrt(A * A + B * B + C * C);
        if (tot > 1.0e-10) { nx = A / tot; ny = B / tot; nz = C / tot; }
        const double dot = (outp.x - p4.x) * nx + (outp.y - p4.y) * ny + (outp.z - p4.z) * nz;
        if (!(dot <= 0.0)) { nx = -nx; ny = -ny; nz = -nz; }
        // cal_line3D (:1078-1092) of (p1, p2) and (p3, outp); cal_intersect_lines3D (:1162-1185)
        const double d1 = sqrt((p2.x - p1.x) * (p2.x - p1.x) + (p2.y - p1.y) * (p2.y - p1.y) + (p2.z - p1.z) * (p2.z - p1.z));
        const double la = (p2.x - p1.x) / d1, lb = (p2.y - p1.y) / d1, lc = (p2.z - p1.z) / d1;
        const double d2 = sqrt((outp.x - p3.x) * (outp.x - p3.x) + (outp.y - p3.y) * (outp.y - p3.y) +
                               (outp.z - p3.z) * (outp.z - p3.z));
        const double ma = (outp.x - p3.x) / d2, mb = (outp.y - p3.y) / d2;
        const double flag = la * mb - ma * lb;
        if (!(fabs(flag) > 1.0e-3)) return;
        const double tu = ma * (p1.y - p3.y) - mb * (p1.x - p3.x);
        const double t = tu / flag;
        const SSPt sectp = {p1.x + la * t, p1.y + lb * t, p1.z + lc * t};
        double v3[3];
        for (int k = 0; k < 3; k++) v3[k] = d.s.vxp[(size_t)k * N + id3];
        double tms, tvs[3], ms, vs[3];
        ss_interp(p1, p2, sectp, d.s.mass[id1], d.s.mass[id2], v1, v2, &tms, tvs);
        ss_interp(p3, sectp, outp, d.s.mass[id3], tms, v3, tvs, &ms, vs);
        for (int k = 0; k < 3; k++) {
            vs[k] -= vpi[k];
            if (form != 1) vs[k] *= ms / (ms + mi);
        }
        const double v = vs[0] * nx + vs[1] * ny + vs[2] * nz;   // decomposition_velocity3D (:1358-1369)
        const double vn[3] = {v * nx, v * ny, v * nz};
        double vt[3] = {vs[0] - vn[0], vs[1] - vn[1], vs[2] - vn[2]};
        if (form == 3) {
            const double mag = (1.0 - zeta) * 2.0 * mi * (dr - dp) / dt / dt;
            fn[0] = mag * nx; fn[1] = mag * ny; fn[2] = mag * nz;
        } else {
            for (int k = 0; k < 3; k++) fn[k] = mi * vn[k] / dt;
        }
        for (int k = 0; k < 3; k++) ft[k] = mi * vt[k] / dt;
        const double mag_fn = sqrt(fn[0] * fn[0] + fn[1] * fn[1] + fn[2] * fn[2]);
        const double mag_ft = sqrt(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
        if (mag_ft > (mag_fn * myu)) {
            for (int k = 0; k < 3; k++) vt[k] = vt[k] * myu * mag_fn / mag_ft;
            for (int k = 0; k < 3; k++) ft[k] = mi * vt[k] / dt;
        }
        double f1n[3], f3n[3], f1t[3], f3t[3], g1n[3], g2n[3], g1t[3], g2t[3];
        ss_interp_force(p3, sectp, outp, fn, f1n, f3n);
        ss_interp_force(p3, sectp, outp, ft, f1t, f3t);
        ss_interp_force(p1, p2, sectp, f3n, g1n, g2n);
        ss_interp_force(p1, p2, sectp, f3t, g1t, g2t);
        // id3 takes + (f1n, f1t); id1 and id2 take - (g1, g2), as the reference applies them
        sid[0] = id3; sid[1] = id1; sid[2] = id2;
        for (int k = 0; k < 3; k++) {
            con[0][k] = f1n[k]; con[0][3 + k] = f1t[k];
            con[1][k] = -g1n[k]; con[1][3 + k] = -g1t[k];
            con[2][k] = -g2n[k]; con[2][3 + k] = -g2t[k];
        }
    }
    for (int q = 0; q < 3; q++) {
        d.s.ss_id[(size_t)q * N + i] = sid[q];
        if (sid[q] >= 0)
            for (int c = 0; c < 6; c++) d.s.ss_con[(size_t)(q * 6 + c) * N + i] = con[q][c];
    }
    for (int k = 0; k < 3; k++) {
        d.s.ss_own[(size_t)k * N + i] = fn[k];
        d.s.ss_own[(size_t)(3 + k) * N + i] = ft[k];
    }
}

// each structure particle's reactions, added in ascending order of the
// caller's indices of the particles they come from (x - y is x + (-y) in IEEE arithmetic, so the
// reference's "-=" reactions are stored negated and added)
__global__ void __launch_bounds__(128) k_ss_struct(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    if (d.s.type[i] != 4) return;
    const int nn = nbr_count(d, i);
    int src[SPH_NB_CAP], srco[SPH_NB_CAP], slot[SPH_NB_CAP];
    int m = 0;
    for (int q = 0; q < nn; q++) {
        const int j = d.s.nbr[(size_t)q * N + i];
        const int tj = d.s.type[j];
        if (!(tj == 1 || tj == 2)) continue;
        for (int s = 0; s < 3; s++)
            if (d.s.ss_id[(size_t)s * N + j] == i) {
                // insertion by source index in the caller's order
                const int jo = d.s.i2o[j];
                int p = m++;
                while (p > 0 && srco[p - 1] > jo) {
                    src[p] = src[p - 1]; srco[p] = srco[p - 1]; slot[p] = slot[p - 1]; p--;
                }
                src[p] = j;
                srco[p] = jo;
                slot[p] = s;
            }
    }
    double f[6] = {0, 0, 0, 0, 0, 0};
    for (int e = 0; e < m; e++)
        for (int c = 0; c < 6; c++) f[c] += d.s.ss_con[(size_t)(slot[e] * 6 + c) * N + src[e]];
    for (int c = 0; c < 6; c++) d.s.ss_fs[(size_t)c * N + i] = f[c];
}

// no_slip_tran / free_slip_tran (CPP_13-boundary.cpp:711-958, 960-1237): each
// wall particle's Shepard sums over its water, soil, air and structure
// neighbours give its stress per phase (soil with the pore terms) and its
// virtual velocity per phase: its own velocity minus the phase's mean velocity
// (no-slip), or plus the mean velocity with the component along the
// wall-particle line removed, from neighbours beyond 0.1 dr (free-slip).  The
// velocities are those after XSPH (and velocity_set_domain), before
// check_domain.
__global__ void __launch_bounds__(128) k_tran_wall(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    if (d.s.type[i] != 0) return;
    const bool free_slip = d.p.flbndy == 4 || d.p.flbndy == 14;
    const int nn = nbr_count(d, i);
    const Pos P = load_pos(d.s.xh, i);
    const double dr = d.p.dr;
    double us[4][6], uv[4][3], down[4];
    for (int p = 0; p < 4; p++) {
        for (int k = 0; k < 6; k++) us[p][k] = 0.0;
        for (int k = 0; k < 3; k++) uv[p][k] = 0.0;
        down[p] = 0.0;
    }
    for (int q = 0; q < nn; q++) {
        const int j = d.s.nbr[(size_t)q * N + i];
        const int tj = d.s.type[j];
        if (tj < 1 || tj > 4) continue;
        const int p = tj - 1;
        real wr[4];
        load_w(d, q, i, wr);
        const double w3 = wr[3], mj = d.s.mass[j], rj = d.s.rho[j];
        double sj[6], vj[3];
        for (int k = 0; k < 6; k++) sj[k] = d.s.sig_next[(size_t)k * N + j];
        for (int k = 0; k < 3; k++) vj[k] = d.s.vx_vb[(size_t)k * N + j];
        if (tj == 2) {
            const double satu = d.s.satu[j], pw = d.s.prew[j], pa = d.s.prea[j];
            for (int k = 0; k < 3; k++) us[p][k] = us[p][k] + mj * (sj[k] - satu * pw + (1 - satu) * pa) * w3 / rj;
            for (int k = 3; k < 6; k++) us[p][k] = us[p][k] + mj * sj[k] * w3 / rj;
        } else {
            for (int k = 0; k < 6; k++) us[p][k] = us[p][k] + mj * sj[k] * w3 / rj;
        }
        if (free_slip) {
            const Pos pj = load_pos(d.s.xh, j);
            const double v1[3] = {P.x - pj.x, P.y - pj.y, P.z - pj.z};
            const double dst = sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
            const double inprod = vj[0] * v1[0] + vj[1] * v1[1] + vj[2] * v1[2];
            if (dst > 0.1 * dr)
                for (int k = 0; k < 3; k++) uv[p][k] = uv[p][k] + mj * (vj[k] - inprod * v1[k] / dst / dst) * w3 / rj;
        } else {
            for (int k = 0; k < 3; k++) uv[p][k] = uv[p][k] + mj * vj[k] * w3 / rj;
        }
        down[p] = down[p] + mj * w3 / rj;
    }
    double its[3];
    for (int k = 0; k < 3; k++) its[k] = d.s.interfss[(size_t)k * N + i];
    for (int p = 0; p < 4; p++) {
        const bool some = fabs(down[p]) > 1.0e-6;
        for (int k = 0; k < 6; k++) d.s.sb[(size_t)(p * 6 + k) * N + i] = some ? us[p][k] / down[p] : 0.0;
        for (int k = 0; k < 3; k++)
            d.s.vb[(size_t)(p * 3 + k) * N + i] =
                some ? (free_slip ? its[k] + uv[p][k] / down[p] : its[k] - uv[p][k] / down[p]) : its[k];
    }
}

// boundary_free_solid (flbndy 5, CPP_13-boundary.cpp:1239-1516): the rigid
// contact of interaction_ss_rigid against the wall particles, with their
// interfss velocities, for the particle's own acceleration; types 1-4 in 2-D,
// every particle in 3-D (the reference's 3-D loop has no type test).  Stores
// zeta (f_t + f_n); k_accel_b divides by the mass after the damping.
template <int ND>
__global__ void __launch_bounds__(128) k_free_solid(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    d.s.fsol_on[i] = 0;
    const int ti = d.s.type[i];
    if (ND == 2 && !(ti >= 1 && ti <= 4)) return;
    const int nn = nbr_count(d, i);
    const double dt = step_dt(d), dr = d.p.dr, myu = d.p.ss_myu, zeta = d.p.ss_zeta;
    int ids[SPH_NB_CAP];
    double dsts[SPH_NB_CAP];
    int total = 0;
    const SSPt p4 = ss_pt(d, i);
    for (int q = 0; q < nn; q++) {
        const int j = d.s.nbr[(size_t)q * N + i];
        if (d.s.type[j] != 0) continue;
        const SSPt pj = ss_pt(d, j);
        const double dd = (p4.x - pj.x) * (p4.x - pj.x) + (p4.y - pj.y) * (p4.y - pj.y) + (p4.z - pj.z) * (p4.z - pj.z);
        ids[total] = j;
        dsts[total] = sqrt(dd);
        total++;
    }
    for (int a = 0; a < 4; a++)
        for (int b = a + 1; b < total; b++)
            if (dsts[a] > dsts[b]) { const int t = ids[a]; ids[a] = ids[b]; ids[b] = t; }
    if (total < ND) return;
    const double mi = d.s.mass[i];
    double vpi[3];
    for (int k = 0; k < 3; k++) vpi[k] = d.s.vxp[(size_t)k * N + i];
    const int id1 = ids[0], id2 = ids[1];
    const SSPt p1 = ss_pt(d, id1), p2 = ss_pt(d, id2);
    double v1[3], v2[3];
    for (int k = 0; k < 3; k++) { v1[k] = d.s.interfss[(size_t)k * N + id1]; v2[k] = d.s.interfss[(size_t)k * N + id2]; }
    double fn[3] = {0, 0, 0}, ft[3] = {0, 0, 0}, f[3];
    if (ND == 2) {
        const double den = p2.y * p1.x - p1.y * p2.x;
        const double A = (p1.y - p2.y) / den, B = (p2.x - p1.x) / den, C = 1.0;
        const double tmp0 = sqrt(A * A + B * B);
        const double dp = (tmp0 > 1.0e-3) ? fabs(A * p4.x + B * p4.y + C) / tmp0 : 0.0;
        const double tmp = sqrt(A * A + B * B);
        const SSPt Q1 = {p4.x + dp * A / tmp, p4.y + dp * B / tmp, 0.0}, Q2 = {p4.x - dp * A / tmp, p4.y - dp * B / tmp, 0.0};
        const double dq = (tmp0 > 1.0e-3) ? fabs(A * Q1.x + B * Q1.y + C) / tmp0 : 0.0;
        SSPt outp = (dq < 1.0e-3) ? Q1 : Q2;
        outp.z = 0.0;
        const double v0x = p2.x - p1.x, v0y = p2.y - p1.y, v0z = p2.z - p1.z;
        const double w1x = outp.x - p1.x, w1y = outp.y - p1.y, w1z = 0.0 - p1.z;
        const double dot00 = v0x * v0x + v0y * v0y + v0z * v0z, dot01 = v0x * w1x + v0y * w1y + v0z * w1z;
        const double u = 1.0 / dot00 * dot01;
        if ((u < 0 || u > 1) || !(dp < 0.5 * dr)) return;
        double nx = 0.0, ny = 0.0;
        const double tot = sqrt(A * A + B * B);
        if (tot > 1.0e-10) { nx = A / tot; ny = B / tot; }
        const double dot = (outp.x - p4.x) * nx + (outp.y - p4.y) * ny + 0.0 * 0.0;
        if (!(dot <= 0.0)) { nx = -nx; ny = -ny; }
        double ms, vs[3];
        ss_interp(p1, p2, outp, d.s.mass[id1], d.s.mass[id2], v1, v2, &ms, vs);
        vs[0] -= vpi[0];
        vs[1] -= vpi[1];
        const double v = vs[0] * nx + vs[1] * ny;
        const double vn[2] = {v * nx, v * ny};
        double vt[2] = {vs[0] - vn[0], vs[1] - vn[1]};
        fn[0] = mi * vn[0] / dt; fn[1] = mi * vn[1] / dt;
        ft[0] = mi * vt[0] / dt; ft[1] = mi * vt[1] / dt;
        const double mag_fn = sqrt(fn[0] * fn[0] + fn[1] * fn[1]), mag_ft = sqrt(ft[0] * ft[0] + ft[1] * ft[1]);
        if (mag_ft > (mag_fn * myu)) {
            vt[0] = vt[0] * myu * mag_fn / mag_ft;
            vt[1] = vt[1] * myu * mag_fn / mag_ft;
            ft[0] = mi * vt[0] / dt; ft[1] = mi * vt[1] / dt;
        }
        f[0] = zeta * (ft[0] + fn[0]);
        f[1] = zeta * (ft[1] + fn[1]);
        f[2] = 0.0;
    } else {
        const int id3 = ids[2];
        const SSPt p3 = ss_pt(d, id3);
        const double den = -p1.x * (p2.y * p3.z - p3.y * p2.z) - p2.x * (p3.y * p1.z - p1.y * p3.z) -
                           p3.x * (p1.y * p2.z - p2.y * p1.z);
        double A = p1.y * (p2.z - p3.z) + p2.y * (p3.z - p1.z) + p3.y * (p1.z - p2.z);
        double B = p1.z * (p2.x - p3.x) + p2.z * (p3.x - p1.x) + p3.z * (p1.x - p2.x);
        double C = p1.x * (p2.y - p3.y) + p2.x * (p3.y - p1.y) + p3.x * (p1.y - p2.y);
        A = A / den; B = B / den; C = C / den;
        const double D = 1.0;
        const double tmp0 = sqrt(A * A + B * B + C * C);
        const double dp = (tmp0 > 1.0e-3) ? fabs(A * p4.x + B * p4.y + C * p4.z + D) / tmp0 : 0.0;
        const double tmp = sqrt(A * A + B * B + C * C);
        const SSPt Q1 = {p4.x + dp * A / tmp, p4.y + dp * B / tmp, p4.z + dp * C / tmp};
        const SSPt Q2 = {p4.x - dp * A / tmp, p4.y - dp * B / tmp, p4.z - dp * C / tmp};
        const double dq = (tmp0 > 1.0e-3) ? fabs(A * Q1.x + B * Q1.y + C * Q1.z + D) / tmp0 : 0.0;
        const SSPt outp = (dq < 1.0e-3) ? Q1 : Q2;
        const double a0[3] = {p3.x - p1.x, p3.y - p1.y, p3.z - p1.z};
        const double a1[3] = {p2.x - p1.x, p2.y - p1.y, p2.z - p1.z};
        const double a2[3] = {outp.x - p1.x, outp.y - p1.y, outp.z - p1.z};
        const double dot00 = a0[0] * a0[0] + a0[1] * a0[1] + a0[2] * a0[2];
        const double dot01 = a0[0] * a1[0] + a0[1] * a1[1] + a0[2] * a1[2];
        const double dot02 = a0[0] * a2[0] + a0[1] * a2[1] + a0[2] * a2[2];
        const double dot11 = a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2];
        const double dot12 = a1[0] * a2[0] + a1[1] * a2[1] + a1[2] * a2[2];
        const double inv = 1 / (dot00 * dot11 - dot01 * dot01);
        const double u = (dot11 * dot02 - dot01 * dot12) * inv;
        bool inside;
        if (u < 0 || u > 1) inside = false;
        else {
            const double v = (dot00 * dot12 - dot01 * dot02) * inv;
            inside = (v < 0 || v > 1) ? false : (u + v <= 1);
        }
        if (!(inside && dp < 0.5 * dr)) return;
        double nx = 0.0, ny = 0.0, nz = 0.0;
        const double tot = sqrt(A * A + B * B + C * C);
        if (tot > 1.0e-10) { nx = A / tot; ny = B / tot; nz = C / tot; }
        const double dot = (outp.x - p4.x) * nx + (outp.y - p4.y) * ny + (outp.z - p4.z) * nz;
        if (!(dot <= 0.0)) { nx = -nx; ny = -ny; nz = -nz; }
        const double d1 = sqrt((p2.x - p1.x) * (p2.x - p1.x) + (p2.y - p1.y) * (p2.y - p1.y) + (p2.z - p1.z) * (p2.z - p1.z));
        const double la = (p2.x - p1.x) / d1, lb = (p2.y - p1.y) / d1, lc = (p2.z - p1.z) / d1;
        const double d2 = sqrt((outp.x - p3.x) * (outp.x - p3.x) + (outp.y - p3.y) * (outp.y - p3.y) +
                               (outp.z - p3.z) * (outp.z - p3.z));
        const double ma = (outp.x - p3.x) / d2, mb = (outp.y - p3.y) / d2;
        const double flag = la * mb - ma * lb;
        if (!(fabs(flag) > 1.0e-3)) return;
        const double tu = ma * (p1.y - p3.y) - mb * (p1.x - p3.x);
        const double t = tu / flag;
        const SSPt sectp = {p1.x + la * t, p1.y + lb * t, p1.z + lc * t};
        double v3[3];
        for (int k = 0; k < 3; k++) v3[k] = d.s.interfss[(size_t)k * N + id3];
        double tms, tvs[3], ms, vs[3];
        ss_interp(p1, p2, sectp, d.s.mass[id1], d.s.mass[id2], v1, v2, &tms, tvs);
        ss_interp(p3, sectp, outp, d.s.mass[id3], tms, v3, tvs, &ms, vs);
        for (int k = 0; k < 3; k++) vs[k] -= vpi[k];
        const double v = vs[0] * nx + vs[1] * ny + vs[2] * nz;
        const double vn[3] = {v * nx, v * ny, v * nz};
        double vt[3] = {vs[0] - vn[0], vs[1] - vn[1], vs[2] - vn[2]};
        for (int k = 0; k < 3; k++) { fn[k] = mi * vn[k] / dt; ft[k] = mi * vt[k] / dt; }
        const double mag_fn = sqrt(fn[0] * fn[0] + fn[1] * fn[1] + fn[2] * fn[2]);
        const double mag_ft = sqrt(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
        if (mag_ft > (mag_fn * myu)) {
            for (int k = 0; k < 3; k++) vt[k] = vt[k] * myu * mag_fn / mag_ft;
            for (int k = 0; k < 3; k++) ft[k] = mi * vt[k] / dt;
        }
        for (int k = 0; k < 3; k++) f[k] = zeta * (ft[k] + fn[k]);
    }
    for (int k = 0; k < 3; k++) d.s.fsol[(size_t)k * N + i] = f[k];
    d.s.fsol_on[i] = 1;
}

// coupled_Water_Soil_Structure (ss acc_type 2, CPP_9-4-derivation_stress.cpp:
// 507-629): the stress divergence between structure and soil / water pairs
// with plain stresses (a water particle with a structure neighbour takes the
// difference form); k_accel_b adds each row sum after the wall stress.
__global__ void __launch_bounds__(128) k_coupled(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    const int ti = d.s.type[i];
    if (!(ti == 4 || ti == 2 || ti == 1)) return;
    const int nn = nbr_count(d, i);
    double si[6];
    for (int k = 0; k < 6; k++) si[k] = d.s.sig_next[(size_t)k * N + i];
    const double ri = d.s.rho[i];
    double tu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int q = 0; q < nn; q++) {
        const int j = d.s.nbr[(size_t)q * N + i];
        const int tj = d.s.type[j];
        const bool plus = (ti == 4 && tj == 2) || (ti == 2 && tj == 4) || (ti == 4 && tj == 1);
        const bool minus = (ti == 1 && tj == 4);
        if (!(plus || minus)) continue;
        real wr[4];
        load_w(d, q, i, wr);
        const double w[3] = {wr[0], wr[1], wr[2]};
        const double mj = d.s.mass[j], rj = d.s.rho[j];
        double sj[6], a[6], b[6];
        for (int k = 0; k < 6; k++) sj[k] = d.s.sig_next[(size_t)k * N + j];
        for (int k = 0; k < 6; k++) { a[k] = sj[k] / rj / rj; b[k] = si[k] / ri / ri; }
        const int cmap[3][3] = {{0, 3, 5}, {3, 1, 4}, {5, 4, 2}};
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) {
                const int m = cmap[r][c];
                tu[r][c] = tu[r][c] + mj * (plus ? a[m] + b[m] : a[m] - b[m]) * w[c];
            }
    }
    for (int r = 0; r < 3; r++) d.s.cpl[(size_t)r * N + i] = tu[r][0] + tu[r][1] + tu[r][2];
}

__global__ void k_step_done(Dev d)
{
    if (threadIdx.x == 0 && blockIdx.x == 0 && *d.s.err == 0) {
        *d.s.step += 1;
        *d.s.tsim = *d.s.tsim + step_dt(d);     // t = t + dt (CPP_1-SPHLoops.cpp:485)
        if (d.p.cfl_on) {
            // the next step's dt: the reduced limit, capped at the input dt;
            // the running minimum starts again from +inf
            const double lim = __longlong_as_double((long long)*d.s.dtmin);
            *d.s.dtv = (lim < d.p.dt) ? lim : d.p.dt;
            *d.s.dtmin = 0x7ff0000000000000ULL;      // +inf
        }
    }
}

// partidel (CPP_15-2-partidel.cpp:19-58), after the update: water within dr
// of 7 dr past either x end of the domain box (of its instance) and above
// y = 0.12 stops and leaves the calculation as type 7
__global__ void __launch_bounds__(256) k_partidel(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    if (d.s.type[i] != 1) return;
    const CellGrid g = cell_grid(d, i);
    const Pos p = load_pos(d.s.xh_next, i);
    const double dr = d.p.dr;
    const double dx1 = fabs(p.x - g.xmax - 7.0 * dr);
    const double dx2 = fabs(p.x - g.xmin + 7.0 * dr);
    const double dy1 = p.y - 0.12;
    if ((dx1 < dr || dx2 < dr) && dy1 > 0.0) {
        d.s.type[i] = 7;
        for (int c = 0; c < 3; c++) {
            d.s.vxp[c * N + i] = 0.0;
            d.s.vx[c * N + i] = 0.0;
            d.s.ax[c * N + i] = 0.0;
        }
    }
}

// Adaptive time step (an extension: the reference keeps dt constant,
// CPP_12-2-dt.cpp:13-20).  For every water, soil, air and structure particle
// after the update, the CFL limit cfl_c h / (c + |v|), c the sound speed of
// its material (Para_Fluid / Para_Soil / Para_Structure::vpu), and the force
// limit cfl_f sqrt(h / |a|); their minimum over the particles, reduced with
// warp shuffles and one 64-bit atomicMin per warp on the bits of the positive
// double (which order as the values do), becomes the next step's dt in
// k_step_done.  Off (not launched) unless sphgpu_set_cfl turns it on.
__global__ void __launch_bounds__(256) k_cfl(Dev d)
{
    const int N = d.p.N, nd = d.p.ndim;
    if (*d.s.err) return;
    double m = __longlong_as_double(0x7ff0000000000000LL);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int t = d.s.type[i];
        if (t < 1 || t > 4) continue;
        const double c = (t == 1 || t == 3) ? d.s.f_vpu[i] : (t == 2) ? d.s.s_vpu[i] : d.p.st_vpu;
        double v2 = 0.0, a2 = 0.0;
        for (int k = 0; k < nd; k++) {
            const double v = d.s.vxp[k * N + i], a = d.s.axp[k * N + i];
            v2 = v2 + v * v;
            a2 = a2 + a * a;
        }
        const double h = load_pos(d.s.xh, i).h;
        double lim = d.p.cfl_c * (h / (c + sqrt(v2)));
        if (a2 > 0.0) {
            const double lf = d.p.cfl_f * sqrt(h / sqrt(a2));
            if (lf < lim) lim = lf;
        }
        if (lim < m) m = lim;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double q = __shfl_xor_sync(0xffffffffu, m, o);
        if (q < m) m = q;
    }
    if ((threadIdx.x & 31) == 0 && m > 0.0)
        atomicMin(d.s.dtmin, (unsigned long long)__double_as_longlong(m));
}

// kernel_gradient_correction (CPP_3-NNPS.cpp:376-496): the inverse of
// L = sum_j m_j / rho_j (x_j - x_i) (x) grad W_ij over same-phase, wall and
// soil/structure neighbours of each soil (type 2) or structure (type 4)
// particle, inverted as inverse_mat_2D / inverse_mat_3D do (:499-558), then
// applied in place to the gradients of all the particle's pair records in
// mat_multiply's order (:85-90), as the reference rewrites wij.  Uses the
// densities of the previous step, as the reference does (it runs before
// density()).  In the bulk form L is formed in FP64 from the FP32 records.
template <int ND, typename R>
__device__ __forceinline__ void kgc_particle(const Dev& d, int i)
{
    const int N = d.p.N;
    const int ti = d.s.type[i];
    const int nn = nbr_count(d, i);
    const Pos P = load_pos(d.s.xh, i);
    const double xi[3] = {P.x, P.y, P.z};
    double L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int q = 0; q < nn; q++) {
        const int j = d.s.nbr[(size_t)q * N + i];
        const int tj = d.s.type[j];
        const bool take = (ti == 2 && (tj == 2 || tj == 0 || tj == 4)) || (ti == 4 && (tj == 4 || tj == 0 || tj == 2));
        if (!take) continue;
        const Pos pj = load_pos(d.s.xh, j);
        const double xj[3] = {pj.x, pj.y, pj.z};
        R wr[4];
        load_w(d, q, i, wr);
        const double w[3] = {wr[0], wr[1], wr[2]};
        const double mr = d.s.mass[j] / d.s.rho[j];
        double xij[3];
        for (int k = 0; k < ND; k++) xij[k] = xj[k] - xi[k];
        for (int a = 0; a < ND; a++)
            for (int b = 0; b < ND; b++) L[a][b] = L[a][b] + mr * xij[a] * w[b];
    }
    double B[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (ND == 2) {
        const double det = L[0][0] * L[1][1] - L[0][1] * L[1][0];
        if (fabs(det) > 1.0e-5) {
            B[0][0] = L[1][1] / det; B[0][1] = -L[0][1] / det;
            B[1][0] = -L[1][0] / det; B[1][1] = L[0][0] / det;
        } else {
            B[0][0] = 1.0; B[1][1] = 1.0;
        }
    } else {
        const double det = L[0][0] * (L[1][1] * L[2][2] - L[1][2] * L[2][1]) - L[1][0] * (L[0][1] * L[2][2] - L[0][2] * L[2][1])
            + L[2][0] * (L[0][1] * L[1][2] - L[0][2] * L[1][1]);
        if (fabs(det) > 1.0e-5) {
            B[0][0] = (L[1][1] * L[2][2] - L[1][2] * L[2][1]) / det;
            B[0][1] = (L[0][2] * L[2][1] - L[0][1] * L[2][2]) / det;
            B[0][2] = (L[0][1] * L[1][2] - L[0][2] * L[1][1]) / det;
            B[1][0] = (L[1][2] * L[2][0] - L[1][0] * L[2][2]) / det;
            B[1][1] = (L[0][0] * L[2][2] - L[0][2] * L[2][0]) / det;
            B[1][2] = (L[1][0] * L[0][2] - L[0][0] * L[1][2]) / det;
            B[2][0] = (L[1][0] * L[2][1] - L[1][1] * L[2][0]) / det;
            B[2][1] = (L[0][1] * L[2][0] - L[0][0] * L[2][1]) / det;
            B[2][2] = (L[0][0] * L[1][1] - L[1][0] * L[0][1]) / det;
        } else {
            B[0][0] = 1.0; B[1][1] = 1.0; B[2][2] = 1.0;
        }
    }
    R a[9];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) a[r * 3 + c] = (R)B[r][c];
    for (int q = 0; q < nn; q++) {
        R w[4];
        load_w(d, q, i, w);
        const R c0 = a[0] * w[0] + a[1] * w[1] + a[2] * w[2];
        const R c1 = a[3] * w[0] + a[4] * w[1] + a[5] * w[2];
        const R c2 = a[6] * w[0] + a[7] * w[1] + a[8] * w[2];
        w[0] = c0; w[1] = c1; w[2] = c2;
        store_w(d, q, i, w);
    }
}

template <int ND>
__global__ void __launch_bounds__(128, SPH_MINB) k_kgc(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    const int ti = d.s.type[i];
    if (!(ti == 2 || ti == 4)) return;
    if (d.p.bulk) kgc_particle<ND, float>(d, i);
    else kgc_particle<ND, double>(d, i);
}

// strain_regu / stress_regu (CPP_7-2-constitutive.cpp:385-450) in Jacobi
// order: on steps with l % step_regu == 0, dst = the same-phase Shepard
// average of src; otherwise dst = src.  For the strain, the values read are
// those after strain_noreg's reset at l == inip (zero_at_inip).
template <int ND>
__global__ void __launch_bounds__(128, SPH_MINB) k_regu(Dev d, const double* src, double* dst, int zero_at_inip)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    const int l = *d.s.step;
    const bool zero = zero_at_inip && l == d.p.inip;
    if (l % d.p.step_regu != 0) {
        for (int k = 0; k < 6; k++) dst[(size_t)k * N + i] = zero ? 0.0 : src[(size_t)k * N + i];
        return;
    }
    const int ti = d.s.type[i], nn = nbr_count(d, i);
    double up[6] = {0, 0, 0, 0, 0, 0}, down = 0.0;
    for (int q = 0; q < nn; q++) {
        const int j = d.s.nbr[(size_t)q * N + i];
        if (d.s.type[j] != ti) continue;
        real wr[4];
        load_w(d, q, i, wr);
        const double w3 = wr[3];
        const double mr = d.s.mass[j] / d.s.rho[j];
        for (int k = 0; k < 6; k++) up[k] = up[k] + mr * w3 * (zero ? 0.0 : src[(size_t)k * N + j]);
        down = down + mr * w3;
    }
    for (int k = 0; k < 6; k++)
        dst[(size_t)k * N + i] = (fabs(down) > 1.0e-6) ? up[k] / down : (zero ? 0.0 : src[(size_t)k * N + i]);
}

}  // namespace SPH_NS

// ---------------------------------------------------------------------------
// host-side launch sequences (enqueued on `st`, capturable into a graph)
using namespace SPH_NS;

static inline unsigned nblk(long n, int b) { return (unsigned)((n + b - 1) / b); }

// threads per block of a tuned pass (128 unless the autotuner chose another
// multiple of 32)
static inline int tbk(const Dev& d, int pass)
{
    const int b = d.p.tb[pass];
    return (b >= 32 && b <= 128 && b % 32 == 0) ? b : 128;
}

#define REC(k) do { if (ev) cudaEventRecord(ev[k], st); } while (0)

#ifndef SPH_BULK32
extern "C" size_t sphk_sort_temp_bytes(int N, int end_bit)
{
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const int*)nullptr, (int*)nullptr, N, 0, end_bit);
    return bytes;
}

// The order sphgpu_set_reorder re-sorts the particle state into: by type
// and material (so that a warp's particles take the same branches of the
// constitutive and momentum passes: co-located phases, such as the water
// and soil particles of a saturated soil, would otherwise alternate), then
// by place on a lattice of spacing dr over the particle's grid (each batched
// instance's own grid, the instances one after another), in rows along the
// grid's longest axis, planes across its shortest.  On a regular arrangement
// the neighbours at one lattice offset from consecutive particles then sit at
// consecutive positions, so the gathers of one list slot by a warp read one
// contiguous run of records, and long rows keep the warps that straddle two
// rows few.  Lattice places are clamped to the grid, so the place key of a
// particle in instance q stays below 8 times the context cell id of instance
// q + 1, and below span = 8 (ctotal + 1) for all.
__global__ void k_order_key(Dev d, unsigned long long span, unsigned long long* key, int* val)
{
    const int i = IDX, N = d.p.N;
    if (i >= N) return;
    const Pos p = load_pos(d.s.xh, i);
    const CellGrid g = cell_grid(d, i);
    const double dr = d.p.dr;
    auto lat = [dr](double x, double lo, int cells) -> unsigned long long {
        const double t = fabs(x - lo) / dr;
        const int n = 2 * cells;
        return (t < (double)n) ? (unsigned long long)t : (unsigned long long)(n - 1);
    };
    const int nd = d.p.ndim;
    const unsigned long long q[3] = {lat(p.x, g.xmin, g.cxm), lat(p.y, g.ymin, g.cym),
                                     nd == 3 ? lat(p.z, g.zmin, g.czm) : 0ull};
    const unsigned long long n[3] = {2ull * g.cxm, 2ull * g.cym, nd == 3 ? 2ull * g.czm : 1ull};
    // axes by extent, longest last (the fastest); ties keep x fastest
    int a[3] = {2, 1, 0};
    for (int u = 0; u < 3; u++)
        for (int v = u + 1; v < 3; v++)
            if (n[a[u]] > n[a[v]]) { const int w = a[u]; a[u] = a[v]; a[v] = w; }
    const unsigned long long k = (q[a[0]] * n[a[1]] + q[a[1]]) * n[a[2]] + q[a[2]];
    const int t = d.s.type[i], m = d.s.matype[i];
    const unsigned long long group = (unsigned long long)((t >= 0 && t < 8) ? t : 7) * 64ull +
                                     (unsigned long long)((m >= 0 && m < 64) ? m : 63);
    key[i] = group * span + 8ull * (unsigned long long)g.base + k;
    val[i] = i;
}

extern "C" size_t sphk_order_temp_bytes(int N, int end_bit)
{
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned long long*)nullptr,
                                    (unsigned long long*)nullptr, (const int*)nullptr, (int*)nullptr, N, 0,
                                    end_bit);
    return bytes;
}

// the re-sort's permutation into vout (vout[i] = the held index that moves
// to i), from the positions of the buffers of *dp; returns the kernels it
// launched
extern "C" int sphk_order_sort(const Dev* dp, void* tmp, size_t bytes, int end_bit, unsigned long long* kin,
                               unsigned long long* kout, int* vin, int* vout, cudaStream_t st)
{
    const Dev& d = *dp;
    const int N = d.p.N;
    const unsigned long long span = 8ull * ((unsigned long long)d.p.ctotal + 1);
    k_order_key<<<nblk(N, 256), 256, 0, st>>>(d, span, kin, vin);
    cub::DeviceRadixSort::SortPairs(tmp, bytes, kin, kout, vin, vout, N, 0, end_bit, st);
    return 1;
}

// Stage names, in launch order; with `ev` non-null, event ev[k] is recorded
// before stage k and ev[SPHK_NSTAGES] after the last one (stages a run does
// not need are recorded with no work between their events).
extern "C" const char* const sphk_stage_names[] = {
    "k_cellkey", "radix_sort", "k_cellreset", "k_cellrange", "k_nnps", "k_nnps_resolve", "k_pairw", "k_kgc",
    "k_density", "k_shepard_eos", "k_strain", "k_regu_eps", "k_stress", "k_regu_sig", "k_stress_2",
    "k_art_rij", "k_accel_a", "k_accel_b", "k_xsph_update", "k_tm_boundary", "k_step_done"};
static_assert(sizeof(sphk_stage_names) / sizeof(sphk_stage_names[0]) == SPHK_NSTAGES, "stage table");
#endif  // !SPH_BULK32

// launch K<ND> for the run's dimension
#define LAUNCH_ND(K, blocks, threads, ...)                                          \
    do {                                                                           \
        if (d.p.ndim == 2) K<2><<<blocks, threads, 0, st>>>(__VA_ARGS__);          \
        else K<3><<<blocks, threads, 0, st>>>(__VA_ARGS__);                        \
    } while (0)
#ifndef SPH_BULK32
// the NNPS stage (+ kernel gradient correction) as three parts, selected by
// the bits of `parts`: 1 parttocell (cell keys, the sort, cell ranges),
// 2 partisearching (the search and the pair records), 4 the kernel gradient
// correction; returns the number of this library's kernels it launched
#if SPHGPU_CHECK
// The bounds-checked build (SPHGPU_CHECK=1): after the search, every index the
// later passes take from it is checked -- each list slot holds a particle
// other than i within [0, N), the slot masks mark exactly the slots of their
// type, the sorted order is a permutation and the cell ranges stay within the
// sorted positions.  A violation sets the error word to SPH_ERR_CHECK (the
// passes after it then return at once) instead of trapping.
__global__ void k_check_lists(Dev d)
{
    const int i = IDX, N = d.p.N;
    if (i >= N || *d.s.err) return;
    bool bad = false;
    const int nn = nbr_count(d, i);
    if (nn < 0 || nn > SPH_NB_CAP) bad = true;
    const int q = d.s.sortpos[i];
    if (q < 0 || q >= N || d.s.pid_sorted[q] != i) bad = true;
    for (int s = 0; s < nn && !bad; s++) {
        const int j = d.s.nbr[(size_t)s * N + i];
        if (j < 0 || j >= N || j == i) { bad = true; break; }
        const int tj = d.s.type[j];
        for (int t = 0; t <= 4; t++) {
            const SlotMask m = type_mask(d, i, t);
            if (m.has(s) != (tj == t)) bad = true;
        }
    }
    const int c = d.s.cell[i];
    if (c >= 0 && c < d.p.ctotal + 4) {
        const int a = d.s.cstart[c], b = d.s.cend[c];
        if (a <= b && (a < 0 || b >= N)) bad = true;
    }
    if (bad) atomicCAS(d.s.err, 0, SPH_ERR_CHECK);
}
#endif

extern "C" int sphk_enqueue_nnps_parts(const Dev* dp, void* sort_tmp, size_t sort_bytes, int end_bit,
                                       cudaStream_t st, cudaEvent_t* ev, int parts)
{
    const Dev& d = *dp;
    const int N = d.p.N;
    int n = 0;
    if (parts & 1) {
        REC(0);
        if (d.p.flr) { LAUNCH_ND(k_rain, 1, 256, d); n++; }
        LAUNCH_ND(k_cellkey, nblk(N, 256), 256, d); n++;
        REC(1);
        size_t bytes = sort_bytes;
        cub::DeviceRadixSort::SortPairs(sort_tmp, bytes, d.s.key_in, d.s.key_out, d.s.val_in, d.s.pid_sorted,
                                        N, 0, end_bit, st);
        REC(2);
        k_cellreset<<<nblk(d.p.ctotal, 256), 256, 0, st>>>(d); n++;
        REC(3);
        k_cellrange<<<nblk(N, 256), 256, 0, st>>>(d); n++;
    }
    if (parts & 2) {
        REC(4);
        LAUNCH_ND(k_nnps, nblk(N, tbk(d, TP_NNPS)), tbk(d, TP_NNPS), d); n++;
        REC(5);
        LAUNCH_ND(k_nnps_resolve, nblk(N, tbk(d, TP_RESOLVE)), tbk(d, TP_RESOLVE), d); n++;
        REC(6);
#if SPHGPU_CHECK
        k_check_lists<<<nblk(N, 128), 128, 0, st>>>(d); n++;
#endif
        LAUNCH_ND(k_pairw, nblk(N, tbk(d, TP_PAIRW)), tbk(d, TP_PAIRW), d); n++;
    }
    if (parts & 4) {
        REC(7);
        if (d.p.flknl > 2) { LAUNCH_ND(k_kgc, nblk(N, 128), 128, d); n++; }
    }
    return n;
}

extern "C" int sphk_enqueue_nnps(const Dev* dp, void* sort_tmp, size_t sort_bytes, int end_bit, cudaStream_t st,
                                 cudaEvent_t* ev)
{
    return sphk_enqueue_nnps_parts(dp, sort_tmp, sort_bytes, end_bit, st, ev, 7);
}
#endif  // !SPH_BULK32

// the rest of the step; `regu` includes the strain/stress regularisation
// passes (which act on steps l with l % step_regu == 0).  The FP32-bulk build
// exports it as sphk_enqueue_physics_bulk32.
extern "C" int SPHK_ENTRY(sphk_enqueue_physics)(const Dev* dp, cudaStream_t st, cudaEvent_t* ev, int regu)
{
    Dev d = *dp;
    d.s.eps_in = regu ? d.s.eps_tmp : d.s.eps;
    const int N = d.p.N;
    int n = 0;
    REC(8);
    LAUNCH_ND(k_density, nblk(N, tbk(d, TP_DENSITY)), tbk(d, TP_DENSITY), d); n++;
    REC(9);
    LAUNCH_ND(k_shepard_eos, nblk(N, tbk(d, TP_SHEPARD)), tbk(d, TP_SHEPARD), d); n++;
    REC(10);
    LAUNCH_ND(k_strain, nblk(N, tbk(d, TP_STRAIN)), tbk(d, TP_STRAIN), d); n++;
    if (d.p.flagum == 1) { k_saturation<<<nblk(N, 128), 128, 0, st>>>(d); n++; }
    REC(11);
    if (regu) { LAUNCH_ND(k_regu, nblk(N, 128), 128, d, d.s.eps, d.s.eps_tmp, 1); n++; }
    REC(12);
    if (regu) {
        if (d.p.ndim == 2) k_stress<2, 1><<<nblk(N, tbk(d, TP_STRESS)), tbk(d, TP_STRESS), 0, st>>>(d);
        else k_stress<3, 1><<<nblk(N, tbk(d, TP_STRESS)), tbk(d, TP_STRESS), 0, st>>>(d);
    } else {
        if (d.p.ndim == 2) k_stress<2, 0><<<nblk(N, tbk(d, TP_STRESS)), tbk(d, TP_STRESS), 0, st>>>(d);
        else k_stress<3, 0><<<nblk(N, tbk(d, TP_STRESS)), tbk(d, TP_STRESS), 0, st>>>(d);
    }
    n++;
    REC(13);
    if (regu) { LAUNCH_ND(k_regu, nblk(N, 128), 128, d, d.s.sig_next, d.s.sig_tmp, 0); n++; }
    REC(14);
    if (regu) {
        if (d.p.ndim == 2) k_stress<2, 2><<<nblk(N, tbk(d, TP_STRESS)), tbk(d, TP_STRESS), 0, st>>>(d);
        else k_stress<3, 2><<<nblk(N, tbk(d, TP_STRESS)), tbk(d, TP_STRESS), 0, st>>>(d);
        n++;
    }
    REC(15);
    const bool art = d.p.art_stre_coe > 0.0;
    if (art) { LAUNCH_ND(k_art_rij, nblk(N, 128), 128, d); n++; }
    REC(16);
    LAUNCH_ND(k_accel_a, nblk(N, tbk(d, TP_ACCEL_A)), tbk(d, TP_ACCEL_A), d); n++;
    if (d.p.flbndy == 5) { LAUNCH_ND(k_free_solid, nblk(N, 128), 128, d); n++; }
    if (d.p.ss_coupled) { k_coupled<<<nblk(N, 128), 128, 0, st>>>(d); n++; }
    if (d.p.ss_type >= 1) {
        LAUNCH_ND(k_ss_pair, nblk(N, 128), 128, d); n++;
        k_ss_struct<<<nblk(N, 128), 128, 0, st>>>(d); n++;
    }
    REC(17);
    {
        const bool drag = d.p.fli > 1, vib = d.p.flv != 0;
        const dim3 g(nblk(N, tbk(d, TP_ACCEL_B))), b(tbk(d, TP_ACCEL_B));
        if (d.p.ndim == 2) {
            if (vib) k_accel_b<2, 0, 0, 1><<<g, b, 0, st>>>(d);
            else k_accel_b<2, 0, 0><<<g, b, 0, st>>>(d);
            if (drag) k_accel_b<2, 1, 1><<<g, b, 0, st>>>(d);
            else k_accel_b<2, 0, 1><<<g, b, 0, st>>>(d);
            if (vib) {
                if (art) k_accel_b_tail<2, 1, 1><<<g, b, 0, st>>>(d);
                else k_accel_b_tail<2, 0, 1><<<g, b, 0, st>>>(d);
            } else {
                if (art) k_accel_b_tail<2, 1><<<g, b, 0, st>>>(d);
                else k_accel_b_tail<2, 0><<<g, b, 0, st>>>(d);
            }
        } else {
            if (vib) k_accel_b<3, 0, 0, 1><<<g, b, 0, st>>>(d);
            else k_accel_b<3, 0, 0><<<g, b, 0, st>>>(d);
            if (drag) k_accel_b<3, 1, 1><<<g, b, 0, st>>>(d);
            else k_accel_b<3, 0, 1><<<g, b, 0, st>>>(d);
            if (vib) {
                if (art) k_accel_b_tail<3, 1, 1><<<g, b, 0, st>>>(d);
                else k_accel_b_tail<3, 0, 1><<<g, b, 0, st>>>(d);
            } else {
                if (art) k_accel_b_tail<3, 1><<<g, b, 0, st>>>(d);
                else k_accel_b_tail<3, 0><<<g, b, 0, st>>>(d);
            }
        }
    }
    n += 3;
    REC(18);
    LAUNCH_ND(k_xsph_update, nblk(N, tbk(d, TP_XSPH)), tbk(d, TP_XSPH), d); n++;
    REC(19);
    if (d.p.flbndy == 2) {
        LAUNCH_ND(k_tm_vb, nblk(N, 128), 128, d); n++;
        k_tm_wall<<<nblk(N, 128), 128, 0, st>>>(d); n++;
    } else if (d.p.flbndy == 3 || d.p.flbndy == 4 || d.p.flbndy == 13 || d.p.flbndy == 14) {
        k_tran_wall<<<nblk(N, 128), 128, 0, st>>>(d); n++;
    }
    if (d.p.flr) { k_partidel<<<nblk(N, 256), 256, 0, st>>>(d); n++; }
    if (d.p.cfl_on) { k_cfl<<<148 * 8, 256, 0, st>>>(d); n++; }
    REC(20);
    k_step_done<<<1, 32, 0, st>>>(d); n++;
    REC(21);
    return n;
}
