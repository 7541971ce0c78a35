// sph_noalloc.cu -- the neighbour search for callers that cannot allocate
// device memory.
//
// Some callers cannot call cudaMalloc at the point where they need neighbour
// lists: code running under a memory pool or budget that forbids new device
// allocations, a real-time loop that must not enter the driver's allocator,
// or a host application that owns all its device buffers and only lends
// pointers to libraries.  sphgpu_nnps_noalloc serves them: the caller passes
// device pointers for the inputs (positions, smoothing lengths, types) and
// the outputs (neighbour counts and lists in the Par_Cell layout), and every
// intermediate the search needs (cell keys, the radix sort's buffers and
// temporary storage, cell ranges, the cell-sorted positions) lives in one
// file-scope __device__ array of fixed size, g_nnps_scratch below.
//
// The array exists once per GPU that loads this library and stays allocated
// until the process exits.  Its device address is looked up once per device,
// with that device current, by the first call made on it, and kept for the
// rest of the process; that first call should therefore be made before any
// stream capture, and a process that resets a device (cudaDeviceReset, which
// discards the module and so the array) must not call the search on that
// device again.  Each call waits for its own stream to read its status, so it
// is synchronous and cannot be captured into a graph.  Every call on a
// device uses the same array and it keeps the previous call's contents: each
// call clears the words that must start at zero (the error word and the cell
// ranges) itself.  Calls that overlap on the GPU (on different streams, or
// from different host threads without ordering) race on the array and must
// not be issued.
//
// The neighbour order and the inclusion test are those of partisearching
// (CPP_3-NNPS.cpp:265-374), as in the context-based engine.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/sphgpu.h"
#include "sph_device.cuh"

namespace {

constexpr int kMaxN = SPHGPU_NOALLOC_MAX_PARTICLES;
constexpr int kMaxCells = SPHGPU_NOALLOC_MAX_CELLS;
// sort temporary storage reserved for kMaxN keys (CUB's onesweep needs far
// less; checked against the exact requirement at set-up)
constexpr size_t kSortBytes = size_t(1) << 20;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffErr = 0;
constexpr size_t kOffKeyIn = align256(kOffErr + 16);
constexpr size_t kOffKeyOut = align256(kOffKeyIn + 4ull * kMaxN);
constexpr size_t kOffValIn = align256(kOffKeyOut + 4ull * kMaxN);
constexpr size_t kOffValOut = align256(kOffValIn + 4ull * kMaxN);
constexpr size_t kOffCell = align256(kOffValOut + 4ull * kMaxN);
constexpr size_t kOffXs = align256(kOffCell + 4ull * kMaxN);
constexpr size_t kOffStart = align256(kOffXs + 32ull * kMaxN);
constexpr size_t kOffEnd = align256(kOffStart + 4ull * (kMaxCells + 4));
constexpr size_t kOffSort = align256(kOffEnd + 4ull * (kMaxCells + 4));
constexpr size_t kScratchBytes = align256(kOffSort + kSortBytes);

}  // namespace

// The scratch of sphgpu_nnps_noalloc: SPHGPU_NOALLOC_SCRATCH_BYTES per GPU.
static __device__ __align__(256) unsigned char g_nnps_scratch[kScratchBytes];

namespace {

struct NaArgs {
    int n, ndim, cxm, cym, czm, ctotal;
    double dr, xmin, ymin, zmin;
    const double* xp;   // caller: n * 3, particle-major
    const double* hl;   // caller: n
    const int* type;    // caller: n
    int* ninflu;        // caller: n
    int* influ;         // caller: n * 100, slot s + 1 of particle i at influ[i * 100 + s + 1]
    unsigned char* scratch;
};

__device__ __forceinline__ int na_to_int_x86(double v)
{
    return (v >= -2147483648.0 && v < 2147483648.0) ? (int)v : INT_MIN;
}

__device__ __forceinline__ int na_cell_link(const NaArgs& a, int c, int slot)
{
    int v;
    if (a.ndim == 2) {
        int ky = slot / 3 + 1, kx = slot % 3 + 1;
        v = (kx - 2) * a.cym + ky - 2 + c;
    } else {
        int kz = slot / 9 + 1, kx = (slot / 3) % 3 + 1, ky = slot % 3 + 1;
        v = (ky - 2) * a.cxm * a.czm + (kx - 2) * a.czm + kz - 2 + c;
    }
    return (v < 0 || v > a.ctotal) ? 0 : v;
}

// cell key of each particle (parttocell, CPP_3-NNPS.cpp:203-257); clears the
// error word and the cell ranges the search reads
__global__ void na_keys(NaArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int* err = reinterpret_cast<int*>(a.scratch + kOffErr);
    int* cstart = reinterpret_cast<int*>(a.scratch + kOffStart);
    int* cend = reinterpret_cast<int*>(a.scratch + kOffEnd);
    for (int c = i; c <= a.ctotal; c += gridDim.x * blockDim.x) {
        cstart[c] = (c == a.ctotal) ? 2000000 : 10000000;
        cend[c] = (c == a.ctotal) ? -2000000 : -10000000;
    }
    if (i >= a.n) return;
    const double xmin[3] = {a.xmin, a.ymin, a.zmin};
    const double dr = 2.0 * a.dr;
    int nx_t[3] = {0, 0, 0};
    for (int j = 0; j < a.ndim; j++) {
        double nx = fabs(a.xp[(size_t)i * 3 + j] - xmin[j]) / dr + 2.0;
        nx_t[j] = na_to_int_x86(nx);
        if (nx_t[j] < 2) nx_t[j] = 2;
    }
    unsigned key;
    if (a.ndim == 2)
        key = (unsigned)a.cym * (unsigned)(nx_t[0] - 1) + (unsigned)nx_t[1];
    else
        key = (unsigned)a.cxm * (unsigned)a.czm * (unsigned)(nx_t[1] - 1) +
              (unsigned)a.czm * (unsigned)(nx_t[0] - 1) + (unsigned)nx_t[2];
    int c = (int)key;
    if (!(c > 0 && c <= a.ctotal)) {
        atomicCAS(err, 0, SPH_ERR_CELL);
        c = 0;
    }
    reinterpret_cast<int*>(a.scratch + kOffCell)[i] = c;
    reinterpret_cast<uint32_t*>(a.scratch + kOffKeyIn)[a.n - 1 - i] = (uint32_t)c;
    reinterpret_cast<int*>(a.scratch + kOffValIn)[a.n - 1 - i] = i;
}

__global__ void na_clear_err(NaArgs a)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *reinterpret_cast<int*>(a.scratch + kOffErr) = 0;
}

__global__ void na_ranges(NaArgs a)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.n) return;
    const uint32_t* key = reinterpret_cast<const uint32_t*>(a.scratch + kOffKeyOut);
    const int* pid = reinterpret_cast<const int*>(a.scratch + kOffValOut);
    int* cstart = reinterpret_cast<int*>(a.scratch + kOffStart);
    int* cend = reinterpret_cast<int*>(a.scratch + kOffEnd);
    const uint32_t c = key[q];
    const bool first = (q == 0) || key[q - 1] != c;
    const bool last = (q == a.n - 1) || key[q + 1] != c;
    if ((int)c == a.ctotal) {
        if (first) atomicMin(&cstart[c], q);
        if (last) atomicMax(&cend[c], q);
    } else {
        if (first) cstart[c] = q;
        if (last) cend[c] = q;
    }
    const int j = pid[q];
    Pos r{a.xp[(size_t)j * 3], a.xp[(size_t)j * 3 + 1], a.xp[(size_t)j * 3 + 2], a.hl[j]};
    store_pos(reinterpret_cast<double*>(a.scratch + kOffXs), q, r);
}

__global__ void __launch_bounds__(128) na_search(NaArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    // a particle outside the grid stops the search (outputs not written);
    // more than 99 neighbours does not, so that every count is written
    const int* err = reinterpret_cast<const int*>(a.scratch + kOffErr);
    if (*err == SPH_ERR_CELL) return;
    int* errw = reinterpret_cast<int*>(a.scratch + kOffErr);
    const int* cell = reinterpret_cast<const int*>(a.scratch + kOffCell);
    const int* pid = reinterpret_cast<const int*>(a.scratch + kOffValOut);
    const int* cstart = reinterpret_cast<const int*>(a.scratch + kOffStart);
    const int* cend = reinterpret_cast<const int*>(a.scratch + kOffEnd);
    const double* xs = reinterpret_cast<const double*>(a.scratch + kOffXs);
    int cnt = 0;
    if (a.type[i] != 7) {
        const int nd = a.ndim, nst = (nd == 2) ? 9 : 27, nc = cell[i];
        const double xi[3] = {a.xp[(size_t)i * 3], a.xp[(size_t)i * 3 + 1], a.xp[(size_t)i * 3 + 2]};
        const double hi = a.hl[i];
        for (int nj = 0; nj < nst; nj++) {
            const int nl = na_cell_link(a, nc, nj);
            if (nl <= 0) continue;
            for (int q = cstart[nl]; q <= cend[nl]; q++) {
                const Pos pj = load_pos(xs, q);
                const double xj[3] = {pj.x, pj.y, pj.z};
                double dst = 0.0;
                for (int k = 0; k < nd; k++) dst = dst + (xi[k] - xj[k]) * (xi[k] - xj[k]);
                dst = sqrt(dst);
                const double ra = (hi + pj.h) / 2;
                const int j = pid[q];
                if (dst <= 2 * ra && i != j) {
                    cnt++;
                    if (cnt <= SPH_NB_CAP) a.influ[(size_t)i * 100 + cnt] = j;
                    else atomicCAS(errw, 0, SPH_ERR_NEIGH);
                }
            }
        }
    }
    a.ninflu[i] = cnt;
}

std::mutex g_setup_mu;
unsigned char* g_scratch_dev[64] = {nullptr};   // per device ordinal

}  // namespace

extern "C" int sphgpu_nnps_noalloc(const sphgpu_params* grid, int n, const double* d_xp, const double* d_hl,
                                   const int* d_type, int* d_ninflu, int* d_influ, void* stream)
{
    if (!grid || !d_xp || !d_hl || !d_type || !d_ninflu || !d_influ) return SPHGPU_E_ARG;
    if (grid->ndim != 2 && grid->ndim != 3) return SPHGPU_E_ARG;
    if (n <= 0 || n > kMaxN) return SPHGPU_E_ARG;              // beyond the fixed scratch
    if (grid->ctotal <= 0 || grid->ctotal > kMaxCells) return SPHGPU_E_ARG;
    if (!(grid->dr > 0.0)) return SPHGPU_E_ARG;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SPHGPU_E_NODEVICE;
    unsigned char* scratch;
    {
        // first call on this device: look the array up with the device current
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_dev[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_nnps_scratch) != cudaSuccess || !p) return SPHGPU_E_CUDA;
            g_scratch_dev[dev] = static_cast<unsigned char*>(p);
        }
        scratch = g_scratch_dev[dev];
    }
    int end_bit = 1;
    while (end_bit < 32 && (1u << end_bit) <= (unsigned)grid->ctotal) end_bit++;
    size_t need = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, need, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const int*)nullptr, (int*)nullptr, n, 0, end_bit);
    if (need > kSortBytes) return SPHGPU_E_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // an error the caller's own earlier work left pending is reported, not
    // taken over: nothing is launched and the error stays where it was
    if (cudaPeekAtLastError() != cudaSuccess) return SPHGPU_E_CUDA;
    NaArgs a;
    a.n = n; a.ndim = grid->ndim; a.cxm = grid->cxm; a.cym = grid->cym; a.czm = grid->czm;
    a.ctotal = grid->ctotal; a.dr = grid->dr; a.xmin = grid->xmin; a.ymin = grid->ymin; a.zmin = grid->zmin;
    a.xp = d_xp; a.hl = d_hl; a.type = d_type; a.ninflu = d_ninflu; a.influ = d_influ; a.scratch = scratch;
    const int threads = 256;
    const int cover = (n > grid->ctotal + 1) ? n : grid->ctotal + 1;
    na_clear_err<<<1, 32, 0, st>>>(a);
    if (cudaPeekAtLastError() != cudaSuccess) return SPHGPU_E_CUDA;
    na_keys<<<(cover + threads - 1) / threads, threads, 0, st>>>(a);
    if (cudaPeekAtLastError() != cudaSuccess) return SPHGPU_E_CUDA;
    size_t bytes = kSortBytes;
    if (cub::DeviceRadixSort::SortPairs(scratch + kOffSort, bytes, reinterpret_cast<uint32_t*>(scratch + kOffKeyIn),
                                        reinterpret_cast<uint32_t*>(scratch + kOffKeyOut),
                                        reinterpret_cast<int*>(scratch + kOffValIn),
                                        reinterpret_cast<int*>(scratch + kOffValOut), n, 0, end_bit,
                                        st) != cudaSuccess)
        return SPHGPU_E_CUDA;
    na_ranges<<<(n + threads - 1) / threads, threads, 0, st>>>(a);
    if (cudaPeekAtLastError() != cudaSuccess) return SPHGPU_E_CUDA;
    na_search<<<(n + 127) / 128, 128, 0, st>>>(a);
    if (cudaPeekAtLastError() != cudaSuccess) return SPHGPU_E_CUDA;
    // the call is synchronous: its status is the error word of this search,
    // read on the caller's stream (no wait on other streams of the device)
    int err = 0;
    if (cudaMemcpyAsync(&err, scratch + kOffErr, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return SPHGPU_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return SPHGPU_E_CUDA;
    return err;
}

extern "C" size_t sphgpu_nnps_noalloc_scratch_bytes(void) { return kScratchBytes; }
