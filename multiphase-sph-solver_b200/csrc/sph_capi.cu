// sph_capi.cu -- host side of the sphgpu C ABI (include/sphgpu.h).
//
// Owns the device buffers of one particle system, converts between the
// caller's particle-major arrays / Particle records and the device's
// component-major layout, evaluates the per-particle material constants, and
// runs time steps as CUDA graphs (one graph per step, two variants that
// alternate the ping-pong buffers of positions and stresses).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/sphgpu.h"
#include "sph_device.cuh"

extern "C" size_t sphk_sort_temp_bytes(int N, int end_bit);
extern "C" int sphk_enqueue_nnps(const Dev* d, void* sort_tmp, size_t sort_bytes, int end_bit, cudaStream_t st,
                                 cudaEvent_t* ev);
extern "C" int sphk_enqueue_nnps_parts(const Dev* d, void* sort_tmp, size_t sort_bytes, int end_bit,
                                       cudaStream_t st, cudaEvent_t* ev, int parts);
extern "C" int sphk_enqueue_physics(const Dev* d, cudaStream_t st, cudaEvent_t* ev, int regu);
extern "C" int sphk_enqueue_physics_bulk32(const Dev* d, cudaStream_t st, cudaEvent_t* ev, int regu);
extern "C" const char* const sphk_stage_names[];
extern "C" size_t sphk_kl_sort_bytes(size_t total);
extern "C" int sphk_kl_order(const double* d_r, int K, int ndim, double* keys_in, double* keys_out, uint32_t* vals_in,
                             uint32_t* vals_out, void* sort_tmp, size_t sort_bytes, cudaStream_t st);
extern "C" int sphk_kl_field(int n, int ndim, int K, int no, int type, const double* x_trans, double mean_value,
                             double sd_value, double coe_depth, double soil_max, double water_max, const double* d_xh,
                             const int* d_type, const void* d_terms, const double* d_sqrt_eig, const double* d_xi,
                             double* d_out, cudaStream_t st);
extern "C" size_t sphk_order_temp_bytes(int N, int end_bit);
extern "C" int sphk_order_sort(const Dev* dp, void* tmp, size_t bytes, int end_bit, unsigned long long* kin,
                               unsigned long long* kout, int* vin, int* vout, cudaStream_t st);
extern "C" size_t sphk_kl_term_bytes(void);
extern "C" int sphk_kl_wait_probe(long long budget, int* d_err, cudaStream_t st);
extern "C" size_t sphk_kl_tc_term_bytes(void);
extern "C" int sphk_kl_synthesize(int n, int ndim, int K, int R, int no, int type, const double* x_trans,
                                  double mean_value, double sd_value, double coe_depth, double soil_max,
                                  double water_max, const double* d_xh, const int* d_type, const void* d_terms,
                                  const double* d_sqrt_eig, const double* d_xi, float* c_hi, float* c_lo,
                                  float* d_out, int* d_err, cudaStream_t st, const void* d_modes,
                                  const int* nmode, const unsigned short* d_tidx);
extern "C" int sphk_rf_cells(const int* ip, const double* dp, const double* d_xh, const int* d_type, int* d_cell,
                             int* d_count, int* d_err, cudaStream_t st);
extern "C" int sphk_rf_factor(const int* ip, const double* dp, double* d_C, cudaStream_t st);
extern "C" int sphk_rf_assign(const int* ip, const double* dp, const double* d_L, const double* d_zeta, double* d_E,
                              const int* d_cell, const int* d_type, double* d_out, cudaStream_t st);

namespace {

thread_local int g_create_error = 0;

// the held order equal to the caller's
__global__ void k_order_identity(int* i2o, int* o2i, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) { i2o[i] = i; o2i[i] = i; }
}

struct FieldDef {
    const char* name;
    int ncomp;
    int is_int;
};

// Particle members the device owns (Class_particle.h:13-103)
const FieldDef kFields[] = {
    {"x", 3, 0}, {"xp", 3, 0}, {"vx", 3, 0}, {"vxp", 3, 0}, {"ax", 3, 0}, {"axp", 3, 0},
    {"ux", 3, 0}, {"strep", 3, 0}, {"interf", 3, 0}, {"interfss", 3, 0},
    {"rho", 1, 0}, {"rhop", 1, 0}, {"mass", 1, 0}, {"hl", 1, 0}, {"pre", 1, 0}, {"prep", 1, 0},
    {"e", 1, 0}, {"eps", 6, 0}, {"sig", 6, 0}, {"adps", 6, 0}, {"tssig", 6, 0}, {"tsqc", 1, 0},
    {"satu", 1, 0}, {"dsatu", 1, 0}, {"suct", 1, 0}, {"cop", 1, 0},
    {"vsig", 1, 0}, {"veps", 1, 0}, {"divq", 1, 0}, {"divr", 1, 0}, {"meps", 1, 0},
    {"prew", 1, 0}, {"prea", 1, 0}, {"porosity", 1, 0}, {"poro_cop", 1, 0}, {"cd", 1, 0},
    {"type", 1, 1}, {"matype", 1, 1}, {"permtype", 1, 1}, {"etype", 1, 1},
};

const FieldDef* find_field(const char* name)
{
    if (!name) return nullptr;
    for (const FieldDef& f : kFields)
        if (std::strcmp(f.name, name) == 0) return &f;
    return nullptr;
}

// byte offsets of the members in the reference's Particle (1064 bytes)
struct AosMember { const char* name; size_t off; };
const AosMember kAos[] = {
    {"x", 0}, {"xp", 24}, {"vx", 48}, {"vxp", 72}, {"ax", 96}, {"axp", 120}, {"ux", 144},
    {"strep", 168}, {"interf", 264}, {"interfss", 288}, {"rho", 312}, {"rhop", 320},
    {"mass", 328}, {"hl", 336}, {"pre", 344}, {"prep", 352}, {"e", 360}, {"eps", 368},
    {"sig", 464}, {"adps", 656}, {"tssig", 704}, {"tsqc", 752}, {"satu", 760}, {"dsatu", 768},
    {"suct", 776}, {"cop", 784}, {"vsig", 792}, {"veps", 800},
    {"divq", 808}, {"divr", 816}, {"meps", 824}, {"prew", 864}, {"prea", 872},
    {"porosity", 880}, {"cd", 888}, {"poro_cop", 896}, {"type", 1048}, {"matype", 1052},
    {"permtype", 1056}, {"etype", 1060},
};
constexpr size_t kParticleBytes = 1064;

}  // namespace

// An allocator whose elements start uninitialised: a resize of a large host
// array then leaves its pages untouched until the copy that fills it, which
// runs on several threads (zero-filling first would cost a single-threaded
// pass over the whole array)
template <typename T>
struct UninitAlloc {
    typedef T value_type;
    UninitAlloc() = default;
    template <typename U> UninitAlloc(const UninitAlloc<U>&) {}
    T* allocate(size_t n) { return static_cast<T*>(::operator new(n * sizeof(T))); }
    void deallocate(T* p, size_t) { ::operator delete(p); }
    template <typename U> void construct(U*) {}
    template <typename U, typename... A> void construct(U* p, A&&... a) { ::new ((void*)p) U(std::forward<A>(a)...); }
    template <typename U> bool operator==(const UninitAlloc<U>&) const { return true; }
    template <typename U> bool operator!=(const UninitAlloc<U>&) const { return false; }
};

struct sphgpu_ctx {
    sphgpu_params P;
    int device = 0;
    int N = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    Dev d[2];              // parity variants: d[p] reads buffers "cur" of parity p
    int parity = 0;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    void* sort_tmp = nullptr;
    size_t sort_bytes = 0;
    int end_bit = 1;
    std::vector<void*> allocs;
    // filled whole by whoever sizes them, so left uninitialised until then
    std::vector<int, UninitAlloc<int>> h_type, h_matype;
    std::vector<double, UninitAlloc<double>> h_x;   // x as uploaded (the reference writes it only in update)
    bool x_tracked = false;
    int l_host = 1;
    double last_ms = 0.0;
    long launches_per_step = 0;
    long last_launches = 0;
    int sticky = 0;
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    // record transfer staging: two pinned host and two device chunks
    void* rec_pinned[2] = {nullptr, nullptr};
    void* rec_dev[2] = {nullptr, nullptr};
    size_t rec_bytes = 0;
    cudaEvent_t rec_ev[2] = {nullptr, nullptr};
    bool regu = false;     // graphs include the strain/stress regularisation passes
    int precision = SPHGPU_PREC_FP64;
    std::vector<sphgpu_fluid, UninitAlloc<sphgpu_fluid>> h_fluid;   // the material records last set
    std::vector<sphgpu_soil, UninitAlloc<sphgpu_soil>> h_soil;      // (K-L fields rewrite members)
    double* mat_pinned = nullptr;     // pinned, 4N: the per-particle material constants set_materials uploads
    int part_done = 0;     // parts of step l run through the method entries: 1 parttocell, 2 partisearching
    sphgpu_rain rain = {};            // the rainfall record (flr 1), nrain as last set
    bool rain_set = false;
    sphgpu_vibration vib = {};        // the vibration table (flv 1, 2) as last set
    std::vector<double> vib_loads;
    bool vib_set = false;
    double vib_par[4] = {0, 0, 0, 0};   // ttime, nsteps, sttime, edtime (checkpoint record)
    bool accb_vib = false;            // accb holds the vibration rows (19N)
    // the output writer: two slots of device staging, pinned host copy,
    // completion event and writer thread
    double* out_dev[2] = {nullptr, nullptr};
    double* out_host[2] = {nullptr, nullptr};
    cudaEvent_t out_ev[2] = {nullptr, nullptr};
    cudaStream_t out_st = nullptr;
    std::thread out_th[2];
    int out_next = 0;
    int out_err = 0;
    // the files several steps append to are appended in call order: each
    // call takes a ticket, and its thread appends when the tickets before it
    // have
    std::mutex out_mu;
    std::condition_variable out_cv;
    long out_ticket = 0, out_turn = 0;
    std::vector<InstGrid> h_inst;     // batched context: the instance table (empty: one system)
    InstGrid* d_inst = nullptr;
    // the re-sorted state (sphgpu_set_reorder): re-sort every reorder_every
    // steps (0: never), steps run since the last re-sort, whether the state
    // is held out of the caller's order; the gather buffer, and the order
    // keys, their sort's permutation and its work space
    int reorder_every = 0;
    long since_sort = 0;
    bool permuted = false;
    void* perm_tmp = nullptr;
    size_t perm_tmp_bytes = 0;
    unsigned long long *ord_kin = nullptr, *ord_kout = nullptr;
    int *ord_vin = nullptr, *ord_vout = nullptr;
    void* ord_tmp = nullptr;
    size_t ord_bytes = 0;
    int ord_end_bit = 0;
    double reorder_ms = 0.0;          // device time of the re-sorts of the last sphgpu_step_profiled
};

namespace {

int cuda_fail(sphgpu_ctx* c, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return 0;
    std::fprintf(stderr, "sphgpu: %s: %s\n", what, cudaGetErrorString(e));
    if (c) c->sticky = SPHGPU_E_CUDA;
    return SPHGPU_E_CUDA;
}
#define CK(call) do { int _r = cuda_fail(c, (call), #call); if (_r) return _r; } while (0)

template <typename T>
int dalloc(sphgpu_ctx* c, T** p, size_t count)
{
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 16);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc");
    cudaMemsetAsync(q, 0, count * sizeof(T) + 16, c->st);
    c->allocs.push_back(q);
    *p = (T*)q;
    return 0;
}

int check_params(const sphgpu_params* P)
{
    if (!P) return SPHGPU_E_ARG;
    if (P->ndim != 2 && P->ndim != 3) return SPHGPU_E_ARG;
    if (P->ntotal <= 0 || P->ctotal <= 0 || P->cxm <= 0 || P->cym <= 0 || P->czm <= 0) return SPHGPU_E_ARG;
    // the search packs a particle index and its type code into one 32-bit word
    if (P->ntotal >= (1 << 28)) return SPHGPU_E_UNSUPPORTED;
    if ((long long)P->cxm * P->cym * P->czm != P->ctotal) return SPHGPU_E_ARG;
    if (!(P->dr > 0.0) || !(P->dt > 0.0)) return SPHGPU_E_ARG;
    if (P->step_regu <= 0) return SPHGPU_E_ARG;
    // flag combinations this engine runs (the others are rejected loudly)
    if (!(P->flbndy >= 1 && P->flbndy <= 5) && P->flbndy != 13 && P->flbndy != 14) return SPHGPU_E_UNSUPPORTED;
    if (P->flknl < 1 || P->flknl > 4) return SPHGPU_E_UNSUPPORTED;
    if (P->flv < 0 || P->flv > 2) return SPHGPU_E_UNSUPPORTED;
    if (P->fli < 0 || P->fli > 3) return SPHGPU_E_UNSUPPORTED;
    if (P->ss_type < 0 || P->ss_type > 3) return SPHGPU_E_UNSUPPORTED;
    if (P->if_move < 0 || P->if_move > 3) return SPHGPU_E_UNSUPPORTED;
    return 0;
}

// the kernels' copy of the run parameters
void fill_dev_params(DevParams& p, const sphgpu_params* P)
{
    const int N = P->ntotal;
    p.N = N; p.ndim = P->ndim; p.flknl = P->flknl; p.flbndy = P->flbndy; p.fli = P->fli;
    p.if_move = P->if_move; p.flv = P->flv; p.inip = P->inip; p.step_regu = P->step_regu;
    p.cxm = P->cxm; p.cym = P->cym; p.czm = P->czm; p.ctotal = P->ctotal;
    p.water_minor = P->water_acc_type != 0; p.air_minor = P->air_acc_type != 0;
    p.first_vbx_wall = N;
    p.dr = P->dr; p.dt = P->dt;
    p.xsph0 = P->xsph[0]; p.xsph1 = P->xsph[1]; p.xsph2 = P->xsph[2];
    for (int a = 0; a < 3; a++) for (int b = 0; b < 2; b++) p.av[a][b] = P->art_vis[a][b];
    p.gx = P->gx; p.gy = P->gy; p.gz = P->gz;
    p.thr_min = P->threshold_min; p.thr_max = P->threshold_max;
    p.interc = P->interc; p.pers = P->pers; p.perl = P->perl; p.perm = P->perm; p.permtype = P->permtype;
    p.coe_bndy = P->coe_bndy;
    for (int k = 0; k < 3; k++) p.move_vx[k] = P->move_vx[k];
    p.xmin = P->xmin; p.xmax = P->xmax; p.ymin = P->ymin; p.ymax = P->ymax; p.zmin = P->zmin; p.zmax = P->zmax;
    p.st_e = P->structure.e; p.st_poi = P->structure.poi;
    p.g_acc = std::sqrt(P->gx * P->gx + P->gy * P->gy + P->gz * P->gz);   // CPP_10-interact1.cpp:28
    p.art_stre_coe = P->art_stre_coe;
    p.ss_type = P->ss_type; p.ss_myu = P->ss_myu; p.ss_zeta = P->ss_zeta;
    p.ss_coupled = (P->ss_type >= 1 && P->ss_type <= 3 && P->ss_acc_type == 2) ? 1 : 0;
    p.flts = P->flts;
    p.flagum = P->flagum;
    p.alphats = P->alphats;
    p.cfl_on = 0; p.cfl_c = 0.0; p.cfl_f = 0.0;
    p.st_vpu = P->structure.vpu;
    p.ninst = 0;
    for (int q = 0; q < TP_COUNT; q++) p.tb[q] = 128;
    p.flr = P->flr == 1 ? 1 : 0;
    p.rain_lp = 0; p.rain_vrain = 0.0; p.rain_press = 0.0;
    p.vib_ttime = 0.0; p.vib_st = 0.0; p.vib_ed = 0.0; p.vib_nsteps = 0;
    p.ff_e = 0.0; p.ff_poi = 0.0;      // pFFBound: Para_Soil() (Class_ParticleProperty.cpp:28-31)
}

// the buffers only some flag settings use, allocated when the flags first
// need them (at create, or when sphgpu_update_params turns the flags on)
int alloc_optional(sphgpu_ctx* c, const sphgpu_params* P)
{
    DevState& s = c->d[0].s;
    const int N = c->N;
    int r = 0;
    auto need = [&](auto*& ptr, size_t count) {
        if (!ptr) r |= dalloc(c, &ptr, count);
    };
    if (P->art_stre_coe > 0.0) need(s.rij, 9 * (size_t)N);
    if (P->ss_type >= 1) {
        need(s.ss_id, 3 * (size_t)N);
        need(s.ss_con, 18 * (size_t)N);
        need(s.ss_own, 6 * (size_t)N);
        need(s.ss_fs, 6 * (size_t)N);
    }
    if (P->ss_type >= 1 && P->ss_type <= 3 && P->ss_acc_type == 2) need(s.cpl, 3 * (size_t)N);
    if (P->flbndy == 5) {
        need(s.fsol, 3 * (size_t)N);
        need(s.fsol_on, (size_t)N);
    }
    if (P->flv > 0) need(s.stiff, (size_t)N);
    if (P->flv != 0 && !c->accb_vib) {
        // the momentum pass's vibration rows: accb grows from 9N to 19N
        double* q = nullptr;
        r |= dalloc(c, &q, 19 * (size_t)N);
        if (q) { s.accb = q; c->d[1].s.accb = q; c->accb_vib = true; }
    }
    if (P->flbndy != 1 && P->flbndy != 5) {
        need(s.vel_bndy, 3 * (size_t)N);
        need(s.vb, 12 * (size_t)N);
        need(s.vx_vb, 3 * (size_t)N);
        if (P->flbndy != 2) need(s.sb, 24 * (size_t)N);
    }
    // the other parity variant shares them
    DevState& t = c->d[1].s;
    t.rij = s.rij; t.ss_id = s.ss_id; t.ss_con = s.ss_con; t.ss_own = s.ss_own; t.ss_fs = s.ss_fs;
    t.cpl = s.cpl; t.fsol = s.fsol; t.fsol_on = s.fsol_on;
    t.vel_bndy = s.vel_bndy; t.vb = s.vb; t.vx_vb = s.vx_vb; t.sb = s.sb;
    t.stiff = s.stiff;
    return r;
}

int end_bit_for(int m)
{
    int b = 1;
    while (b < 32 && (1u << b) <= (unsigned)m) b++;
    return b;
}

// the physics stages of one step in the context's precision form
int enqueue_physics(const sphgpu_ctx* c, const Dev* d, cudaEvent_t* ev)
{
    const int regu = c->regu ? 1 : 0;
    if (c->precision == SPHGPU_PREC_FP32_BULK) return sphk_enqueue_physics_bulk32(d, c->st, ev, regu);
    return sphk_enqueue_physics(d, c->st, ev, regu);
}

// (re)build the two step graphs: NNPS + physics for parity 0 and 1
int build_graphs(sphgpu_ctx* c)
{
    for (int p = 0; p < 2; p++) {
        if (c->exec[p]) { cudaGraphExecDestroy(c->exec[p]); c->exec[p] = nullptr; }
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
        int n = sphk_enqueue_nnps(&c->d[p], c->sort_tmp, c->sort_bytes, c->end_bit, c->st, nullptr);
        n += enqueue_physics(c, &c->d[p], nullptr);
        cudaError_t e = cudaStreamEndCapture(c->st, &g);
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&c->exec[p], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
        c->launches_per_step = n;
    }
    return 0;
}

void invalidate_graphs(sphgpu_ctx* c)
{
    for (int p = 0; p < 2; p++)
        if (c->exec[p]) { cudaGraphExecDestroy(c->exec[p]); c->exec[p] = nullptr; }
}

// ---------------------------------------------------------------------------
// Re-sorted state.  With sphgpu_set_reorder(c, R), R > 0, sphgpu_step gathers
// the whole particle state on the device every R steps into a spatial order
// (k_order_key: by type and material, then rows of a lattice of spacing dr),
// so that the neighbour gathers of every pass read nearby records whatever
// order the caller's particles came in or have mixed into.  i2o / o2i map
// between the held order and the caller's; the kernels whose result depends
// on the caller's numbering (the cell keys' tie order, the rain rows,
// check_domain's first wall, tm_boundary's default wall, the structure's
// reaction order) read them, so every result is the caller's order's.  The
// entries that exchange per-particle data with the host or run part of a
// step first put the state back in the caller's order; the result-file
// snapshot writes its rows through i2o instead.

// one array of the state: cols columns of esz-byte elements, column-major
// (element (i, k) at k N + i) or, with aos set, records of cols elements
struct PermArr { void* p; int esz; int cols; int aos; };

// the arrays a later step reads (every device-owned Particle member, the
// material constants, the walls' per-phase records, the stiffness of the
// last stress update, the batched instance of each particle); the per-step
// intermediates and the search's arrays are rewritten by the next step
std::vector<PermArr> perm_arrays(const sphgpu_ctx* c, int parity)
{
    const DevState& s = c->d[parity].s;
    std::vector<PermArr> v;
    auto i4 = [&](void* p) { if (p) v.push_back({p, 4, 1, 0}); };
    auto f8 = [&](void* p, int cols) { if (p) v.push_back({p, 8, cols, 0}); };
    i4(s.type); i4(s.matype); i4(s.etype); i4(s.permtype); i4(s.f_bhtype); i4(s.pinst);
    for (double* p : {s.mass, s.cd, s.f_dens, s.f_por, s.f_vpu, s.f_vis, s.f_c, s.f_smin, s.f_tanfai,
                      s.s_e, s.s_poi, s.s_eps0, s.s_dens, s.s_kapa, s.s_por, s.s_vpu, s.s_cop, s.s_sitas,
                      s.s_sitar, s.s_ds, s.s_c, s.s_fs, s.s_ann, s.s_zmf, s.s_ramda, s.s_sme0, s.s_yalf,
                      s.s_ykap, s.s_yalf_dil})
        f8(p, 1);
    f8(s.s_ext, SX_COUNT);
    if (s.xh) v.push_back({s.xh, 8, 4, 1});
    for (double* p : {s.vx, s.vxp, s.axp, s.ax, s.ux, s.interf, s.interfss, s.strep, s.vel_bndy, s.vx_vb})
        f8(p, 3);
    for (double* p : {s.rho, s.rhop, s.pre, s.prep, s.porosity, s.poro_cop, s.e, s.tsqc, s.satu, s.dsatu,
                      s.suct, s.cop, s.prew, s.prea, s.vsig, s.veps, s.divq, s.divr, s.meps, s.stiff})
        f8(p, 1);
    for (double* p : {s.sig, s.eps, s.adps, s.tssig}) f8(p, 6);
    f8(s.vb, 12);
    f8(s.sb, 24);
    return v;
}

// One array of the state on the device for the fused gather: the array, its
// gather buffer (a part of the context's scratch), element size, columns and
// layout as PermArr.
struct PermDev { void* arr; void* tmp; int esz, cols, aos, pad; };

// tmp = arr gathered by perm, for every array of the table in one launch: one
// thread per particle position q takes element(s) perm[q] of each array in
// turn, four loads in flight before their stores.  The reads are gathers of a
// nearly sorted permutation, the writes coalesced.  An AoS array (the
// position records) has an even number of doubles per record, moved as pairs.
__global__ void __launch_bounds__(256) k_perm_gather_all(const PermDev* __restrict__ tab, int na,
                                                         const int* __restrict__ perm, int N)
{
    const int qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= N) return;
    const size_t q = (size_t)qi, p = (size_t)perm[qi], n = (size_t)N;
    for (int a = 0; a < na; a++) {
        const PermDev e = tab[a];
        if (e.esz == 4) {
            const int* s = static_cast<const int*>(e.arr);
            int* d = static_cast<int*>(e.tmp);
            for (int k = 0; k < e.cols; k++) d[k * n + q] = s[k * n + p];
        } else if (e.aos) {
            const double2* s = static_cast<const double2*>(e.arr);
            double2* d = static_cast<double2*>(e.tmp);
            const int h = e.cols / 2;
            for (int k = 0; k < h; k++) d[q * h + k] = s[p * h + k];
        } else {
            const double* s = static_cast<const double*>(e.arr);
            double* d = static_cast<double*>(e.tmp);
            for (int k0 = 0; k0 < e.cols; k0 += 4) {
                double v[4];
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (k0 + u < e.cols) v[u] = s[(size_t)(k0 + u) * n + p];
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (k0 + u < e.cols) d[(size_t)(k0 + u) * n + q] = v[u];
            }
        }
    }
}

// arr = tmp for every array of the table (the gathered state back into the
// arrays the step graphs were captured with), one thread per position
__global__ void __launch_bounds__(256) k_perm_copy_all(const PermDev* __restrict__ tab, int na, int N)
{
    const int qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= N) return;
    const size_t q = (size_t)qi, n = (size_t)N;
    for (int a = 0; a < na; a++) {
        const PermDev e = tab[a];
        if (e.esz == 4) {
            const int* s = static_cast<const int*>(e.tmp);
            int* d = static_cast<int*>(e.arr);
            for (int k = 0; k < e.cols; k++) d[k * n + q] = s[k * n + q];
        } else if (e.aos) {
            const double2* s = static_cast<const double2*>(e.tmp);
            double2* d = static_cast<double2*>(e.arr);
            const int h = e.cols / 2;
            for (int k = 0; k < h; k++) d[q * h + k] = s[q * h + k];
        } else {
            const double* s = static_cast<const double*>(e.tmp);
            double* d = static_cast<double*>(e.arr);
            for (int k0 = 0; k0 < e.cols; k0 += 4) {
                double v[4];
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (k0 + u < e.cols) v[u] = s[(size_t)(k0 + u) * n + q];
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (k0 + u < e.cols) d[(size_t)(k0 + u) * n + q] = v[u];
            }
        }
    }
}

__global__ void k_copy_int(const int* __restrict__ src, int* __restrict__ dst, int n)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) dst[t] = src[t];
}

// after a re-sort by perm: the held particle i is the caller's i2o[perm[i]]
__global__ void k_order_compose(const int* __restrict__ perm, const int* __restrict__ i2o, int* __restrict__ out,
                                int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = i2o[perm[i]];
}

__global__ void k_order_inverse(const int* __restrict__ i2o, int* __restrict__ o2i, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) o2i[i2o[i]] = i;
}

unsigned perm_blocks(size_t n) { return (unsigned)((n + 255) / 256); }

int ensure_perm_tmp(sphgpu_ctx* c, size_t bytes)
{
    if (c->perm_tmp_bytes >= bytes) return 0;
    if (c->perm_tmp) {
        CK(cudaStreamSynchronize(c->st));
        cudaFree(c->perm_tmp);
    }
    c->perm_tmp = nullptr;
    c->perm_tmp_bytes = 0;
    CK(cudaMalloc(&c->perm_tmp, bytes));
    c->perm_tmp_bytes = bytes;
    return 0;
}

// every array of the state (the buffers of `parity`) gathered by perm, on
// the context's stream, and the maps moved with them.  The scratch holds the
// device table of the arrays, each array's gather buffer and the new i2o.
int enqueue_permute(sphgpu_ctx* c, int parity, const int* perm)
{
    const std::vector<PermArr> arr = perm_arrays(c, parity);
    const int N = c->N;
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t table_bytes = up(sizeof(PermDev) * arr.size());
    std::vector<PermDev> tab(arr.size());
    size_t off = table_bytes;
    for (size_t a = 0; a < arr.size(); a++) {
        if (arr[a].aos && arr[a].cols % 2 != 0) return SPHGPU_E_ARG;
        tab[a] = PermDev{arr[a].p, nullptr, arr[a].esz, arr[a].cols, arr[a].aos, 0};
        off += up((size_t)arr[a].esz * arr[a].cols * N);
    }
    const size_t i2o_off = off;
    int r = ensure_perm_tmp(c, i2o_off + up(4 * (size_t)N));
    if (r) return r;
    char* base = static_cast<char*>(c->perm_tmp);
    off = table_bytes;
    for (size_t a = 0; a < arr.size(); a++) {
        tab[a].tmp = base + off;
        off += up((size_t)arr[a].esz * arr[a].cols * N);
    }
    const PermDev* dtab = reinterpret_cast<const PermDev*>(base);
    CK(cudaMemcpyAsync(base, tab.data(), sizeof(PermDev) * tab.size(), cudaMemcpyHostToDevice, c->st));
    k_perm_gather_all<<<perm_blocks(N), 256, 0, c->st>>>(dtab, (int)tab.size(), perm, N);
    k_perm_copy_all<<<perm_blocks(N), 256, 0, c->st>>>(dtab, (int)tab.size(), N);
    const DevState& s = c->d[parity].s;
    int* tmp = reinterpret_cast<int*>(base + i2o_off);
    k_order_compose<<<perm_blocks(N), 256, 0, c->st>>>(perm, s.i2o, tmp, N);
    k_copy_int<<<perm_blocks(N), 256, 0, c->st>>>(tmp, s.i2o, N);
    k_order_inverse<<<perm_blocks(N), 256, 0, c->st>>>(s.i2o, s.o2i, N);
    CK(cudaGetLastError());
    return 0;
}

// the state re-sorted into the order of k_order_key over its current
// positions (the buffers of `parity`)
int sort_state(sphgpu_ctx* c, int parity)
{
    const int N = c->N;
    if (!c->ord_tmp) {
        // each buffer allocated once (a failed call leaves the others for the next)
        int r = 0;
        if (!c->ord_kin) r |= dalloc(c, &c->ord_kin, (size_t)N);
        if (!c->ord_kout) r |= dalloc(c, &c->ord_kout, (size_t)N);
        if (!c->ord_vin) r |= dalloc(c, &c->ord_vin, (size_t)N);
        if (!c->ord_vout) r |= dalloc(c, &c->ord_vout, (size_t)N);
        if (r) return r;
        // keys stay below 512 groups x 8 (ctotal + 1): the bits the sort looks at
        const unsigned long long top = 512ull * 8ull * ((unsigned long long)c->P.ctotal + 1);
        int b = 1;
        while (b < 64 && (1ull << b) <= top) b++;
        c->ord_end_bit = b;
        c->ord_bytes = sphk_order_temp_bytes(N, b);
        void* t = nullptr;
        CK(cudaMalloc(&t, c->ord_bytes + 256));
        c->allocs.push_back(t);
        c->ord_tmp = t;
    }
    sphk_order_sort(&c->d[parity], c->ord_tmp, c->ord_bytes, c->ord_end_bit, c->ord_kin, c->ord_kout, c->ord_vin,
                    c->ord_vout, c->st);
    int r = enqueue_permute(c, parity, c->ord_vout);
    if (r) return r;
    c->permuted = true;
    c->since_sort = 0;
    return 0;
}

// the state put back in the caller's order (a no-op when it is there), done
// when the call returns
int to_caller_order(sphgpu_ctx* c)
{
    if (!c->permuted) return 0;
    cudaSetDevice(c->device);
    // perm = o2i: the gathers and the new i2o (the identity) read it before
    // the last launch of enqueue_permute rewrites it (the identity too)
    int r = enqueue_permute(c, c->parity, c->d[c->parity].s.o2i);
    if (r) return r;
    CK(cudaStreamSynchronize(c->st));
    c->permuted = false;
    c->since_sort = 1L << 40;
    return 0;
}

// the re-sort due before the next step, if any
int sort_if_due(sphgpu_ctx* c, int parity)
{
    if (c->reorder_every <= 0 || c->since_sort < c->reorder_every) return 0;
    return sort_state(c, parity);
}

// a loop over [0, n) split across host threads (gathers and copies of large
// host arrays run at the host's memory bandwidth, not one core's)
void par_for(size_t n, const std::function<void(size_t, size_t)>& body)
{
    unsigned T = std::thread::hardware_concurrency();
    if (T == 0) T = 4;
    if (T > 16) T = 16;
    if (n < 4096 || T == 1) { body(0, n); return; }
    std::vector<std::thread> th;
    const size_t per = (n + T - 1) / T;
    for (unsigned t = 0; t < T; t++) {
        const size_t a = t * per, b = std::min(n, a + per);
        if (a < b) th.emplace_back(body, a, b);
    }
    for (auto& x : th) x.join();
}

// writes one byte of every 4 KB page of [p, p + bytes) on all cores, so
// that the pages are mapped before a timed copy into them
void prefault(void* p, size_t bytes)
{
    char* b = static_cast<char*>(p);
    par_for((bytes + 4095) / 4096, [&](size_t a, size_t e) {
        for (size_t q = a; q < e; q++) b[q * 4096] = 0;
    });
}

int ensure_pinned(sphgpu_ctx* c, size_t bytes)
{
    if (c->pinned_bytes >= bytes) return 0;
    if (c->pinned) cudaFreeHost(c->pinned);
    c->pinned = nullptr;
    c->pinned_bytes = 0;
    CK(cudaMallocHost(&c->pinned, bytes));
    c->pinned_bytes = bytes;
    return 0;
}

// device pointer behind a field name for the current parity
void* field_ptr(sphgpu_ctx* c, const char* name)
{
    DevState& s = c->d[c->parity].s;
    struct { const char* n; void* p; } tab[] = {
        {"vx", s.vx}, {"vxp", s.vxp}, {"ax", s.ax}, {"axp", s.axp}, {"ux", s.ux},
        {"strep", s.strep}, {"interf", s.interf}, {"interfss", s.interfss}, {"rho", s.rho},
        {"rhop", s.rhop}, {"mass", s.mass}, {"pre", s.pre}, {"prep", s.prep},
        {"e", s.e}, {"eps", s.eps}, {"sig", s.sig}, {"adps", s.adps}, {"tssig", s.tssig}, {"tsqc", s.tsqc},
        {"satu", s.satu}, {"dsatu", s.dsatu}, {"suct", s.suct}, {"cop", s.cop},
        {"vsig", s.vsig}, {"veps", s.veps}, {"divq", s.divq}, {"divr", s.divr}, {"meps", s.meps},
        {"prew", s.prew}, {"prea", s.prea}, {"porosity", s.porosity}, {"poro_cop", s.poro_cop},
        {"cd", s.cd}, {"type", s.type}, {"matype", s.matype}, {"permtype", s.permtype}, {"etype", s.etype},
    };
    for (auto& t : tab)
        if (std::strcmp(t.n, name) == 0) return t.p;
    return nullptr;
}

// the first wall (index order) with matype > 2 in [a, b), or b
int first_vbx_wall(const sphgpu_ctx* c, int a, int b)
{
    if (!c->h_type.empty() && !c->h_matype.empty())
        for (int i = a; i < b; i++)
            if (c->h_type[i] == 0 && c->h_matype[i] > 2) return i;
    return b;
}

void update_static_params(sphgpu_ctx* c)
{
    const int w0 = first_vbx_wall(c, 0, c->N);
    for (int p = 0; p < 2; p++) c->d[p].p.first_vbx_wall = w0;
    if (!c->h_inst.empty()) {
        for (InstGrid& g : c->h_inst) g.first_vbx_wall = first_vbx_wall(c, g.first, g.first + g.count);
        cuda_fail(c, cudaMemcpyAsync(c->d_inst, c->h_inst.data(), sizeof(InstGrid) * c->h_inst.size(),
                                     cudaMemcpyHostToDevice, c->st), "cudaMemcpyAsync");
        cuda_fail(c, cudaStreamSynchronize(c->st), "cudaStreamSynchronize");
    }
    invalidate_graphs(c);
}

int check_particles(sphgpu_ctx* c)
{
    if (c->h_type.empty() || c->h_matype.empty()) return SPHGPU_E_STATE;
    if (c->P.flr == 1 && !c->rain_set) return SPHGPU_E_STATE;
    if (c->P.flv >= 1 && !c->vib_set) return SPHGPU_E_STATE;
    // the vibration damping reads damp1 / damp2 from the extended soil block
    bool ext = c->P.flagum == 1 || c->P.flv > 0;
    for (int i = 0; i < c->N; i++) {
        const int t = c->h_type[i], m = c->h_matype[i];
        // matype 30-49 and >= 60 match no branch of strain_to_stress
        if (t == 2) {
            if ((m >= 30 && m < 50) || m >= 60)
                return SPHGPU_E_UNSUPPORTED;
            if (m % 10 == 3 || m % 10 == 8) ext = true;
        }
    }
    // those models and the saturation pass read material members that
    // sphgpu_set_materials uploads once it has seen them in use
    if (ext && !c->d[0].s.s_ext) return SPHGPU_E_STATE;
    return 0;
}

}  // namespace

namespace {

// One device-owned Particle member in the record transfer: its byte offset
// in the caller's record, its components, where it lives on the device
// (kind 0: doubles, component-major; 1: int; 2: x, y, z of the position
// records xh; 3: h of xh) and its byte offset in the packed download record.
struct RecMember {
    int off, nc, kind, pk;
    void* dst;
};
constexpr int kMaxRecMembers = 48;
constexpr int kRecChunk = 65536;          // records per staged chunk

// caller records -> SoA state, one thread per record of the chunk
__global__ void k_rec_unpack(const char* recs, size_t stride, int i0, int cnt, int N, const RecMember* tab, int nt)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnt) return;
    const char* r = recs + (size_t)t * stride;
    const size_t i = (size_t)i0 + t;
    for (int m = 0; m < nt; m++) {
        const RecMember e = tab[m];
        const double* v = reinterpret_cast<const double*>(r + e.off);
        if (e.kind == 0) {
            for (int k = 0; k < e.nc; k++) static_cast<double*>(e.dst)[(size_t)k * N + i] = v[k];
        } else if (e.kind == 1) {
            static_cast<int*>(e.dst)[i] = *reinterpret_cast<const int*>(r + e.off);
        } else if (e.kind == 2) {
            for (int k = 0; k < 3; k++) static_cast<double*>(e.dst)[i * 4 + k] = v[k];
        } else {
            static_cast<double*>(e.dst)[i * 4 + 3] = v[0];
        }
    }
}

// SoA state -> packed records of the owned members (P bytes each)
__global__ void k_rec_pack(char* out, size_t P, int i0, int cnt, int N, const RecMember* tab, int nt)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnt) return;
    char* r = out + (size_t)t * P;
    const size_t i = (size_t)i0 + t;
    for (int m = 0; m < nt; m++) {
        const RecMember e = tab[m];
        double* v = reinterpret_cast<double*>(r + e.pk);
        if (e.kind == 0) {
            for (int k = 0; k < e.nc; k++) v[k] = static_cast<const double*>(e.dst)[(size_t)k * N + i];
        } else if (e.kind == 1) {
            *reinterpret_cast<int*>(r + e.pk) = static_cast<const int*>(e.dst)[i];
        } else if (e.kind == 2) {
            for (int k = 0; k < 3; k++) v[k] = static_cast<const double*>(e.dst)[i * 4 + k];
        } else {
            v[0] = static_cast<const double*>(e.dst)[i * 4 + 3];
        }
    }
}

// the table of device-owned members (all but x, which the host keeps) for
// the current parity, and the packed record size
int rec_table(sphgpu_ctx* c, std::vector<RecMember>& tab, size_t* packed)
{
    tab.clear();
    size_t pk = 0;
    for (const AosMember& m : kAos) {
        if (std::strcmp(m.name, "x") == 0) continue;
        const FieldDef* f = find_field(m.name);
        RecMember e;
        e.off = (int)m.off;
        e.nc = f->ncomp;
        e.pk = (int)pk;
        if (std::strcmp(m.name, "xp") == 0) { e.kind = 2; e.dst = c->d[c->parity].s.xh; }
        else if (std::strcmp(m.name, "hl") == 0) { e.kind = 3; e.dst = c->d[c->parity].s.xh; }
        else { e.kind = f->is_int ? 1 : 0; e.dst = field_ptr(c, m.name); }
        if (!e.dst) return SPHGPU_E_ARG;
        pk += f->is_int ? 8 : 8 * (size_t)f->ncomp;   // ints keep an 8-byte slot
        tab.push_back(e);
    }
    if ((int)tab.size() > kMaxRecMembers) return SPHGPU_E_ARG;
    *packed = pk;
    return 0;
}

int ensure_rec_staging(sphgpu_ctx* c, size_t bytes)
{
    if (c->rec_bytes >= bytes) return 0;
    for (int b = 0; b < 2; b++) {
        if (c->rec_pinned[b]) cudaFreeHost(c->rec_pinned[b]);
        if (c->rec_dev[b]) cudaFree(c->rec_dev[b]);
        c->rec_pinned[b] = c->rec_dev[b] = nullptr;
    }
    c->rec_bytes = 0;
    for (int b = 0; b < 2; b++) {
        CK(cudaMallocHost(&c->rec_pinned[b], bytes));
        CK(cudaMalloc(&c->rec_dev[b], bytes + sizeof(RecMember) * kMaxRecMembers));
        if (!c->rec_ev[b]) CK(cudaEventCreateWithFlags(&c->rec_ev[b], cudaEventDisableTiming));
    }
    c->rec_bytes = bytes;
    return 0;
}

// n caller records of `stride` bytes (8-byte aligned) -> the device arrays of
// `tab`, in chunks: a chunk is copied into a pinned buffer on several host
// threads while the previous one crosses PCIe and k_rec_unpack scatters it
// With `keep` non-null the records are also copied there (n x stride bytes),
// in the same pass over the caller's array.
int push_records(sphgpu_ctx* c, const char* base, int n, size_t stride, const std::vector<RecMember>& tab,
                 char* keep = nullptr)
{
    int r = ensure_rec_staging(c, std::max((size_t)kRecChunk * stride, c->rec_bytes));
    if (r) return r;
    CK(cudaStreamSynchronize(c->st));
    RecMember* dtab[2];
    for (int b = 0; b < 2; b++) {
        dtab[b] = reinterpret_cast<RecMember*>(static_cast<char*>(c->rec_dev[b]) + c->rec_bytes);
        CK(cudaMemcpy(dtab[b], tab.data(), sizeof(RecMember) * tab.size(), cudaMemcpyHostToDevice));
    }
    int k = 0;
    for (int i0 = 0; i0 < n; i0 += kRecChunk, k++) {
        const int b = k & 1, cnt = std::min(kRecChunk, n - i0);
        if (k >= 2) CK(cudaEventSynchronize(c->rec_ev[b]));
        char* pin = static_cast<char*>(c->rec_pinned[b]);
        const char* src = base + (size_t)i0 * stride;
        const size_t bytes = (size_t)cnt * stride;
        char* kp = keep ? keep + (size_t)i0 * stride : nullptr;
        par_for(bytes, [&](size_t a, size_t e) {
            std::memcpy(pin + a, src + a, e - a);
            if (kp) std::memcpy(kp + a, src + a, e - a);
        });
        CK(cudaMemcpyAsync(c->rec_dev[b], pin, bytes, cudaMemcpyHostToDevice, c->st));
        k_rec_unpack<<<(cnt + 255) / 256, 256, 0, c->st>>>(static_cast<const char*>(c->rec_dev[b]), stride, i0, cnt,
                                                           c->N, dtab[b], (int)tab.size());
        CK(cudaGetLastError());
        CK(cudaEventRecord(c->rec_ev[b], c->st));
    }
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

}  // namespace

extern "C" {

int sphgpu_abi_version(void) { return SPHGPU_ABI_VERSION; }

int sphgpu_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

const char* sphgpu_error_string(int code)
{
    switch (code) {
    case 0: return "no error";
    case 3: return "particle outside the cell grid (parttocell)";
    case 5: return "more than 99 neighbours (partisearching)";
    case SPHGPU_E_ARG: return "bad argument";
    case SPHGPU_E_CUDA: return "CUDA runtime error";
    case SPHGPU_E_NODEVICE: return "no CUDA device";
    case SPHGPU_E_UNSUPPORTED: return "flag combination not supported by the engine";
    case SPHGPU_E_STATE: return "call order (state not uploaded)";
    case SPHGPU_E_KL_TIMEOUT: return "a tensor-core completion wait expired";
    default: return "unknown error";
    }
}

int sphgpu_last_create_error(void) { return g_create_error; }

sphgpu_ctx* sphgpu_create(const sphgpu_params* P, int device)
{
    g_create_error = check_params(P);
    if (g_create_error) return nullptr;
    int ndev = sphgpu_device_count();
    if (ndev <= 0 || device < 0 || device >= ndev) { g_create_error = SPHGPU_E_NODEVICE; return nullptr; }
    sphgpu_ctx* c = new sphgpu_ctx();
    c->P = *P;
    c->device = device;
    c->N = P->ntotal;
    auto fail = [&](int code) { g_create_error = code; sphgpu_destroy(c); return (sphgpu_ctx*)nullptr; };
    if (cudaSetDevice(device) != cudaSuccess) return fail(SPHGPU_E_NODEVICE);
    // an error an earlier, unrelated call left as the last error (not a
    // sticky one, which every call below would report) is not this
    // context's: cleared, so that the launch checks below see their own
    cudaGetLastError();
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) return fail(SPHGPU_E_CUDA);
    cudaEventCreate(&c->ev0);
    cudaEventCreate(&c->ev1);
    const int N = c->N, M = P->ctotal + 4;
    Dev& d = c->d[0];
    fill_dev_params(d.p, P);
    DevState& s = d.s;
    int r = 0;
    r |= dalloc(c, &s.type, N); r |= dalloc(c, &s.matype, N); r |= dalloc(c, &s.etype, N); r |= dalloc(c, &s.permtype, N);
    r |= dalloc(c, &s.mass, N); r |= dalloc(c, &s.cd, N);
    r |= dalloc(c, &s.f_dens, N); r |= dalloc(c, &s.f_por, N); r |= dalloc(c, &s.f_vpu, N); r |= dalloc(c, &s.f_vis, N);
    r |= dalloc(c, &s.f_c, N); r |= dalloc(c, &s.f_smin, N); r |= dalloc(c, &s.f_tanfai, N); r |= dalloc(c, &s.f_bhtype, N);
    r |= dalloc(c, &s.s_e, N); r |= dalloc(c, &s.s_poi, N); r |= dalloc(c, &s.s_eps0, N); r |= dalloc(c, &s.s_dens, N);
    r |= dalloc(c, &s.s_kapa, N); r |= dalloc(c, &s.s_por, N); r |= dalloc(c, &s.s_vpu, N); r |= dalloc(c, &s.s_cop, N);
    r |= dalloc(c, &s.s_sitas, N); r |= dalloc(c, &s.s_sitar, N); r |= dalloc(c, &s.s_ds, N);
    r |= dalloc(c, &s.s_c, N); r |= dalloc(c, &s.s_fs, N);
    r |= dalloc(c, &s.s_ann, N); r |= dalloc(c, &s.s_zmf, N); r |= dalloc(c, &s.s_ramda, N); r |= dalloc(c, &s.s_sme0, N);
    r |= dalloc(c, &s.s_yalf, N); r |= dalloc(c, &s.s_ykap, N); r |= dalloc(c, &s.s_yalf_dil, N);
    r |= dalloc(c, &s.xh, 4 * (size_t)N); r |= dalloc(c, &s.xh_next, 4 * (size_t)N); r |= dalloc(c, &s.xs, 4 * (size_t)N); r |= dalloc(c, &s.xsf, 4 * (size_t)N);
    r |= dalloc(c, &s.de, 6 * (size_t)N); r |= dalloc(c, &s.we, 6 * (size_t)N); r |= dalloc(c, &s.color, N);
    r |= dalloc(c, &s.sr, 8 * (size_t)N);
    r |= dalloc(c, &s.eps_tmp, 6 * (size_t)N); r |= dalloc(c, &s.sig_tmp, 6 * (size_t)N);
    r |= alloc_optional(c, P);
    r |= dalloc(c, &s.vx, 3 * (size_t)N); r |= dalloc(c, &s.vx_next, 4 * (size_t)N);
    r |= dalloc(c, &s.vxp, 3 * (size_t)N); r |= dalloc(c, &s.axp, 3 * (size_t)N); r |= dalloc(c, &s.ax, 3 * (size_t)N);
    r |= dalloc(c, &s.ux, 3 * (size_t)N);
    r |= dalloc(c, &s.rho, N); r |= dalloc(c, &s.rho_c, 2 * (size_t)N); r |= dalloc(c, &s.svr, 4 * (size_t)N); r |= dalloc(c, &s.pmr, 4 * (size_t)N); r |= dalloc(c, &s.dr4, 4 * (size_t)N); r |= dalloc(c, &s.rrho, 4 * (size_t)N); r |= dalloc(c, &s.nv, 4 * (size_t)N); r |= dalloc(c, &s.rhop, N); r |= dalloc(c, &s.pre, N);
    r |= dalloc(c, &s.prep, N); r |= dalloc(c, &s.porosity, N); r |= dalloc(c, &s.poro_cop, N); r |= dalloc(c, &s.e, N);
    r |= dalloc(c, &s.sig, 6 * (size_t)N); r |= dalloc(c, &s.sig_next, 6 * (size_t)N);
    r |= dalloc(c, &s.eps, 6 * (size_t)N); r |= dalloc(c, &s.adps, 6 * (size_t)N);
    r |= dalloc(c, &s.tssig, 6 * (size_t)N); r |= dalloc(c, &s.tsqc, N);
    r |= dalloc(c, &s.dsatu, N); r |= dalloc(c, &s.suct, N);
    r |= dalloc(c, &s.satu, N); r |= dalloc(c, &s.cop, N); r |= dalloc(c, &s.prew, N); r |= dalloc(c, &s.prea, N);
    r |= dalloc(c, &s.interf, 3 * (size_t)N); r |= dalloc(c, &s.interfss, 3 * (size_t)N); r |= dalloc(c, &s.strep, 3 * (size_t)N);
    r |= dalloc(c, &s.vsig, N); r |= dalloc(c, &s.veps, N); r |= dalloc(c, &s.divq, N); r |= dalloc(c, &s.divr, N);
    r |= dalloc(c, &s.meps, N);
    r |= dalloc(c, &s.i2o, N); r |= dalloc(c, &s.o2i, N);
    r |= dalloc(c, &s.cell, N); r |= dalloc(c, &s.key_in, N); r |= dalloc(c, &s.key_out, N);
    r |= dalloc(c, &s.val_in, N); r |= dalloc(c, &s.pid_sorted, N);
    r |= dalloc(c, &s.cstart, M); r |= dalloc(c, &s.cend, M);
    r |= dalloc(c, &s.nnb, N); r |= dalloc(c, &s.nbr, (size_t)SPH_NB_CAP * N);
    r |= dalloc(c, &s.nps, N); r |= dalloc(c, &s.sortpos, N); r |= dalloc(c, &s.pts, N);
    if (!s.accb) r |= dalloc(c, &s.accb, 9 * (size_t)N);   // (19N when alloc_optional sized it for vibration)
    r |= dalloc(c, &s.nbrs, (size_t)SPH_NB_CAP * N);
    r |= dalloc(c, &s.nbm, 10 * (size_t)N);
    r |= dalloc(c, &s.nbw, 4 * (size_t)SPH_NB_CAP * N);
    r |= dalloc(c, &s.err, 1); r |= dalloc(c, &s.step, 1);
    r |= dalloc(c, &s.dtv, 1); r |= dalloc(c, &s.dtmin, 1); r |= dalloc(c, &s.nrain, 1); r |= dalloc(c, &s.tsim, 1);
    if (r) return fail(SPHGPU_E_CUDA);
    // cell_info() constructor values (Class_NNPS.cpp:68-72): the range of the
    // last cell, which the reference never resets, starts from them
    std::vector<int> st(M, 2000000), en(M, -2000000);
    if (cudaMemcpyAsync(s.cstart, st.data(), sizeof(int) * M, cudaMemcpyHostToDevice, c->st) != cudaSuccess ||
        cudaMemcpyAsync(s.cend, en.data(), sizeof(int) * M, cudaMemcpyHostToDevice, c->st) != cudaSuccess)
        return fail(SPHGPU_E_CUDA);
    int one = 1;
    if (cudaMemcpyAsync(s.step, &one, sizeof(int), cudaMemcpyHostToDevice, c->st) != cudaSuccess)
        return fail(SPHGPU_E_CUDA);
    k_order_identity<<<(N + 255) / 256, 256, 0, c->st>>>(s.i2o, s.o2i, N);
    if (cudaPeekAtLastError() != cudaSuccess) return fail(SPHGPU_E_CUDA);
    c->end_bit = end_bit_for(P->ctotal);
    c->sort_bytes = sphk_sort_temp_bytes(N, c->end_bit);
    if (cudaMalloc(&c->sort_tmp, c->sort_bytes + 256) != cudaSuccess) return fail(SPHGPU_E_CUDA);
    c->allocs.push_back(c->sort_tmp);
    // the staging buffers of the record transfers, sized for Particle and
    // material records, allocated with the rest of the state
    if (ensure_rec_staging(c, (size_t)kRecChunk * std::max({(size_t)kParticleBytes, sizeof(sphgpu_fluid),
                                                             sizeof(sphgpu_soil)})))
        return fail(SPHGPU_E_CUDA);
    // the host copies the record calls fill (positions, types, material
    // records): their storage reserved and its pages touched here, so that
    // the transfers copy at memory speed instead of taking a page fault per
    // 4 KB.  They stay empty (not set) until a call fills them, and sizing
    // them to N then reuses this storage.
    if (cudaMallocHost(&c->mat_pinned, sizeof(double) * 4 * (size_t)N) != cudaSuccess) return fail(SPHGPU_E_CUDA);
    c->h_x.reserve((size_t)N * 3);
    c->h_type.reserve(N);
    c->h_matype.reserve(N);
    c->h_fluid.reserve(N);
    c->h_soil.reserve(N);
    prefault(c->h_x.data(), sizeof(double) * 3 * (size_t)N);
    prefault(c->h_type.data(), sizeof(int) * (size_t)N);
    prefault(c->h_matype.data(), sizeof(int) * (size_t)N);
    prefault(c->h_fluid.data(), sizeof(sphgpu_fluid) * (size_t)N);
    prefault(c->h_soil.data(), sizeof(sphgpu_soil) * (size_t)N);
    c->d[1] = c->d[0];
    std::swap(c->d[1].s.xh, c->d[1].s.xh_next);
    std::swap(c->d[1].s.sig, c->d[1].s.sig_next);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return fail(SPHGPU_E_CUDA);
    return c;
}

void sphgpu_destroy(sphgpu_ctx* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    for (int b = 0; b < 2; b++)
        if (c->out_th[b].joinable()) c->out_th[b].join();
    for (int b = 0; b < 2; b++) {
        if (c->out_host[b]) cudaFreeHost(c->out_host[b]);
        if (c->out_ev[b]) cudaEventDestroy(c->out_ev[b]);
    }
    if (c->out_st) cudaStreamDestroy(c->out_st);
    if (c->st) cudaStreamSynchronize(c->st);
    invalidate_graphs(c);
    for (void* p : c->allocs) cudaFree(p);
    if (c->perm_tmp) cudaFree(c->perm_tmp);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->mat_pinned) cudaFreeHost(c->mat_pinned);
    for (int b = 0; b < 2; b++) {
        if (c->rec_pinned[b]) cudaFreeHost(c->rec_pinned[b]);
        if (c->rec_dev[b]) cudaFree(c->rec_dev[b]);
        if (c->rec_ev[b]) cudaEventDestroy(c->rec_ev[b]);
    }
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
}

int sphgpu_get_params(const sphgpu_ctx* c, sphgpu_params* out)
{
    if (!c || !out) return SPHGPU_E_ARG;
    *out = c->P;
    return 0;
}

int sphgpu_get_step(const sphgpu_ctx* c) { return c ? c->l_host : -1; }

int sphgpu_set_precision(sphgpu_ctx* c, int mode)
{
    if (!c || (mode != SPHGPU_PREC_FP64 && mode != SPHGPU_PREC_FP32_BULK)) return SPHGPU_E_ARG;
    if (mode != c->precision) {
        cudaSetDevice(c->device);
        CK(cudaStreamSynchronize(c->st));
        c->precision = mode;
        for (int p = 0; p < 2; p++) c->d[p].p.bulk = (mode == SPHGPU_PREC_FP32_BULK) ? 1 : 0;
        invalidate_graphs(c);
    }
    return 0;
}

int sphgpu_get_precision(const sphgpu_ctx* c) { return c ? c->precision : -1; }

int sphgpu_set_step(sphgpu_ctx* c, int l)
{
    if (!c) return SPHGPU_E_ARG;
    cudaSetDevice(c->device);
    CK(cudaMemcpyAsync(c->d[0].s.step, &l, sizeof(int), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->l_host = l;
    c->part_done = 0;
    return 0;
}

int sphgpu_field_info(const char* name, int* ncomp, int* elem_type)
{
    const FieldDef* f = find_field(name);
    if (!f) return SPHGPU_E_ARG;
    if (ncomp) *ncomp = f->ncomp;
    if (elem_type) *elem_type = f->is_int;
    return 0;
}

int sphgpu_set_field(sphgpu_ctx* c, const char* name, const void* host, size_t count)
{
    const FieldDef* f = find_field(name);
    if (!c || !f || !host) return SPHGPU_E_ARG;
    const int N = c->N, nc = f->ncomp;
    if (count != (size_t)N * nc) return SPHGPU_E_ARG;
    cudaSetDevice(c->device);
    if (const int ro = to_caller_order(c)) return ro;
    if (std::strcmp(name, "x") == 0) {
        c->h_x.assign((const double*)host, (const double*)host + (size_t)N * 3);
        c->x_tracked = true;
        return 0;
    }
    if (std::strcmp(name, "xp") == 0 || std::strcmp(name, "hl") == 0) {
        // (x, y, z, h) records: read-modify-write of the current buffer
        std::vector<double> rec((size_t)N * 4);
        double* xh = c->d[c->parity].s.xh;
        CK(cudaMemcpy(rec.data(), xh, sizeof(double) * rec.size(), cudaMemcpyDeviceToHost));
        const double* h = (const double*)host;
        if (nc == 3) {
            for (int i = 0; i < N; i++)
                for (int k = 0; k < 3; k++) rec[(size_t)i * 4 + k] = h[(size_t)i * 3 + k];
        } else {
            for (int i = 0; i < N; i++) rec[(size_t)i * 4 + 3] = h[i];
        }
        CK(cudaMemcpy(xh, rec.data(), sizeof(double) * rec.size(), cudaMemcpyHostToDevice));
        return 0;
    }
    const size_t esz = f->is_int ? 4 : 8;
    int r = ensure_pinned(c, count * esz);
    if (r) return r;
    // particle-major -> component-major
    if (f->is_int) {
        std::memcpy(c->pinned, host, count * esz);
        const int* h = (const int*)host;
        if (std::strcmp(name, "type") == 0) { c->h_type.assign(h, h + N); update_static_params(c); }
        if (std::strcmp(name, "matype") == 0) { c->h_matype.assign(h, h + N); update_static_params(c); }
    } else {
        const double* h = (const double*)host;
        double* o = (double*)c->pinned;
        for (int k = 0; k < nc; k++)
            for (int i = 0; i < N; i++) o[(size_t)k * N + i] = h[(size_t)i * nc + k];
    }
    void* dst = field_ptr(c, name);
    if (!dst) return SPHGPU_E_ARG;
    CK(cudaMemcpyAsync(dst, c->pinned, count * esz, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

int sphgpu_get_field(sphgpu_ctx* c, const char* name, void* host, size_t count)
{
    const FieldDef* f = find_field(name);
    if (!c || !f || !host) return SPHGPU_E_ARG;
    const int N = c->N, nc = f->ncomp;
    if (count != (size_t)N * nc) return SPHGPU_E_ARG;
    cudaSetDevice(c->device);
    if (const int ro = to_caller_order(c)) return ro;
    if (std::strcmp(name, "x") == 0) {
        // Particle::x is written only by update (CPP_12-1-update.cpp:30-47):
        // after a step it equals xp for moving particles and keeps its
        // uploaded value for the rest
        std::vector<double> xp((size_t)N * 3);
        int r = sphgpu_get_field(c, "xp", xp.data(), xp.size());
        if (r) return r;
        double* o = (double*)host;
        for (size_t q = 0; q < xp.size(); q++) o[q] = c->x_tracked ? c->h_x[q] : 0.0;
        if (c->l_host > 1 && !c->h_type.empty()) {
            for (int i = 0; i < N; i++) {
                const int t = c->h_type[i], m = c->h_matype.empty() ? 0 : c->h_matype[i];
                if (t != 0 || m == 2 || m == 3 || m == 4 || m == 5)
                    for (int k = 0; k < c->P.ndim; k++) o[(size_t)i * 3 + k] = xp[(size_t)i * 3 + k];
            }
        }
        return 0;
    }
    if (std::strcmp(name, "xp") == 0 || std::strcmp(name, "hl") == 0) {
        std::vector<double> rec((size_t)N * 4);
        CK(cudaMemcpy(rec.data(), c->d[c->parity].s.xh, sizeof(double) * rec.size(), cudaMemcpyDeviceToHost));
        double* o = (double*)host;
        if (nc == 3) {
            for (int i = 0; i < N; i++)
                for (int k = 0; k < 3; k++) o[(size_t)i * 3 + k] = rec[(size_t)i * 4 + k];
        } else {
            for (int i = 0; i < N; i++) o[i] = rec[(size_t)i * 4 + 3];
        }
        return 0;
    }
    const size_t esz = f->is_int ? 4 : 8;
    int r = ensure_pinned(c, count * esz);
    if (r) return r;
    void* src = field_ptr(c, name);
    if (!src) return SPHGPU_E_ARG;
    CK(cudaMemcpyAsync(c->pinned, src, count * esz, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (f->is_int) {
        std::memcpy(host, c->pinned, count * esz);
    } else {
        const double* s = (const double*)c->pinned;
        double* o = (double*)host;
        for (int k = 0; k < nc; k++)
            for (int i = 0; i < N; i++) o[(size_t)i * nc + k] = s[(size_t)k * N + i];
    }
    return 0;
}

int sphgpu_set_materials(sphgpu_ctx* c, const sphgpu_fluid* fl, const sphgpu_soil* so, int n)
{
    if (!c || n != c->N) return SPHGPU_E_ARG;
    cudaSetDevice(c->device);
    if (const int ro = to_caller_order(c)) return ro;
    // the host copies (K-L fields rewrite members of them and upload them
    // again), written in the same pass that stages the caller's records for
    // the device; the per-particle constants below read the caller's records
    char* keep_f = nullptr;
    char* keep_s = nullptr;
    if (fl && fl != c->h_fluid.data()) {
        c->h_fluid.resize(n);
        keep_f = reinterpret_cast<char*>(c->h_fluid.data());
    }
    if (so && so != c->h_soil.data()) {
        c->h_soil.resize(n);
        keep_s = reinterpret_cast<char*>(c->h_soil.data());
    }
    const int N = c->N;
    DevState& s = c->d[0].s;
    // the per-particle constants, in the pinned block (N doubles each)
    double* buf = c->mat_pinned;
    auto put = [&](double* dst, const double* src) -> int {
        CK(cudaMemcpyAsync(dst, src, sizeof(double) * N, cudaMemcpyHostToDevice, c->st));
        CK(cudaStreamSynchronize(c->st));
        return 0;
    };
    // a particle whose inputs have the bits of the previous particle's takes
    // its results (particles of one material share their records)
    auto same = [](double a, double b) { return std::memcmp(&a, &b, sizeof(double)) == 0; };
    auto m = [](size_t off, void* dst, int kind = 0) { return RecMember{(int)off, 1, kind, 0, dst}; };
    int r = 0;
    if (fl) {
        const std::vector<RecMember> tab = {
            m(offsetof(sphgpu_fluid, dens), s.f_dens), m(offsetof(sphgpu_fluid, porosity), s.f_por),
            m(offsetof(sphgpu_fluid, vpu), s.f_vpu), m(offsetof(sphgpu_fluid, vis), s.f_vis),
            m(offsetof(sphgpu_fluid, c), s.f_c), m(offsetof(sphgpu_fluid, strain_min), s.f_smin),
            m(offsetof(sphgpu_fluid, bhtype), s.f_bhtype, 1)};
        r = push_records(c, reinterpret_cast<const char*>(fl), N, sizeof(sphgpu_fluid), tab, keep_f);
        if (r) {
            if (keep_f) c->h_fluid.clear();   // not filled
            return r;
        }
        // Bingham friction: tan of the angle, CPP_7-2-constitutive.cpp:42-43
        par_for(N, [&](size_t a, size_t b) {
            double lf = 0.0, v = 0.0;
            for (size_t i = a; i < b; i++) {
                if (i == a || !same(fl[i].fai, lf)) { lf = fl[i].fai; v = std::tan(lf * 0.0174532925199); }
                buf[i] = v;
            }
        });
        r |= put(s.f_tanfai, buf);
    }
    if (so) {
        const std::vector<RecMember> tab = {
            m(offsetof(sphgpu_soil, e), s.s_e), m(offsetof(sphgpu_soil, poi), s.s_poi),
            m(offsetof(sphgpu_soil, eps0), s.s_eps0), m(offsetof(sphgpu_soil, dens), s.s_dens),
            m(offsetof(sphgpu_soil, kapa), s.s_kapa), m(offsetof(sphgpu_soil, porosity), s.s_por),
            m(offsetof(sphgpu_soil, vpu), s.s_vpu), m(offsetof(sphgpu_soil, cop), s.s_cop),
            m(offsetof(sphgpu_soil, sitas), s.s_sitas), m(offsetof(sphgpu_soil, sitar), s.s_sitar),
            m(offsetof(sphgpu_soil, ds), s.s_ds), m(offsetof(sphgpu_soil, c), s.s_c),
            m(offsetof(sphgpu_soil, fs), s.s_fs), m(offsetof(sphgpu_soil, ann), s.s_ann),
            m(offsetof(sphgpu_soil, zmf), s.s_zmf), m(offsetof(sphgpu_soil, ramda), s.s_ramda),
            m(offsetof(sphgpu_soil, sme0), s.s_sme0)};
        r = push_records(c, reinterpret_cast<const char*>(so), N, sizeof(sphgpu_soil), tab, keep_s);
        if (r) {
            if (keep_s) c->h_soil.clear();   // not filled
            return r;
        }
        // Drucker-Prager cone constants with the reference's own libm calls
        // (dpmodel1 / dpmodel_bui / DPModel_check, CPP_8-1-consfactor.cpp:294-349,
        // 461-529, 783-803); they depend only on the material record.
        double* ya = buf + N;
        double* yk = buf + 2 * (size_t)N;
        double* yd = buf + 3 * (size_t)N;
        par_for(N, [&](size_t a, size_t b) {
            double lf = 0.0, lb = 0.0, lc = 0.0, ls = 0.0, va = 0.0, vk = 0.0, vd = 0.0;
            for (size_t i = a; i < b; i++) {
                const sphgpu_soil& q = so[i];
                if (i == a || !same(q.fai, lf) || !same(q.beta, lb) || !same(q.c, lc) || !same(q.fs, ls)) {
                    lf = q.fai; lb = q.beta; lc = q.c; ls = q.fs;
                    const double fai = std::atan(std::tan(q.fai * 0.0174532925166667) / q.fs);
                    const double fai_dil = std::atan(std::tan(q.beta * 0.0174532925166667) / q.fs);
                    const double ci = q.c / q.fs;
                    const double sf = std::sin(fai), sd = std::sin(fai_dil);
                    va = sf / std::sqrt(9.0 + 3.0 * sf * sf);
                    vk = 3.0 * ci * std::cos(fai) / std::sqrt(9.0 + 3.0 * sf * sf);
                    // dilatancy slope, used by the Bui form (matype % 10 == 5) only
                    vd = sd / std::sqrt(9.0 + 3.0 * sd * sd);
                }
                ya[i] = va; yk[i] = vk; yd[i] = vd;
            }
        });
        r |= put(s.s_yalf, ya);
        r |= put(s.s_ykap, yk);
        r |= put(s.s_yalf_dil, yd);
        // the members only unsaturated Cam-clay (matype % 10 == 3), the
        // saturation pass and fractional-order Cam-clay (8) read, allocated
        // on first use; pow(c, 4) of fractional_mcc with the host's libm
        // (CPP_8-5-consfactor-focc.cpp:158)
        bool need = c->P.flagum == 1 || c->P.flv > 0;
        for (int i = 0; i < N && !need && i < (int)c->h_matype.size(); i++) {
            const int mt = c->h_matype[i] % 10;
            need = (mt == 3 || mt == 8);
        }
        if (need && !s.s_ext) {
            double* q = nullptr;
            if (dalloc(c, &q, (size_t)SX_COUNT * N)) return SPHGPU_E_CUDA;
            for (int p = 0; p < 2; p++) c->d[p].s.s_ext = q;
            invalidate_graphs(c);
        }
        if (s.s_ext) {
            std::vector<double> ext((size_t)SX_COUNT * N);
            par_for(N, [&](size_t a, size_t b) {
                for (size_t i = a; i < b; i++) {
                    const sphgpu_soil& q = so[i];
                    const double v[SX_COUNT] = {q.epss, q.epsr, q.bnn, q.beta, q.sd, q.sw, q.c1, q.c2,
                                                q.g0, q.etao, q.zet, q.damp1, q.damp2, std::pow(q.c, 4)};
                    for (int k = 0; k < SX_COUNT; k++) ext[(size_t)k * N + i] = v[k];
                }
            });
            CK(cudaMemcpyAsync(s.s_ext, ext.data(), sizeof(double) * ext.size(), cudaMemcpyHostToDevice, c->st));
            CK(cudaStreamSynchronize(c->st));
        }
    }
    return r ? SPHGPU_E_CUDA : 0;
}

int sphgpu_particle_layout(const char* name, size_t* offset, int* ncomp)
{
    if (!name) return SPHGPU_E_ARG;
    for (const AosMember& m : kAos)
        if (std::strcmp(m.name, name) == 0) {
            if (offset) *offset = m.off;
            if (ncomp) *ncomp = find_field(name)->ncomp;
            return 0;
        }
    return SPHGPU_E_ARG;
}

// Records are moved in chunks through two pinned and two device buffers: the
// host copies a chunk of whole records (on several threads) while the
// previous chunk crosses PCIe and a kernel scatters its members into the
// device's component-major arrays (the reverse on download, where only the
// device-owned members of the caller's records are written).
// member by member through the field calls, for records that are not 8-byte
// aligned
int upload_by_fields(sphgpu_ctx* c, const char* base, int n, size_t stride)
{
    for (const AosMember& m : kAos) {
        const FieldDef* f = find_field(m.name);
        const size_t nc = f->ncomp;
        if (f->is_int) {
            std::vector<int> v((size_t)n);
            for (int i = 0; i < n; i++) std::memcpy(&v[i], base + (size_t)i * stride + m.off, 4);
            int r = sphgpu_set_field(c, m.name, v.data(), v.size());
            if (r) return r;
        } else {
            std::vector<double> v((size_t)n * nc);
            for (int i = 0; i < n; i++) std::memcpy(&v[(size_t)i * nc], base + (size_t)i * stride + m.off, 8 * nc);
            int r = sphgpu_set_field(c, m.name, v.data(), v.size());
            if (r) return r;
        }
    }
    return 0;
}

int download_by_fields(sphgpu_ctx* c, char* base, int n, size_t stride)
{
    for (const AosMember& m : kAos) {
        const FieldDef* f = find_field(m.name);
        const size_t nc = f->ncomp;
        if (f->is_int) {
            std::vector<int> v((size_t)n);
            int r = sphgpu_get_field(c, m.name, v.data(), v.size());
            if (r) return r;
            for (int i = 0; i < n; i++) std::memcpy(base + (size_t)i * stride + m.off, &v[i], 4);
        } else {
            std::vector<double> v((size_t)n * nc);
            int r = sphgpu_get_field(c, m.name, v.data(), v.size());
            if (r) return r;
            for (int i = 0; i < n; i++) std::memcpy(base + (size_t)i * stride + m.off, &v[(size_t)i * nc], 8 * nc);
        }
    }
    return 0;
}

int sphgpu_upload_particles(sphgpu_ctx* c, const void* particles, int n, size_t stride)
{
    if (!c || !particles || n != c->N || stride < kParticleBytes) return SPHGPU_E_ARG;
    if (const int ro = to_caller_order(c)) return ro;
    if (stride % 8 != 0 || ((uintptr_t)particles) % 8 != 0)
        return upload_by_fields(c, (const char*)particles, n, stride);
    cudaSetDevice(c->device);
    const char* base = (const char*)particles;
    std::vector<RecMember> tab;
    size_t P = 0;
    int r = rec_table(c, tab, &P);
    if (r) return r;
    // the host copies of x, type and matype
    c->h_x.resize((size_t)n * 3);
    c->h_type.resize(n);
    c->h_matype.resize(n);
    par_for((size_t)n, [&](size_t a, size_t b) {
        for (size_t i = a; i < b; i++) {
            const char* rec = base + i * stride;
            std::memcpy(&c->h_x[i * 3], rec + 0, 24);
            std::memcpy(&c->h_type[i], rec + 1048, 4);
            std::memcpy(&c->h_matype[i], rec + 1052, 4);
        }
    });
    c->x_tracked = true;
    r = push_records(c, base, n, stride, tab);
    if (r) return r;
    update_static_params(c);
    return 0;
}

int sphgpu_download_particles(sphgpu_ctx* c, void* particles, int n, size_t stride)
{
    if (!c || !particles || n != c->N || stride < kParticleBytes) return SPHGPU_E_ARG;
    if (const int ro = to_caller_order(c)) return ro;
    if (stride % 8 != 0 || ((uintptr_t)particles) % 8 != 0)
        return download_by_fields(c, (char*)particles, n, stride);
    cudaSetDevice(c->device);
    char* base = (char*)particles;
    std::vector<RecMember> tab;
    size_t P = 0;
    int r = rec_table(c, tab, &P);
    if (r) return r;
    r = ensure_rec_staging(c, std::max((size_t)kRecChunk * stride, (size_t)kRecChunk * P));
    if (r) return r;
    CK(cudaStreamSynchronize(c->st));
    RecMember* dtab[2];
    for (int b = 0; b < 2; b++) {
        dtab[b] = reinterpret_cast<RecMember*>(static_cast<char*>(c->rec_dev[b]) + c->rec_bytes);
        CK(cudaMemcpy(dtab[b], tab.data(), sizeof(RecMember) * tab.size(), cudaMemcpyHostToDevice));
    }
    // Particle::x as get_field("x") reports it: the uploaded x, and xp for
    // the particles update() moves once a step has run
    const bool moved = c->l_host > 1 && !c->h_type.empty();
    const int nd = c->P.ndim;
    auto scatter = [&](int i0, int cnt, const char* pin) {
        par_for((size_t)cnt, [&](size_t a, size_t e) {
            for (size_t t = a; t < e; t++) {
                const char* src = pin + t * P;
                const size_t i = (size_t)i0 + t;
                char* rec = base + i * stride;
                for (const RecMember& m : tab) {
                    const size_t len = (m.kind == 1) ? 4 : 8 * (size_t)m.nc;
                    std::memcpy(rec + m.off, src + m.pk, len);
                }
                double x[3];
                for (int q = 0; q < 3; q++) x[q] = c->x_tracked ? c->h_x[i * 3 + q] : 0.0;
                if (moved) {
                    const int ty = c->h_type[i], ma = c->h_matype.empty() ? 0 : c->h_matype[i];
                    if (ty != 0 || ma == 2 || ma == 3 || ma == 4 || ma == 5)
                        std::memcpy(x, rec + 24, sizeof(double) * nd);
                }
                std::memcpy(rec, x, 24);
            }
        });
    };
    int k = 0, prev_i0 = -1, prev_cnt = 0, prev_b = 0;
    for (int i0 = 0; i0 < n; i0 += kRecChunk, k++) {
        const int b = k & 1, cnt = std::min(kRecChunk, n - i0);
        k_rec_pack<<<(cnt + 255) / 256, 256, 0, c->st>>>(static_cast<char*>(c->rec_dev[b]), P, i0, cnt, c->N, dtab[b],
                                                         (int)tab.size());
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(c->rec_pinned[b], c->rec_dev[b], (size_t)cnt * P, cudaMemcpyDeviceToHost, c->st));
        CK(cudaEventRecord(c->rec_ev[b], c->st));
        if (prev_i0 >= 0) {
            CK(cudaEventSynchronize(c->rec_ev[prev_b]));
            scatter(prev_i0, prev_cnt, static_cast<const char*>(c->rec_pinned[prev_b]));
        }
        prev_i0 = i0; prev_cnt = cnt; prev_b = b;
    }
    if (prev_i0 >= 0) {
        CK(cudaEventSynchronize(c->rec_ev[prev_b]));
        scatter(prev_i0, prev_cnt, static_cast<const char*>(c->rec_pinned[prev_b]));
    }
    return 0;
}

namespace {

// Runs step l up to and including `upto` (1 parttocell, 2 partisearching,
// 3 the rest of the step through update) from where the method entries left
// it, with direct launches on the context's stream; returns the step's error
// code.  A completed step advances l and the parity as sphgpu_step does.
int run_parts(sphgpu_ctx* c, int upto)
{
    if (c->sticky) return c->sticky;
    if (upto >= 3) {
        int r = check_particles(c);
        if (r) return r;
    }
    cudaSetDevice(c->device);
    if (c->part_done == 0) {
        // the method entries run on the caller's order
        int r = to_caller_order(c);
        if (r) return r;
    }
    const Dev* d = &c->d[c->parity];
    int parts = 0;
    if (c->part_done < 1 && upto >= 1) parts |= 1;
    if (c->part_done < 2 && upto >= 2) parts |= 2;
    if (upto >= 3) parts |= 4;
    if (parts) sphk_enqueue_nnps_parts(d, c->sort_tmp, c->sort_bytes, c->end_bit, c->st, nullptr, parts);
    if (upto >= 3) {
        if (!c->regu && c->l_host % c->P.step_regu == 0) { c->regu = true; invalidate_graphs(c); }
        enqueue_physics(c, d, nullptr);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->st));
    int err = 0, l = 0;
    CK(cudaMemcpy(&err, c->d[0].s.err, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&l, c->d[0].s.step, sizeof(int), cudaMemcpyDeviceToHost));
    if (upto >= 3) {
        c->parity = (c->parity + (l - c->l_host)) & 1;
        c->l_host = l;
        if (err == 0) c->part_done = 0;
    } else if (err == 0) {
        c->part_done = upto;
    }
    return err;
}

}  // namespace

int sphgpu_parttocell(sphgpu_ctx* c)
{
    if (!c) return SPHGPU_E_ARG;
    if (c->part_done >= 1) return SPHGPU_E_STATE;     // step l's cell lists are already built
    return run_parts(c, 1);
}

int sphgpu_partisearching(sphgpu_ctx* c)
{
    if (!c) return SPHGPU_E_ARG;
    if (c->part_done >= 2) return SPHGPU_E_STATE;
    return run_parts(c, 2);
}

int sphgpu_update(sphgpu_ctx* c)
{
    if (!c) return SPHGPU_E_ARG;
    return run_parts(c, 3);
}

int sphgpu_update_params(sphgpu_ctx* c, const sphgpu_params* P)
{
    if (!c) return SPHGPU_E_ARG;
    if (!c->h_inst.empty()) return SPHGPU_E_STATE;   // a batched context keeps its instances' grids
    int r = check_params(P);
    if (r) return r;
    const sphgpu_params& Q = c->P;
    // the particle count and the cell grid the buffers were sized for stay
    if (P->ndim != Q.ndim || P->ntotal != Q.ntotal || P->cxm != Q.cxm || P->cym != Q.cym || P->czm != Q.czm ||
        P->ctotal != Q.ctotal || P->xmin != Q.xmin || P->ymin != Q.ymin || P->zmin != Q.zmin ||
        P->xmax != Q.xmax || P->ymax != Q.ymax || P->zmax != Q.zmax)
        return SPHGPU_E_ARG;
    cudaSetDevice(c->device);
    r = alloc_optional(c, P);
    if (r) return r;
    for (int p = 0; p < 2; p++) {
        DevParams& dp = c->d[p].p;
        const DevParams keep = dp;
        fill_dev_params(dp, P);
        dp.first_vbx_wall = keep.first_vbx_wall;
        dp.bulk = keep.bulk;
        dp.cfl_on = keep.cfl_on; dp.cfl_c = keep.cfl_c; dp.cfl_f = keep.cfl_f;
        dp.rain_lp = keep.rain_lp; dp.rain_vrain = keep.rain_vrain; dp.rain_press = keep.rain_press;
        dp.vib_ttime = keep.vib_ttime; dp.vib_st = keep.vib_st; dp.vib_ed = keep.vib_ed;
        dp.vib_nsteps = keep.vib_nsteps;
        for (int q = 0; q < TP_COUNT; q++) dp.tb[q] = keep.tb[q];
    }
    c->P = *P;
    invalidate_graphs(c);
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

sphgpu_ctx* sphgpu_create_batched(const sphgpu_params* shared, const sphgpu_instance* inst, int ninst, int device)
{
    g_create_error = SPHGPU_E_ARG;
    if (!shared || !inst || ninst <= 0) return nullptr;
    // rain rows are released from the end of the whole particle array
    if (shared->flr == 1) { g_create_error = SPHGPU_E_UNSUPPORTED; return nullptr; }
    // the instances follow one another in the particle order, each with a
    // grid of its own; the context numbers their cells one after another
    std::vector<InstGrid> tab(ninst);
    long long total = 0, cells = 0;
    for (int q = 0; q < ninst; q++) {
        const sphgpu_instance& a = inst[q];
        if (a.first != total || a.count <= 0) return nullptr;
        if (a.cxm <= 0 || a.cym <= 0 || a.czm <= 0 || (long long)a.cxm * a.cym * a.czm != a.ctotal) return nullptr;
        InstGrid& g = tab[q];
        g.xmin = a.xmin; g.ymin = a.ymin; g.zmin = a.zmin; g.xmax = a.xmax; g.ymax = a.ymax; g.zmax = a.zmax;
        g.cxm = a.cxm; g.cym = a.cym; g.czm = a.czm; g.ctotal = a.ctotal;
        g.cell_base = (int)cells;
        g.first = a.first; g.count = a.count;
        g.first_vbx_wall = a.first + a.count;
        total += a.count;
        cells += (long long)a.ctotal + 1;
        if (total >= (1LL << 28) || cells >= (1LL << 30)) { g_create_error = SPHGPU_E_UNSUPPORTED; return nullptr; }
    }
    sphgpu_params P = *shared;
    P.ntotal = (int)total;
    P.cxm = (int)cells; P.cym = 1; P.czm = 1; P.ctotal = (int)cells;
    P.xmin = tab[0].xmin; P.ymin = tab[0].ymin; P.zmin = tab[0].zmin;
    P.xmax = tab[0].xmax; P.ymax = tab[0].ymax; P.zmax = tab[0].zmax;
    sphgpu_ctx* c = sphgpu_create(&P, device);
    if (!c) return nullptr;
    c->h_inst = tab;
    std::vector<int> pinst((size_t)total);
    for (int q = 0; q < ninst; q++)
        for (int i = tab[q].first; i < tab[q].first + tab[q].count; i++) pinst[i] = q;
    int* d_pinst = nullptr;
    int r = dalloc(c, &c->d_inst, (size_t)ninst);
    r |= dalloc(c, &d_pinst, (size_t)total);
    if (!r) r |= cuda_fail(c, cudaMemcpyAsync(d_pinst, pinst.data(), sizeof(int) * total, cudaMemcpyHostToDevice,
                                              c->st), "cudaMemcpyAsync");
    if (r) {
        sphgpu_destroy(c);
        g_create_error = SPHGPU_E_CUDA;
        return nullptr;
    }
    for (int p = 0; p < 2; p++) {
        c->d[p].p.ninst = ninst;
        c->d[p].s.inst = c->d_inst;
        c->d[p].s.pinst = d_pinst;
    }
    update_static_params(c);
    if (c->sticky) {
        sphgpu_destroy(c);
        g_create_error = SPHGPU_E_CUDA;
        return nullptr;
    }
    g_create_error = 0;
    return c;
}

int sphgpu_instance_count(const sphgpu_ctx* c) { return c ? (int)c->h_inst.size() : -1; }

int sphgpu_step(sphgpu_ctx* c, int nsteps)
{
    if (!c || nsteps < 0) return SPHGPU_E_ARG;
    if (c->sticky) return c->sticky;
    if (nsteps == 0) return 0;
    int r = check_particles(c);
    if (r) return r;
    // a step the method entries began is completed first
    if (c->part_done) {
        r = run_parts(c, 3);
        if (r || nsteps == 1) return r;
        nsteps--;
    }
    // the regularisation passes (strain_regu / stress_regu) join the step
    // graphs from the first call whose steps include one with l % step_regu == 0
    if (!c->regu)
        for (long long l = c->l_host; l < (long long)c->l_host + nsteps; l++)
            if (l % c->P.step_regu == 0) { c->regu = true; invalidate_graphs(c); break; }
    cudaSetDevice(c->device);
    if (!c->exec[0] || !c->exec[1]) {
        r = build_graphs(c);
        if (r) return r;
    }
    const int l0 = c->l_host;
    CK(cudaEventRecord(c->ev0, c->st));
    for (int s = 0; s < nsteps; s++) {
        const int p = (c->parity + s) & 1;
        r = sort_if_due(c, p);
        if (r) return r;
        CK(cudaGraphLaunch(c->exec[p], c->st));
        c->since_sort++;
    }
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaStreamSynchronize(c->st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_ms = ms;
    c->last_launches = c->launches_per_step * nsteps;
    int err = 0, l = 0;
    CK(cudaMemcpy(&err, c->d[0].s.err, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&l, c->d[0].s.step, sizeof(int), cudaMemcpyDeviceToHost));
    c->parity = (c->parity + (l - l0)) & 1;
    c->l_host = l;
    return err;
}

int sphgpu_set_reorder(sphgpu_ctx* c, int every_steps)
{
    if (!c || every_steps < 0) return SPHGPU_E_ARG;
    c->reorder_every = every_steps;
    c->since_sort = 1L << 40;        // the first re-sort before the next step
    return 0;
}

int sphgpu_get_reorder(const sphgpu_ctx* c) { return c ? c->reorder_every : -1; }

int sphgpu_get_order(sphgpu_ctx* c, int* i2o)
{
    if (!c || !i2o) return SPHGPU_E_ARG;
    cudaSetDevice(c->device);
    CK(cudaMemcpyAsync(i2o, c->d[0].s.i2o, sizeof(int) * (size_t)c->N, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

double sphgpu_last_reorder_ms(const sphgpu_ctx* c) { return c ? c->reorder_ms : 0.0; }

int sphgpu_set_cfl(sphgpu_ctx* c, double cfl, double cfl_force)
{
    if (!c) return SPHGPU_E_ARG;
    if (cfl > 0.0 && !(cfl_force > 0.0)) return SPHGPU_E_ARG;
    cudaSetDevice(c->device);
    const int on = cfl > 0.0 ? 1 : 0;
    // the first step after turning it on runs with the input dt
    const double dt0 = c->P.dt;
    const unsigned long long inf = 0x7ff0000000000000ULL;
    CK(cudaMemcpyAsync(c->d[0].s.dtv, &dt0, sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->d[0].s.dtmin, &inf, sizeof(inf), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int p = 0; p < 2; p++) {
        c->d[p].p.cfl_on = on;
        c->d[p].p.cfl_c = on ? cfl : 0.0;
        c->d[p].p.cfl_f = on ? cfl_force : 0.0;
    }
    invalidate_graphs(c);
    return 0;
}

namespace {

// Checkpoint file: a header, every device-owned Particle member (as
// sphgpu_get_field gives it), the material records, and the device state
// outside Particle that a later step reads: the walls' per-phase velocities
// and stresses (cl_bndy_pair / clVar_Boundary), the range of the cell the
// reference never resets, and the rain and time-step words.
constexpr char kCkMagic[8] = {'S', 'P', 'H', 'G', 'P', 'U', 'C', 'K'};
constexpr uint32_t kCkVersion = 1;

struct CkHeader {
    char magic[8];
    uint32_t version, ndim;
    int32_t n, ctotal, step, precision, regu, cfl_on;
    double cfl_c, cfl_f;
    int32_t rain_set, has_fluid, has_soil, nextra;
    sphgpu_rain rain;
};

struct CkExtra { const char* name; void* ptr; size_t bytes; bool host; };

std::vector<CkExtra> ck_extras(sphgpu_ctx* c)
{
    const DevState& s = c->d[c->parity].s;
    const size_t N = (size_t)c->N;
    const size_t last = (size_t)c->P.ctotal;
    std::vector<CkExtra> v;
    auto add = [&](const char* name, void* p, size_t bytes) { if (p) v.push_back({name, p, bytes, false}); };
    add("vel_bndy", s.vel_bndy, 3 * N * 8);
    add("vb", s.vb, 12 * N * 8);
    add("vx_vb", s.vx_vb, 3 * N * 8);
    add("sb", s.sb, 24 * N * 8);
    add("cstart_last", s.cstart + last, 4);
    add("cend_last", s.cend + last, 4);
    add("nrain", s.nrain, 4);
    add("dtv", s.dtv, 8);
    add("dtmin", s.dtmin, 8);
    add("tsim", s.tsim, 8);
    add("stiff", s.stiff, N * 8);
    // the vibration table, from the host copies (sphgpu_set_vibration again
    // on load)
    if (c->vib_set) {
        v.push_back({"vib_par", c->vib_par, sizeof(c->vib_par), true});
        v.push_back({"vib_loads", c->vib_loads.data(), c->vib_loads.size() * 8, true});
    }
    return v;
}

}  // namespace

int sphgpu_checkpoint_save(sphgpu_ctx* c, const char* path)
{
    if (!c || !path) return SPHGPU_E_ARG;
    if (c->sticky) return c->sticky;
    if (c->part_done) return SPHGPU_E_STATE;          // between steps only
    if (const int ro = to_caller_order(c)) return ro;
    FILE* f = std::fopen(path, "wb");
    if (!f) return SPHGPU_E_ARG;
    int rc = 0;
    CkHeader h = {};
    std::memcpy(h.magic, kCkMagic, 8);
    h.version = kCkVersion;
    h.ndim = (uint32_t)c->P.ndim;
    h.n = c->N; h.ctotal = c->P.ctotal; h.step = c->l_host; h.precision = c->precision; h.regu = c->regu;
    h.cfl_on = c->d[0].p.cfl_on; h.cfl_c = c->d[0].p.cfl_c; h.cfl_f = c->d[0].p.cfl_f;
    h.rain_set = c->rain_set; h.rain = c->rain;
    h.has_fluid = c->h_fluid.empty() ? 0 : 1;
    h.has_soil = c->h_soil.empty() ? 0 : 1;
    std::vector<CkExtra> ex = ck_extras(c);
    h.nextra = (int32_t)ex.size();
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    std::vector<char> buf;
    for (const FieldDef& fd : kFields) {
        if (!ok) break;
        const size_t count = (size_t)c->N * fd.ncomp, bytes = count * (fd.is_int ? 4 : 8);
        buf.resize(bytes);
        rc = sphgpu_get_field(c, fd.name, buf.data(), count);
        if (rc) break;
        ok = std::fwrite(buf.data(), 1, bytes, f) == bytes;
    }
    if (!rc && ok && h.has_fluid) ok = std::fwrite(c->h_fluid.data(), sizeof(sphgpu_fluid), c->N, f) == (size_t)c->N;
    if (!rc && ok && h.has_soil) ok = std::fwrite(c->h_soil.data(), sizeof(sphgpu_soil), c->N, f) == (size_t)c->N;
    for (const CkExtra& e : ex) {
        if (rc || !ok) break;
        buf.resize(e.bytes);
        if (e.host) std::memcpy(buf.data(), e.ptr, e.bytes);
        else if (cuda_fail(c, cudaMemcpy(buf.data(), e.ptr, e.bytes, cudaMemcpyDeviceToHost), "cudaMemcpy")) {
            rc = SPHGPU_E_CUDA;
            break;
        }
        char name[16] = {};
        std::strncpy(name, e.name, 15);
        const uint64_t b = e.bytes;
        ok = std::fwrite(name, 1, 16, f) == 16 && std::fwrite(&b, 8, 1, f) == 1 &&
             std::fwrite(buf.data(), 1, e.bytes, f) == e.bytes;
    }
    if (std::fclose(f) != 0) ok = false;
    if (rc) return rc;
    return ok ? 0 : SPHGPU_E_ARG;
}

int sphgpu_checkpoint_load(sphgpu_ctx* c, const char* path)
{
    if (!c || !path) return SPHGPU_E_ARG;
    if (c->sticky) return c->sticky;
    if (const int ro = to_caller_order(c)) return ro;
    FILE* f = std::fopen(path, "rb");
    if (!f) return SPHGPU_E_ARG;
    CkHeader h;
    int rc = 0;
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, kCkMagic, 8) != 0 ||
        h.version != kCkVersion || (int)h.ndim != c->P.ndim || h.n != c->N || h.ctotal != c->P.ctotal) {
        std::fclose(f);
        return SPHGPU_E_ARG;
    }
    std::vector<char> buf;
    for (const FieldDef& fd : kFields) {
        const size_t count = (size_t)c->N * fd.ncomp, bytes = count * (fd.is_int ? 4 : 8);
        buf.resize(bytes);
        if (std::fread(buf.data(), 1, bytes, f) != bytes) { rc = SPHGPU_E_ARG; break; }
        rc = sphgpu_set_field(c, fd.name, buf.data(), count);
        if (rc) break;
    }
    std::vector<sphgpu_fluid> fl;
    std::vector<sphgpu_soil> so;
    if (!rc && h.has_fluid) {
        fl.resize(c->N);
        if (std::fread(fl.data(), sizeof(sphgpu_fluid), c->N, f) != (size_t)c->N) rc = SPHGPU_E_ARG;
    }
    if (!rc && h.has_soil) {
        so.resize(c->N);
        if (std::fread(so.data(), sizeof(sphgpu_soil), c->N, f) != (size_t)c->N) rc = SPHGPU_E_ARG;
    }
    if (!rc && (h.has_fluid || h.has_soil))
        rc = sphgpu_set_materials(c, h.has_fluid ? fl.data() : nullptr, h.has_soil ? so.data() : nullptr, c->N);
    if (!rc) rc = sphgpu_set_step(c, h.step);
    if (!rc) rc = sphgpu_set_precision(c, h.precision);
    if (!rc && h.rain_set) rc = sphgpu_set_rain(c, &h.rain);
    if (!rc && h.cfl_on) rc = sphgpu_set_cfl(c, h.cfl_c, h.cfl_f);
    // the device words and arrays last, over what the calls above set
    std::vector<CkExtra> ex = ck_extras(c);
    std::vector<double> vpar, vload;
    for (int q = 0; q < h.nextra && !rc; q++) {
        char name[16];
        uint64_t b = 0;
        if (std::fread(name, 1, 16, f) != 16 || std::fread(&b, 8, 1, f) != 1) { rc = SPHGPU_E_ARG; break; }
        name[15] = 0;
        buf.resize(b);
        if (std::fread(buf.data(), 1, b, f) != b) { rc = SPHGPU_E_ARG; break; }
        if (std::strcmp(name, "vib_par") == 0 || std::strcmp(name, "vib_loads") == 0) {
            std::vector<double>& dst = (name[4] == 'p') ? vpar : vload;
            dst.resize(b / 8);
            std::memcpy(dst.data(), buf.data(), dst.size() * 8);
            continue;
        }
        for (const CkExtra& e : ex)
            if (!e.host && std::strcmp(e.name, name) == 0 && e.bytes == b &&
                cuda_fail(c, cudaMemcpy(e.ptr, buf.data(), b, cudaMemcpyHostToDevice), "cudaMemcpy"))
                rc = SPHGPU_E_CUDA;
    }
    if (!rc && vpar.size() == 4 && c->P.flv >= 1) {
        const sphgpu_vibration v = {vpar[0], (int)vpar[1], vpar[2], vpar[3]};
        if (vload.size() == 3 * (size_t)v.nsteps) rc = sphgpu_set_vibration(c, &v, vload.data());
    }
    std::fclose(f);
    if (!rc && h.regu && !c->regu) { c->regu = true; invalidate_graphs(c); }
    return rc;
}

namespace {

constexpr int kOutCols = 49;    // output_total's 47 values, type and matype, per particle

// one row of output_total (CPP_14-2-output.cpp:78-131) per particle, as
// doubles in its column order: xp, ux, |ux|, then ax and vx for moving
// particles or interfss and interf for walls, pre, prea, prew, sig, strep,
// eps, adps, vsig, veps, meps, divq, divr, satu, suct, interfss, type, matype
__global__ void k_out_pack(Dev d, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, N = d.p.N;
    if (i == 0) out[(size_t)N * kOutCols] = *d.s.tsim;
    if (i >= N) return;
    const DevState& s = d.s;
    double* o = out + (size_t)s.i2o[i] * kOutCols;     // row of the caller's index
    const Pos p = load_pos(s.xh, i);
    o[0] = p.x; o[1] = p.y; o[2] = p.z;
    const double u0 = s.ux[i], u1 = s.ux[N + i], u2 = s.ux[2 * N + i];
    o[3] = u0; o[4] = u1; o[5] = u2;
    o[6] = sqrt(u0 * u0 + u1 * u1 + u2 * u2);
    const int t = s.type[i];
    for (int k = 0; k < 3; k++) {
        o[7 + k] = (t != 0) ? s.ax[k * N + i] : s.interfss[k * N + i];
        o[10 + k] = (t != 0) ? s.vx[k * N + i] : s.interf[k * N + i];
    }
    o[13] = s.pre[i]; o[14] = s.prea[i]; o[15] = s.prew[i];
    for (int k = 0; k < 6; k++) o[16 + k] = s.sig[k * N + i];
    for (int k = 0; k < 3; k++) o[22 + k] = s.strep[k * N + i];
    for (int k = 0; k < 6; k++) o[25 + k] = s.eps[k * N + i];
    for (int k = 0; k < 6; k++) o[31 + k] = s.adps[k * N + i];
    o[37] = s.vsig[i]; o[38] = s.veps[i]; o[39] = s.meps[i]; o[40] = s.divq[i]; o[41] = s.divr[i];
    o[42] = s.satu[i]; o[43] = s.suct[i];
    for (int k = 0; k < 3; k++) o[44 + k] = s.interfss[k * N + i];
    o[47] = (double)t;
    o[48] = (double)s.matype[i];
}

// output_total's file, written from the packed rows (its name, header and
// row format are the reference's, so the two files compare byte for byte)
int write_odb(const char* dir, int l, const double* rows, int n)
{
    char path[1024];
    std::snprintf(path, sizeof(path), "%s/data-%010d.odb", dir, l);
    FILE* f = std::fopen(path, "w");
    if (!f) return SPHGPU_E_ARG;
    static const char* kStars =
        "*************************************************************************************************\n";
    std::fputs(kStars, f);
    std::fprintf(f, "%10d %14.6e\n", l, rows[(size_t)n * kOutCols]);
    // rows formatted in parallel, in chunks, and written in order
    const int chunk = 65536;
    const int nchunk = (n + chunk - 1) / chunk;
    std::vector<std::string> text(nchunk);
    par_for((size_t)nchunk, [&](size_t a, size_t b) {
        char line[1024];
        for (size_t q = a; q < b; q++) {
            std::string& out = text[q];
            const int i0 = (int)q * chunk, i1 = std::min(n, i0 + chunk);
            out.reserve((size_t)(i1 - i0) * 700);
            for (int i = i0; i < i1; i++) {
                const double* o = rows + (size_t)i * kOutCols;
                const int len = std::snprintf(line, sizeof(line),
                    "%5d %14.6e %14.6e %14.6e %14.6e %14.6e %14.6e "
                    "%14.6e %14.6e %14.6e %14.6e %14.6e %14.6e %14.6e "
                    "%14.6e %14.6e %14.6e %14.6e %14.6e %14.6e "
                    "%14.6e %14.6e %14.6e %14.6e %14.6e %14.6e "
                    "%14.6e %14.6e %14.6e %14.6e %14.6e %14.6e "
                    "%14.6e %14.6e %14.6e %14.6e %14.6e %14.6e "
                    "%14.6e %14.6e %14.6e %14.6e  %14.6e %14.6e "
                    "%14.6e %14.6e %14.6e "
                    "%14.6e %4d %4d\n",
                    i + 1, o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7], o[8], o[9], o[10], o[11], o[12],
                    o[13], o[14], o[15], o[16], o[17], o[18], o[19], o[20], o[21], o[22], o[23], o[24],
                    o[25], o[26], o[27], o[28], o[29], o[30], o[31], o[32], o[33], o[34], o[35], o[36],
                    o[37], o[38], o[39], o[40], o[41], o[42], o[43], o[44], o[45], o[46], (int)o[47],
                    (int)o[48]);
                out.append(line, (size_t)len);
            }
        }
    });
    bool ok = true;
    for (const std::string& t : text) ok = ok && std::fwrite(t.data(), 1, t.size(), f) == t.size();
    std::fputs(kStars, f);
    if (std::fclose(f) != 0) ok = false;
    return ok ? 0 : SPHGPU_E_ARG;
}

// the ten-character step number of output_impact's file name
// (CPP_14-2-output.cpp:150-181): zero-padded below 1e8, empty from there on
std::string step10(int l)
{
    if (l < 0 || l >= 100000000) return std::string();
    char b[16];
    std::snprintf(b, sizeof(b), "%010d", l);
    return std::string(b);
}

// output_flowdist (CPP_14-2-output.cpp:222-320): each phase's extent per axis,
// appended to "Flowing distance.dat"
int append_flowdist(const char* dir, int l, const double* rows, int n)
{
    double mx[4][3], mn[4][3];
    for (int p = 0; p < 4; p++)
        for (int k = 0; k < 3; k++) { mn[p][k] = 10000.0; mx[p][k] = -10000.0; }
    for (int i = 0; i < n; i++) {
        const double* o = rows + (size_t)i * kOutCols;
        const int t = (int)o[47];
        if (t < 1 || t > 4) continue;
        for (int k = 0; k < 3; k++) {
            mx[t - 1][k] = std::fmax(o[k], mx[t - 1][k]);
            mn[t - 1][k] = std::fmin(o[k], mn[t - 1][k]);
        }
    }
    for (int p = 0; p < 4; p++)
        for (int k = 0; k < 3; k++) {
            if (std::fabs(mn[p][k] - 10000.0) < 0.0001) mn[p][k] = 0.0;
            if (std::fabs(mx[p][k] + 10000.0) < 0.0001) mx[p][k] = 0.0;
        }
    const std::string path = std::string(dir) + "/Flowing distance.dat";
    FILE* f = std::fopen(path.c_str(), "a");
    if (!f) return SPHGPU_E_ARG;
    std::fprintf(f, "\nStep%9d            X                       Y                      Z\n", l);
    std::fprintf(f, "-----------------------------------------------------------------------------------\n");
    std::fprintf(f, "                  max           min        max         min        max         min   \n");
    static const char* kRow[4] = {"Water Phase:   ", "Soil Phase:    ", "Air Phase:     ", "Structure:      "};
    for (int p = 0; p < 4; p++)
        std::fprintf(f, "%s%5.3e    %5.3e   %5.3e   %5.3e   %5.3e   %5.3e \n", kRow[p], mx[p][0], mn[p][0], mx[p][1],
                     mn[p][1], mx[p][2], mn[p][2]);
    return std::fclose(f) == 0 ? 0 : SPHGPU_E_ARG;
}

// output_impact (CPP_14-2-output.cpp:139-220): the walls of matype >= 1 into
// Impact-force<l>.inp, their force sum prew dr^(ndim-1) as a line of
// Total_Force.dat
int write_impact(const char* dir, int l, const double* rows, int n, int ndim, double dr)
{
    const std::string path = std::string(dir) + "/Impact-force" + step10(l) + ".inp";
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return SPHGPU_E_ARG;
    std::fprintf(f, "No.  X   Y  Z  Pre_Dens  Pre_water  Pre_Air  SIGXX  SIGYY  SIGZZ  SIGXY  SIGYZ  SIGZX\n");
    int row = 1;
    double total_f = 0.0;
    for (int i = 0; i < n; i++) {
        const double* o = rows + (size_t)i * kOutCols;
        if (!((int)o[47] == 0 && (int)o[48] >= 1)) continue;
        std::fprintf(f, "%5d %14.6e %14.6e %14.6e %14.6e %14.6e %14.6e %14.6e %14.6e %14.6e %14.6e %14.6e %14.6e \n",
                     row, o[0], o[1], o[2], o[13], o[15], o[14], o[16], o[17], o[18], o[19], o[20], o[21]);
        row += 1;
        total_f += o[15] * std::pow(dr, ndim - 1);
    }
    bool ok = std::fclose(f) == 0;
    const std::string tot = std::string(dir) + "/Total_Force.dat";
    FILE* g = std::fopen(tot.c_str(), "a");
    if (!g) return SPHGPU_E_ARG;
    std::fprintf(g, "Step%9d, Total force is %14.6e N\n", l, total_f);
    ok = (std::fclose(g) == 0) && ok;
    return ok ? 0 : SPHGPU_E_ARG;
}

// mgf (CPP_14-1-outmgf.cpp:12-104): a frame of AVS_MGF.mgf -- the cell box's
// edges, then one sphere of radius 1.1 dr per particle of types 0-4 and 7 in
// its phase's colour (the count line says every particle)
int append_mgf(const char* dir, int l, int fop, const double* rows, int n, int ndim, double dr0, const double bmin[3],
               const double bmax[3])
{
    const std::string path = std::string(dir) + "/AVS_MGF.mgf";
    FILE* f = std::fopen(path.c_str(), "a");
    if (!f) return SPHGPU_E_ARG;
    const double dr = 1.1 * dr0;
    std::fprintf(f, "step%d\n", (int)(l / fop));
    auto edge = [&](double x, double y, double z) {
        std::fprintf(f, "%6.4f %6.4f %6.4f %6.4f %6.4f %6.4f\n", x, y, z, 0.5, 0.5, 0.5);
    };
    if (ndim == 2) {
        std::fprintf(f, " disjoint line\n boundary\n color\n 8\n");
        const double c2[8][2] = {{bmin[0], bmin[1]}, {bmax[0], bmin[1]}, {bmax[0], bmin[1]}, {bmax[0], bmax[1]},
                                 {bmax[0], bmax[1]}, {bmin[0], bmax[1]}, {bmin[0], bmax[1]}, {bmin[0], bmin[1]}};
        for (int q = 0; q < 8; q++) edge(c2[q][0], c2[q][1], 0.0);
    } else if (ndim == 3) {
        std::fprintf(f, " disjoint line\n boundary\n color\n 24\n");
        // bottom, top (the bottom's square at zmax), then the four verticals
        const double sq[8][2] = {{bmin[0], bmin[1]}, {bmax[0], bmin[1]}, {bmax[0], bmin[1]}, {bmax[0], bmax[1]},
                                 {bmax[0], bmax[1]}, {bmin[0], bmax[1]}, {bmin[0], bmax[1]}, {bmin[0], bmin[1]}};
        for (int q = 0; q < 8; q++) edge(sq[q][0], sq[q][1], bmin[2]);
        for (int q = 0; q < 8; q++) edge(sq[q][0], sq[q][1], bmax[2]);
        const double vt[4][2] = {{bmin[0], bmin[1]}, {bmax[0], bmin[1]}, {bmax[0], bmax[1]}, {bmin[0], bmax[1]}};
        for (int q = 0; q < 4; q++) { edge(vt[q][0], vt[q][1], bmin[2]); edge(vt[q][0], vt[q][1], bmax[2]); }
    }
    std::fprintf(f, " sphere\n particles\n color\n %d\n", n);
    // the particle lines, formatted in parallel chunks and written in order
    const int chunk = 65536;
    const int nchunk = (n + chunk - 1) / chunk;
    std::vector<std::string> text(nchunk);
    par_for((size_t)nchunk, [&](size_t a, size_t b) {
        char line[256];
        for (size_t q = a; q < b; q++) {
            std::string& out = text[q];
            const int i0 = (int)q * chunk, i1 = std::min(n, i0 + chunk);
            for (int i = i0; i < i1; i++) {
                const double* o = rows + (size_t)i * kOutCols;
                double r, g, bl;
                switch ((int)o[47]) {
                case 0: r = 0.80; g = 0.80; bl = 0.80; break;
                case 1: r = 0.2; g = 0.47; bl = 0.87; break;
                case 2: r = 0.87; g = 0.87; bl = 0.2; break;
                case 3: r = 0.0; g = 1.0; bl = 0.67; break;
                case 4: r = 0.73; g = 0.47; bl = 0.07; break;
                case 7: r = 0.5; g = 0.5; bl = 0.5; break;
                default: continue;
                }
                const int len = std::snprintf(line, sizeof(line), "%6.4f %6.4f %6.4f %6.4f %6.4f %6.4f %6.4f\n", o[0],
                                              o[1], o[2], dr, r, g, bl);
                out.append(line, (size_t)len);
            }
        }
    });
    bool ok = true;
    for (const std::string& t : text) ok = ok && std::fwrite(t.data(), 1, t.size(), f) == t.size();
    if (std::fclose(f) != 0) ok = false;
    return ok ? 0 : SPHGPU_E_ARG;
}

}  // namespace

int sphgpu_output_begin(sphgpu_ctx* c, const char* dir)
{
    if (!c || !dir || std::strlen(dir) > 900) return SPHGPU_E_ARG;
    // the files SPH_Calculation opens before its loop (CPP_1-SPHLoops.cpp:
    // 185-230), with the AVS header it writes (:452-453)
    const std::string d(dir);
    FILE* f = std::fopen((d + "/Flowing distance.dat").c_str(), "w");
    if (!f) return SPHGPU_E_ARG;
    std::fclose(f);
    f = std::fopen((d + "/Total_Force.dat").c_str(), "w");
    if (!f) return SPHGPU_E_ARG;
    std::fclose(f);
    f = std::fopen((d + "/AVS_MGF.mgf").c_str(), "w");
    if (!f) return SPHGPU_E_ARG;
    std::fprintf(f, "# Micro AVS Geom:2.10\n# SPH simulation\n");
    std::fprintf(f, "%d\n", (int)(c->P.loop / c->P.fop));
    return std::fclose(f) == 0 ? 0 : SPHGPU_E_ARG;
}

int sphgpu_output_total(sphgpu_ctx* c, const char* dir) { return sphgpu_output_step(c, dir, SPHGPU_OUT_ODB); }

int sphgpu_output_step(sphgpu_ctx* c, const char* dir, int what)
{
    if (!c || !dir || std::strlen(dir) > 900) return SPHGPU_E_ARG;
    if (what & ~(SPHGPU_OUT_ODB | SPHGPU_OUT_FLOWDIST | SPHGPU_OUT_IMPACT | SPHGPU_OUT_MGF)) return SPHGPU_E_ARG;
    if (c->sticky) return c->sticky;
    if (c->part_done) return SPHGPU_E_STATE;          // between steps only
    cudaSetDevice(c->device);
    const int slot = c->out_next;
    if (c->out_th[slot].joinable()) c->out_th[slot].join();      // the slot's previous file
    const size_t bytes = sizeof(double) * ((size_t)c->N * kOutCols + 1);
    if (!c->out_dev[slot]) {
        if (!c->out_st) CK(cudaStreamCreateWithFlags(&c->out_st, cudaStreamNonBlocking));
        int r = dalloc(c, &c->out_dev[slot], (size_t)c->N * kOutCols + 1);
        if (r) return r;
        CK(cudaMallocHost(&c->out_host[slot], bytes));
        CK(cudaEventCreateWithFlags(&c->out_ev[slot], cudaEventDisableTiming));
    }
    // the snapshot on the step stream (the next step waits for it); the copy
    // to the host on the writer's stream, overlapping the next steps
    k_out_pack<<<(c->N + 255) / 256, 256, 0, c->st>>>(c->d[c->parity], c->out_dev[slot]);
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->out_ev[slot], c->st));
    CK(cudaStreamWaitEvent(c->out_st, c->out_ev[slot], 0));
    CK(cudaMemcpyAsync(c->out_host[slot], c->out_dev[slot], bytes, cudaMemcpyDeviceToHost, c->out_st));
    CK(cudaEventRecord(c->out_ev[slot], c->out_st));
    const int l = c->l_host - 1, n = c->N, dev = c->device, nd = c->P.ndim, fop = c->P.fop;
    const double dr = c->P.dr;
    const double bmin[3] = {c->P.xmin, c->P.ymin, c->P.zmin}, bmax[3] = {c->P.xmax, c->P.ymax, c->P.zmax};
    std::string where(dir);
    double* host = c->out_host[slot];
    cudaEvent_t ev = c->out_ev[slot];
    const long ticket = c->out_ticket++;
    c->out_th[slot] = std::thread([=]() {
        cudaSetDevice(dev);
        int rc = (cudaEventSynchronize(ev) == cudaSuccess) ? 0 : SPHGPU_E_CUDA;
        if (!rc && (what & SPHGPU_OUT_ODB)) rc = write_odb(where.c_str(), l, host, n);
        // the appended files in call order (every ticket takes its turn,
        // also after an error)
        std::unique_lock<std::mutex> lk(c->out_mu);
        c->out_cv.wait(lk, [&] { return c->out_turn == ticket; });
        if (!rc && (what & SPHGPU_OUT_FLOWDIST)) rc = append_flowdist(where.c_str(), l, host, n);
        if (!rc && (what & SPHGPU_OUT_IMPACT)) rc = write_impact(where.c_str(), l, host, n, nd, dr);
        if (!rc && (what & SPHGPU_OUT_MGF) && fop > 0)
            rc = append_mgf(where.c_str(), l, fop, host, n, nd, dr, bmin, bmax);
        if (rc && c->out_err == 0) c->out_err = rc;
        c->out_turn++;
        lk.unlock();
        c->out_cv.notify_all();
    });
    c->out_next ^= 1;
    return 0;
}

int sphgpu_output_wait(sphgpu_ctx* c)
{
    if (!c) return SPHGPU_E_ARG;
    for (int b = 0; b < 2; b++)
        if (c->out_th[b].joinable()) c->out_th[b].join();
    const int rc = c->out_err;
    c->out_err = 0;
    return rc;
}

int sphgpu_set_rain(sphgpu_ctx* c, const sphgpu_rain* rain)
{
    if (!c || !rain) return SPHGPU_E_ARG;
    if (c->P.flr != 1) return SPHGPU_E_STATE;
    if (rain->rtype != 1) return SPHGPU_E_UNSUPPORTED;
    if (rain->nrain < 0 || rain->nrain > c->N || rain->nhor < 0) return SPHGPU_E_ARG;
    sphgpu_rain r = *rain;
    if (r.nhor == 0) r.nhor = 35;            // initial_pro's default (CPP_2-initialf.cpp:201-202)
    // rainini (CPP_15-1-rain.cpp:11-23): nrain / nhor in integer arithmetic
    const double temp = r.nrain / r.nhor + 1.0;
    const int lp = (int)((c->P.loop - c->P.inip) / temp);
    cudaSetDevice(c->device);
    CK(cudaMemcpyAsync(c->d[0].s.nrain, &r.nrain, sizeof(int), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int p = 0; p < 2; p++) {
        c->d[p].p.rain_lp = lp;
        c->d[p].p.rain_vrain = r.drop_velocity;
        c->d[p].p.rain_press = r.press_factor;
    }
    c->rain = r;
    c->rain_set = true;
    invalidate_graphs(c);
    return 0;
}

int sphgpu_get_rain(sphgpu_ctx* c, sphgpu_rain* rain)
{
    if (!c || !rain) return SPHGPU_E_ARG;
    if (!c->rain_set) return SPHGPU_E_STATE;
    *rain = c->rain;
    cudaSetDevice(c->device);
    CK(cudaMemcpyAsync(&rain->nrain, c->d[0].s.nrain, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

int sphgpu_set_vibration(sphgpu_ctx* c, const sphgpu_vibration* v, const double* loads)
{
    if (!c || !v) return SPHGPU_E_ARG;
    if (c->P.flv < 1) return SPHGPU_E_STATE;
    if (v->nsteps < 1) return 7;                      // initial_pro's vibration steps error (CPP_2-initialf.cpp:262-268)
    if (!loads || !(v->ttime > 0.0) || !std::isfinite(v->ttime) || v->sttime != v->sttime || v->edtime != v->edtime)
        return SPHGPU_E_ARG;
    cudaSetDevice(c->device);
    const size_t n = 3 * (size_t)v->nsteps;
    if (c->vib_loads.size() != n) {
        double* q = nullptr;
        if (dalloc(c, &q, n)) return SPHGPU_E_CUDA;
        for (int p = 0; p < 2; p++) c->d[p].s.vib_loads = q;
    }
    c->vib_loads.assign(loads, loads + n);
    CK(cudaMemcpyAsync(c->d[0].s.vib_loads, c->vib_loads.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int p = 0; p < 2; p++) {
        DevParams& dp = c->d[p].p;
        dp.vib_ttime = v->ttime; dp.vib_nsteps = v->nsteps; dp.vib_st = v->sttime; dp.vib_ed = v->edtime;
    }
    c->vib = *v;
    c->vib_par[0] = v->ttime; c->vib_par[1] = v->nsteps; c->vib_par[2] = v->sttime; c->vib_par[3] = v->edtime;
    c->vib_set = true;
    invalidate_graphs(c);
    return 0;
}

int sphgpu_get_dt(sphgpu_ctx* c, double* dt)
{
    if (!c || !dt) return SPHGPU_E_ARG;
    if (!c->d[0].p.cfl_on) { *dt = c->P.dt; return 0; }
    cudaSetDevice(c->device);
    CK(cudaMemcpyAsync(dt, c->d[0].s.dtv, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

int sphgpu_nnps(sphgpu_ctx* c, int* ninflu, int* influ)
{
    if (!c) return SPHGPU_E_ARG;
    if (c->sticky) return c->sticky;
    cudaSetDevice(c->device);
    if (const int ro = to_caller_order(c)) return ro;
    sphk_enqueue_nnps(&c->d[c->parity], c->sort_tmp, c->sort_bytes, c->end_bit, c->st, nullptr);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->st));
    int err = 0;
    CK(cudaMemcpy(&err, c->d[0].s.err, sizeof(int), cudaMemcpyDeviceToHost));
    const int N = c->N;
    if (ninflu) CK(cudaMemcpy(ninflu, c->d[0].s.nnb, sizeof(int) * N, cudaMemcpyDeviceToHost));
    if (influ) {
        std::vector<int> cnt(N), nb((size_t)SPH_NB_CAP * N);
        CK(cudaMemcpy(cnt.data(), c->d[0].s.nnb, sizeof(int) * N, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(nb.data(), c->d[0].s.nbr, sizeof(int) * nb.size(), cudaMemcpyDeviceToHost));
        for (int i = 0; i < N; i++) {
            int* row = influ + (size_t)i * 100;
            std::memset(row, 0, sizeof(int) * 100);
            const int m = cnt[i] < SPH_NB_CAP ? cnt[i] : SPH_NB_CAP;
            for (int s = 0; s < m; s++) row[s + 1] = nb[(size_t)s * N + i];
        }
    }
    return err;
}

int sphgpu_synchronize(sphgpu_ctx* c)
{
    if (!c) return SPHGPU_E_ARG;
    cudaSetDevice(c->device);
    CK(cudaStreamSynchronize(c->st));
    return c->sticky;
}

int sphgpu_stage_count(void) { return SPHK_NSTAGES; }

const char* sphgpu_stage_name(int k)
{
    return (k >= 0 && k < SPHK_NSTAGES) ? sphk_stage_names[k] : nullptr;
}

int sphgpu_step_profiled(sphgpu_ctx* c, int nsteps, double* stage_ms)
{
    if (!c || nsteps < 0 || !stage_ms) return SPHGPU_E_ARG;
    if (c->sticky) return c->sticky;
    int r = check_particles(c);
    if (r) return r;
    if (!c->regu)
        for (long long l = c->l_host; l < (long long)c->l_host + nsteps; l++)
            if (l % c->P.step_regu == 0) { c->regu = true; invalidate_graphs(c); break; }
    cudaSetDevice(c->device);
    cudaEvent_t ev[SPHK_NSTAGES + 1];
    for (int k = 0; k <= SPHK_NSTAGES; k++) CK(cudaEventCreate(&ev[k]));
    for (int k = 0; k < SPHK_NSTAGES; k++) stage_ms[k] = 0.0;
    int err = 0;
    c->reorder_ms = 0.0;
    for (int s = 0; s < nsteps && err == 0; s++) {
        const Dev* d = &c->d[c->parity];
        if (c->reorder_every > 0 && c->since_sort >= c->reorder_every) {
            CK(cudaEventRecord(c->ev0, c->st));
            r = sort_state(c, c->parity);
            if (r) return r;
            CK(cudaEventRecord(c->ev1, c->st));
            CK(cudaEventSynchronize(c->ev1));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, c->ev0, c->ev1);
            c->reorder_ms += ms;
        }
        sphk_enqueue_nnps(d, c->sort_tmp, c->sort_bytes, c->end_bit, c->st, ev);
        enqueue_physics(c, d, ev);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(c->st));
        c->since_sort++;
        for (int k = 0; k < SPHK_NSTAGES; k++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
            stage_ms[k] += ms;
        }
        int l = 0;
        CK(cudaMemcpy(&err, c->d[0].s.err, sizeof(int), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&l, c->d[0].s.step, sizeof(int), cudaMemcpyDeviceToHost));
        c->parity = (c->parity + (l - c->l_host)) & 1;
        c->l_host = l;
    }
    for (int k = 0; k <= SPHK_NSTAGES; k++) cudaEventDestroy(ev[k]);
    return err;
}

namespace {

static_assert(TP_COUNT == SPHGPU_TUNE_PASSES, "tuned passes");

// the stages (sphk_stage_names) whose device time each tuned pass is
const char* const kTuneStages[TP_COUNT][2] = {
    {"k_nnps", nullptr}, {"k_nnps_resolve", nullptr}, {"k_pairw", nullptr}, {"k_density", nullptr},
    {"k_shepard_eos", nullptr}, {"k_strain", nullptr}, {"k_stress", "k_stress_2"}, {"k_accel_a", nullptr},
    {"k_accel_b", nullptr}, {"k_xsph_update", nullptr},
};

int stage_index(const char* name)
{
    for (int k = 0; k < SPHK_NSTAGES; k++)
        if (std::strcmp(sphk_stage_names[k], name) == 0) return k;
    return -1;
}

void set_tb(sphgpu_ctx* c, const int* tb)
{
    for (int p = 0; p < 2; p++)
        for (int q = 0; q < TP_COUNT; q++) c->d[p].p.tb[q] = tb[q];
    invalidate_graphs(c);
}

// what a tuned shape is kept for: the GPU model and the run's shape
std::string tune_key(const sphgpu_ctx* c)
{
    cudaDeviceProp prop;
    std::string name = "unknown";
    if (cudaGetDeviceProperties(&prop, c->device) == cudaSuccess) name = prop.name;
    for (char& ch : name)
        if (ch == ' ') ch = '_';
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s/ndim%d/n%d/flbndy%d/fli%d/ss%d/prec%d/inst%d", name.c_str(), c->P.ndim,
                  c->N, c->P.flbndy, c->P.fli, c->P.ss_type, c->precision, (int)c->h_inst.size());
    return buf;
}

}  // namespace

int sphgpu_set_launch(sphgpu_ctx* c, const int* tb, int n)
{
    if (!c || !tb || n != TP_COUNT) return SPHGPU_E_ARG;
    for (int q = 0; q < n; q++)
        if (tb[q] < 32 || tb[q] > 128 || tb[q] % 32 != 0) return SPHGPU_E_ARG;
    set_tb(c, tb);
    return 0;
}

int sphgpu_get_launch(const sphgpu_ctx* c, int* tb, int n)
{
    if (!c || !tb || n != TP_COUNT) return SPHGPU_E_ARG;
    for (int q = 0; q < n; q++) tb[q] = c->d[0].p.tb[q];
    return 0;
}

int sphgpu_autotune(sphgpu_ctx* c, int steps, const char* cache_path, double* table)
{
    if (!c || steps <= 0) return SPHGPU_E_ARG;
    const std::string key = tune_key(c);
    if (cache_path) {
        if (FILE* f = std::fopen(cache_path, "r")) {
            char line[512];
            int found = 0, tb[TP_COUNT];
            while (std::fgets(line, sizeof(line), f)) {
                char k[300];
                int v[TP_COUNT];
                if (std::sscanf(line, "%299s %d %d %d %d %d %d %d %d %d %d", k, &v[0], &v[1], &v[2], &v[3], &v[4],
                                &v[5], &v[6], &v[7], &v[8], &v[9]) == 1 + TP_COUNT && key == k) {
                    std::memcpy(tb, v, sizeof(tb));
                    found = 1;
                }
            }
            std::fclose(f);
            if (found && sphgpu_set_launch(c, tb, TP_COUNT) == 0) return 0;
        }
    }
    const int cand[4] = {32, 64, 96, 128};
    double t[4][TP_COUNT];
    std::vector<double> stage_ms(SPHK_NSTAGES);
    for (int a = 0; a < 4; a++) {
        int tb[TP_COUNT];
        for (int q = 0; q < TP_COUNT; q++) tb[q] = cand[a];
        set_tb(c, tb);
        int rc = sphgpu_step_profiled(c, steps, stage_ms.data());
        if (rc) return rc;
        for (int q = 0; q < TP_COUNT; q++) {
            t[a][q] = 0.0;
            for (int e = 0; e < 2; e++)
                if (kTuneStages[q][e]) {
                    const int k = stage_index(kTuneStages[q][e]);
                    if (k >= 0) t[a][q] += stage_ms[k] / steps;
                }
            if (table) table[a * TP_COUNT + q] = t[a][q];
        }
    }
    int best[TP_COUNT];
    for (int q = 0; q < TP_COUNT; q++) {
        // another shape replaces the default of 128 only when it is faster by
        // more than the step-to-step spread of the timings (3%)
        int b = 3;
        for (int a = 0; a < 3; a++)
            if (t[a][q] < 0.97 * t[3][q] && t[a][q] < t[b][q]) b = a;
        best[q] = cand[b];
    }
    set_tb(c, best);
    if (cache_path) {
        if (FILE* f = std::fopen(cache_path, "a")) {
            std::fprintf(f, "%s", key.c_str());
            for (int q = 0; q < TP_COUNT; q++) std::fprintf(f, " %d", best[q]);
            std::fprintf(f, "\n");
            std::fclose(f);
        }
    }
    return 0;
}

int sphgpu_autotune_reorder(sphgpu_ctx* c, int steps, int every, int* chosen, double* ms)
{
    if (!c || steps <= 0 || every <= 0 || !chosen) return SPHGPU_E_ARG;
    if (c->part_done) return SPHGPU_E_STATE;
    std::vector<double> stage_ms(SPHK_NSTAGES);
    auto sum = [&]() {
        double t = 0.0;
        for (double v : stage_ms) t += v;
        return t / steps;
    };
    // the caller's order, no re-sorts
    int rc = to_caller_order(c);
    if (rc) return rc;
    c->reorder_every = 0;
    rc = sphgpu_step_profiled(c, steps, stage_ms.data());
    if (rc) return rc;
    const double plain = sum();
    // re-sorted before the first of the same number of steps
    sphgpu_set_reorder(c, every);
    rc = sphgpu_step_profiled(c, steps, stage_ms.data());
    if (rc) return rc;
    const double sorted = sum();
    // the re-sort's own time, charged at one per `every` steps: a re-sort of
    // the re-sorted state, as every re-sort after the first is (the first,
    // from the caller's order, moves every record and is paid once)
    cudaSetDevice(c->device);
    CK(cudaEventRecord(c->ev0, c->st));
    rc = sort_state(c, c->parity);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaEventSynchronize(c->ev1));
    float resort_ms = 0.f;
    cudaEventElapsedTime(&resort_ms, c->ev0, c->ev1);
    const double cost = resort_ms / every;
    // the re-sorted order is kept only when it is faster by more than the
    // step-to-step spread of the timings (3%)
    *chosen = (sorted + cost < 0.97 * plain) ? every : 0;
    if (ms) { ms[0] = plain; ms[1] = sorted; ms[2] = cost; }
    if (*chosen == 0) {
        rc = to_caller_order(c);
        if (rc) return rc;
    }
    c->reorder_every = *chosen;
    return 0;
}

double sphgpu_last_step_ms(const sphgpu_ctx* c) { return c ? c->last_ms : 0.0; }
long sphgpu_last_step_launches(const sphgpu_ctx* c) { return c ? c->last_launches : 0; }
void* sphgpu_stream(sphgpu_ctx* c) { return c ? (void*)c->st : nullptr; }


// ---------------------------------------------------------------------------
// Karhunen-Loeve random fields (CPP_17-1_K-L_expansion_non.cpp)

namespace {

const double kKlPi = 3.141592653;     // Header_Parameters.h:10
const double kKlPrec = 1.0e-6;        // CPP_17-1:21

// solve_wi (CPP_17-1:275-345): the positive roots w of 2/l - w tan(w a)
// (odd terms) and 2/l tan(w a) + w (even terms) per axis, by bisection
// between the reference's bounds, in FP64 with the C library's tan.
void kl_solve_wi(std::vector<double>& wi, const double a_x[3], const double rl[3], int ndim, int K)
{
    wi.assign((size_t)K * 3, 0.0);
    std::vector<double> up(K), lo(K);
    for (int d = 0; d < ndim; d++) {
        const double a = a_x[d], dira = rl[d];
        for (int i = 0; i < K; i++) {
            if ((i + 1) % 2 == 1) { up[i] = (i + 0.5) * kKlPi / a; lo[i] = i * kKlPi / a; }
            else { up[i] = (i + 1.0) * kKlPi / a; lo[i] = (i + 0.5) * kKlPi / a; }
        }
        for (int i = 0; i < K; i++) {
            double x1 = lo[i] + kKlPrec, x2 = up[i] - kKlPrec, xm, f1, fm;
            const bool odd = (i + 1) % 2 == 1;
            xm = odd ? (x1 + x2) * 0.5 : (x1 + x2) / 2.0;
            do {
                if (odd) {
                    f1 = 2.0 / dira - x1 * std::tan(x1 * a);
                    fm = 2.0 / dira - xm * std::tan(xm * a);
                } else {
                    f1 = 2.0 / dira * std::tan(x1 * a) + x1;
                    fm = 2.0 / dira * std::tan(xm * a) + xm;
                }
                if ((f1 * fm) < 0.0) x2 = xm;
                else x1 = xm;
                xm = (x1 + x2) * 0.5;
            } while (std::fabs(fm) > kKlPrec);
            wi[(size_t)i * 3 + d] = xm;
        }
    }
}

struct HostKLTerm { double w, alpha; int use_cos; int pad; };

// The expansion of one field: per term the selected 1-D root, normalisation
// and parity on each axis, and sqrt(lambda); terms in the reference's order.
struct KLPlan {
    std::vector<HostKLTerm> terms;   // K x ndim
    std::vector<double> sqrt_eig;    // K
    std::vector<int> ids;            // K x ndim: the 1-D eigenfunction index of each term on each axis
};

int kl_plan(sphgpu_ctx* c, const double a[3], const sphgpu_kl_field& f, int K, KLPlan& plan)
{
    const int nd = c->P.ndim;
    std::vector<double> wi;
    kl_solve_wi(wi, a, f.rl_value, nd, K);
    // 1-D eigenvalues (equation_ramdai, CPP_17-1:36-41)
    std::vector<double> r((size_t)K * 3, 0.0);
    for (int d = 0; d < nd; d++)
        for (int i = 0; i < K; i++) {
            const double w = wi[(size_t)i * 3 + d], dirac = f.rl_value[d];
            r[(size_t)i * 3 + d] = 4.0 * dirac / (4.0 + w * w * dirac * dirac);
        }
    const size_t total = (nd == 2) ? (size_t)K * K : (size_t)K * K * K;
    if (total > 0xffffffffull) return SPHGPU_E_ARG;
    const size_t sort_bytes = sphk_kl_sort_bytes(total);
    void* buf = nullptr;
    const size_t off_r = 0, off_ki = 256 * ((sizeof(double) * 3 * K + 255) / 256);
    const size_t off_ko = off_ki + 256 * ((8 * total + 255) / 256);
    const size_t off_vi = off_ko + 256 * ((8 * total + 255) / 256);
    const size_t off_vo = off_vi + 256 * ((4 * total + 255) / 256);
    const size_t off_tmp = off_vo + 256 * ((4 * total + 255) / 256);
    const size_t bytes = off_tmp + sort_bytes;
    CK(cudaMalloc(&buf, bytes));
    char* b = (char*)buf;
    int rc = 0;
    do {
        if (cuda_fail(c, cudaMemcpyAsync(b + off_r, r.data(), sizeof(double) * 3 * K, cudaMemcpyHostToDevice, c->st),
                      "cudaMemcpyAsync")) { rc = SPHGPU_E_CUDA; break; }
        if (sphk_kl_order((const double*)(b + off_r), K, nd, (double*)(b + off_ki), (double*)(b + off_ko),
                          (uint32_t*)(b + off_vi), (uint32_t*)(b + off_vo), b + off_tmp, sort_bytes, c->st)) {
            rc = cuda_fail(c, cudaGetLastError(), "K-L eigenvalue ordering");
            if (!rc) rc = SPHGPU_E_CUDA;
            break;
        }
        std::vector<double> eig(K);
        std::vector<uint32_t> idx(K);
        if (cuda_fail(c, cudaMemcpyAsync(eig.data(), b + off_ko, 8 * (size_t)K, cudaMemcpyDeviceToHost, c->st),
                      "cudaMemcpyAsync") ||
            cuda_fail(c, cudaMemcpyAsync(idx.data(), b + off_vo, 4 * (size_t)K, cudaMemcpyDeviceToHost, c->st),
                      "cudaMemcpyAsync") ||
            cuda_fail(c, cudaStreamSynchronize(c->st), "cudaStreamSynchronize")) { rc = SPHGPU_E_CUDA; break; }
        // the terms: per axis the root of the selected 1-D index, its
        // normalisation (solve_faii, CPP_17-1:44-59) and cos / sin parity
        std::vector<HostKLTerm>& terms = plan.terms;
        std::vector<double>& se = plan.sqrt_eig;
        terms.assign((size_t)K * nd, HostKLTerm{});
        se.assign(K, 0.0);
        plan.ids.assign((size_t)K * nd, 0);
        for (int j = 0; j < K; j++) {
            int id[3];
            if (nd == 2) { id[0] = (int)(idx[j] / K); id[1] = (int)(idx[j] % K); }
            else {
                id[0] = (int)(idx[j] / ((uint32_t)K * K));
                id[1] = (int)((idx[j] / K) % K);
                id[2] = (int)(idx[j] % K);
            }
            for (int d = 0; d < nd; d++) {
                plan.ids[(size_t)j * nd + d] = id[d];
                const double w = wi[(size_t)id[d] * 3 + d], ad = a[d];
                HostKLTerm& t = terms[(size_t)j * nd + d];
                t.w = w;
                t.use_cos = ((id[d] + 1) % 2 == 1) ? 1 : 0;
                t.alpha = t.use_cos ? 1.0 / std::sqrt(std::sin(2.0 * w * ad) / 2.0 / w + ad)
                                    : 1.0 / std::sqrt(-std::sin(2.0 * w * ad) / 2.0 / w + ad);
                t.pad = 0;
            }
            se[j] = std::sqrt(eig[j]);
        }
    } while (0);
    cudaFree(buf);
    return rc;
}

// One field of SpatialVariables_Generate_2D / _3D for the context's
// particles; d_out receives the values (NaN where the field writes none).
int kl_one_field(sphgpu_ctx* c, const double a[3], const double x_trans[3], double soil_max, double water_max,
                 const sphgpu_kl_field& f, const double* xi, int K, double* d_out, int first = 0, int count = -1)
{
    if (count < 0) count = c->N - first;
    const int nd = c->P.ndim;
    if (f.type != 1 && f.type != 2) return 14;
    KLPlan plan;
    int rc = kl_plan(c, a, f, K, plan);
    if (rc) return rc;
    void* buf = nullptr;
    const size_t off_se = 256 * ((sizeof(HostKLTerm) * plan.terms.size() + 255) / 256);
    const size_t off_xi = off_se + 256 * ((8 * (size_t)K + 255) / 256);
    CK(cudaMalloc(&buf, off_xi + 8 * (size_t)K));
    char* b = (char*)buf;
    do {
        if (cuda_fail(c, cudaMemcpyAsync(b, plan.terms.data(), sizeof(HostKLTerm) * plan.terms.size(),
                                         cudaMemcpyHostToDevice, c->st), "cudaMemcpyAsync") ||
            cuda_fail(c, cudaMemcpyAsync(b + off_se, plan.sqrt_eig.data(), 8 * (size_t)K, cudaMemcpyHostToDevice,
                                         c->st), "cudaMemcpyAsync") ||
            cuda_fail(c, cudaMemcpyAsync(b + off_xi, xi, 8 * (size_t)K, cudaMemcpyHostToDevice, c->st),
                      "cudaMemcpyAsync")) { rc = SPHGPU_E_CUDA; break; }
        const DevState& s = c->d[c->parity].s;
        if (sphk_kl_field(count, nd, K, f.no, f.type, x_trans, f.mean_value, f.sd_value, f.coe_depth, soil_max,
                          water_max, s.xh + 4 * (size_t)first, s.type + first, b, (const double*)(b + off_se),
                          (const double*)(b + off_xi), d_out + first, c->st)) { rc = SPHGPU_E_CUDA; break; }
        if (cuda_fail(c, cudaStreamSynchronize(c->st), "cudaStreamSynchronize")) { rc = SPHGPU_E_CUDA; break; }
    } while (0);
    cudaFree(buf);
    return rc;
}

// the field domain: the non-boundary box widened by 20% per side
// (CPP_17-1:70-90, 166-186); soil_max / water_max along y (2-D) or z (3-D)
int kl_dom(int nd, const sphgpu_kl_domain* dom, double a[3], double xt[3], double* soil_max, double* water_max)
{
    const double lo[3] = {dom->xmin_nb, dom->ymin_nb, dom->zmin_nb};
    const double hi[3] = {dom->xmax_nb, dom->ymax_nb, dom->zmax_nb};
    for (int d = 0; d < 3; d++) a[d] = xt[d] = 0.0;
    for (int d = 0; d < nd; d++) {
        const double xmin = lo[d] - 0.2 * (hi[d] - lo[d]), xmax = hi[d] + 0.2 * (hi[d] - lo[d]);
        xt[d] = (xmax + xmin) / 2.0;
        a[d] = (xmax - xmin) / 2.0;
    }
    *soil_max = dom->soil_max[nd == 2 ? 1 : 2];
    *water_max = dom->water_max[nd == 2 ? 1 : 2];
    return (a[0] == 0.0 || a[1] == 0.0) ? 13 : 0;
}

// the field's values written into the host copies of the material records
void kl_store(sphgpu_ctx* c, int no, const double* v, int first, int count)
{
    for (int i = first; i < first + count; i++) {
        if (v[i] != v[i]) continue;
        switch (no) {
        case 0: c->h_soil[i].fai = v[i]; break;
        case 1: c->h_soil[i].c = v[i]; break;
        case 2: c->h_soil[i].cop = v[i]; break;
        case 3: c->h_soil[i].ds = v[i]; break;
        case 4: c->h_fluid[i].fai = v[i]; break;
        case 5: c->h_fluid[i].c = v[i]; break;
        }
    }
}

int kl_run(sphgpu_ctx* c, const sphgpu_kl_domain* dom, const sphgpu_kl_field* fields, int nfields,
           const double* const* xis, int K, double* out)
{
    if (!c || !dom || !fields || nfields <= 0 || K <= 0) return SPHGPU_E_ARG;
    if (c->h_type.empty() || (c->h_soil.empty() && c->h_fluid.empty())) return SPHGPU_E_STATE;
    for (int q = 0; q < nfields; q++) {
        if (fields[q].no < 0 || fields[q].no > 5) return SPHGPU_E_ARG;
        if (fields[q].no <= 3 && c->h_soil.empty()) return SPHGPU_E_STATE;
        if (fields[q].no >= 4 && c->h_fluid.empty()) return SPHGPU_E_STATE;
    }
    cudaSetDevice(c->device);
    if (const int ro = to_caller_order(c)) return ro;
    const int nd = c->P.ndim, N = c->N;
    double a[3], xt[3], soil_max, water_max;
    if (kl_dom(nd, dom, a, xt, &soil_max, &water_max)) return 13;
    double* d_out = nullptr;
    CK(cudaMalloc(&d_out, sizeof(double) * N));
    std::vector<double> v(N);
    int rc = 0;
    for (int q = 0; q < nfields && !rc; q++) {
        rc = kl_one_field(c, a, xt, soil_max, water_max, fields[q], xis[q], K, d_out);
        if (rc) break;
        if (cuda_fail(c, cudaMemcpy(v.data(), d_out, sizeof(double) * N, cudaMemcpyDeviceToHost), "cudaMemcpy")) {
            rc = SPHGPU_E_CUDA;
            break;
        }
        if (out) std::memcpy(out + (size_t)q * N, v.data(), sizeof(double) * N);
        kl_store(c, fields[q].no, v.data(), 0, N);
    }
    cudaFree(d_out);
    if (rc) return rc;
    return sphgpu_set_materials(c, c->h_fluid.empty() ? nullptr : c->h_fluid.data(),
                                c->h_soil.empty() ? nullptr : c->h_soil.data(), N);
}

}  // namespace

int sphgpu_kl_generate_batched(sphgpu_ctx* c, const sphgpu_kl_domain* doms, const sphgpu_kl_field* f,
                               const double* xi, int K, double* out)
{
    if (!c || !doms || !f || !xi || K <= 0 || c->h_inst.empty()) return SPHGPU_E_ARG;
    if (f->no < 0 || f->no > 5) return SPHGPU_E_ARG;
    if (c->h_type.empty() || (f->no <= 3 && c->h_soil.empty()) || (f->no >= 4 && c->h_fluid.empty()))
        return SPHGPU_E_STATE;
    cudaSetDevice(c->device);
    if (const int ro = to_caller_order(c)) return ro;
    const int nd = c->P.ndim, N = c->N;
    double* d_out = nullptr;
    CK(cudaMalloc(&d_out, sizeof(double) * N));
    int rc = 0;
    for (size_t q = 0; q < c->h_inst.size() && !rc; q++) {
        double a[3], xt[3], soil_max, water_max;
        if (kl_dom(nd, &doms[q], a, xt, &soil_max, &water_max)) { rc = 13; break; }
        rc = kl_one_field(c, a, xt, soil_max, water_max, *f, xi + q * (size_t)K, K, d_out, c->h_inst[q].first,
                          c->h_inst[q].count);
    }
    std::vector<double> v;
    if (!rc) {
        v.resize(N);
        if (cuda_fail(c, cudaMemcpy(v.data(), d_out, sizeof(double) * N, cudaMemcpyDeviceToHost), "cudaMemcpy"))
            rc = SPHGPU_E_CUDA;
    }
    cudaFree(d_out);
    if (rc) return rc;
    if (out) std::memcpy(out, v.data(), sizeof(double) * N);
    kl_store(c, f->no, v.data(), 0, N);
    return sphgpu_set_materials(c, c->h_fluid.empty() ? nullptr : c->h_fluid.data(),
                                c->h_soil.empty() ? nullptr : c->h_soil.data(), N);
}

int sphgpu_kl_generate(sphgpu_ctx* c, const sphgpu_kl_domain* dom, const sphgpu_kl_field* fields, int nfields,
                       const double* xi, int K, double* out)
{
    if (!xi || nfields <= 0) return SPHGPU_E_ARG;
    std::vector<const double*> xis(nfields);
    for (int q = 0; q < nfields; q++) xis[q] = xi + (size_t)q * K;
    return kl_run(c, dom, fields, nfields, xis.data(), K, out);
}

int sphgpu_kl_generate_corr(sphgpu_ctx* c, const sphgpu_kl_domain* dom, const sphgpu_kl_field pair[2],
                            double coe, const double* u2, int K, double* out)
{
    if (!pair || !u2 || K <= 0) return SPHGPU_E_ARG;
    // the correlation coefficient of the underlying normals
    // (CPP_17-2:115-131): for lognormal fields from the fields' COVs
    double coefficient = coe;
    if (pair[0].type == 2) {
        const double m0 = pair[0].mean_value, s0 = pair[0].sd_value, m1 = pair[1].mean_value, s1 = pair[1].sd_value;
        coefficient = std::log(1.0 + coe * (s0 / m0) * (s1 / m1));
        coefficient = coefficient / std::sqrt(std::log(1.0 + s0 * s0 / m0 / m0) * std::log(1.0 + s1 * s1 / m1 / m1));
    }
    // zeta = u2 [1, coefficient; 0, sqrt(1 - coefficient^2)] (matrix_multi, CPP_17-2:21-35, 133-140)
    const double cm[4] = {1.0, coefficient, 0.0, std::sqrt(1.0 - coefficient * coefficient)};
    std::vector<double> z0(K), z1(K);
    for (int i = 0; i < K; i++) {
        double t0 = 0.0, t1 = 0.0;
        t0 = t0 + u2[(size_t)i * 2 + 0] * cm[0];
        t0 = t0 + u2[(size_t)i * 2 + 1] * cm[2];
        t1 = t1 + u2[(size_t)i * 2 + 0] * cm[1];
        t1 = t1 + u2[(size_t)i * 2 + 1] * cm[3];
        z0[i] = t0;
        z1[i] = t1;
    }
    const double* xis[2] = {z0.data(), z1.data()};
    return kl_run(c, dom, pair, 2, xis, K, out);
}

// ---------------------------------------------------------------------------
// correlation-matrix random fields (flspv 3, 4 and 5)

namespace {

// the cells: the non-boundary box widened by 10% per side, cells of
// cell_ndx spacings, their base offset as CPP_17-3:100-132 (2-D) and
// :482-517 (3-D) compute it.  41: no cells, or 15,000 or more.
struct RFGeom { int nc[3]; double base[3]; double cdx; int total; };

int rf_geom(int nd, double dr, const sphgpu_kl_domain* dom, double cell_ndx, RFGeom& g)
{
    const double lo[3] = {dom->xmin_nb, dom->ymin_nb, dom->zmin_nb};
    const double hi[3] = {dom->xmax_nb, dom->ymax_nb, dom->zmax_nb};
    double xmin[3] = {0, 0, 0}, xmax[3] = {0, 0, 0};
    g.cdx = cell_ndx * dr;
    g.total = 0;
    for (int d = 0; d < 3; d++) { g.nc[d] = 1; g.base[d] = 0.0; }
    for (int d = 0; d < nd; d++) {
        xmin[d] = lo[d] - 0.1 * (hi[d] - lo[d]);
        xmax[d] = hi[d] + 0.1 * (hi[d] - lo[d]);
        const double q = (xmax[d] - xmin[d]) / g.cdx;
        if (!(q >= 0.0 && q < 15000.0)) return 41;      // also a zero, negative or NaN cell edge
        g.nc[d] = (int)q + 1;
    }
    const long long total = (long long)g.nc[0] * g.nc[1] * g.nc[2];
    if (!(total > 0 && total < 15000)) return 41;
    g.total = (int)total;
    for (int d = 0; d < nd; d++) g.base[d] = -(g.nc[d] * g.cdx - (xmax[d] - xmin[d])) / 2.0 + 0.01 * dr + xmin[d];
    return 0;
}

void rf_pack(const sphgpu_ctx* c, const RFGeom& g, const sphgpu_kl_field& f, const sphgpu_rf_flags& fl,
             int depth_axis, int log_exp, int ip[10], double dp[15])
{
    const int nd = c->P.ndim;
    ip[0] = nd; ip[1] = c->N; ip[2] = f.no; ip[3] = f.type; ip[4] = fl.flag_auto;
    for (int d = 0; d < 3; d++) ip[5 + d] = g.nc[d];
    ip[8] = depth_axis; ip[9] = log_exp;
    const double pi = 3.141592653;                       // Header_Parameters.h:10
    for (int d = 0; d < 3; d++) { dp[d] = g.base[d]; dp[3 + d] = f.rl_value[d]; }
    dp[6] = g.cdx; dp[7] = c->P.dr;
    dp[8] = f.mean_value; dp[9] = f.sd_value; dp[10] = f.coe_depth;
    dp[11] = fl.beta * pi / 180.0; dp[12] = fl.beta_1 * pi / 180.0;
    dp[13] = 0.0; dp[14] = 0.0;
}

// The device side of one call: cells once, then for every field its factor
// (re-used while the correlation lengths stay the same), E = L zeta and the
// particles' values.  zetas[q] holds the normals of field q (total values);
// out receives nfields x N values.
int rf_run(sphgpu_ctx* c, const sphgpu_kl_domain* dom, const sphgpu_kl_field* fields, int nfields,
           const sphgpu_rf_flags* fl, const double* const* zetas, const int* depth_axis, int log_exp, double* out)
{
    cudaSetDevice(c->device);
    if (const int ro = to_caller_order(c)) return ro;
    const int nd = c->P.ndim, N = c->N;
    RFGeom g;
    int rc = rf_geom(nd, c->P.dr, dom, fl->cell_ndx, g);
    if (rc) return rc;
    const double soil_max = dom->soil_max[nd == 2 ? 1 : 2], water_max = dom->water_max[nd == 2 ? 1 : 2];
    const size_t T = (size_t)g.total;
    const size_t off_count = 256 * ((4 * (size_t)N + 255) / 256);
    const size_t off_err = off_count + 256 * ((4 * T + 255) / 256);
    const size_t off_zeta = off_err + 256;
    const size_t off_E = off_zeta + 256 * ((8 * T + 255) / 256);
    const size_t off_out = off_E + 256 * ((8 * T + 255) / 256);
    const size_t off_C = off_out + 256 * ((8 * (size_t)N + 255) / 256);
    void* buf = nullptr;
    CK(cudaMalloc(&buf, off_C + 8 * T * T));
    char* b = (char*)buf;
    int* d_cell = (int*)b;
    int* d_count = (int*)(b + off_count);
    int* d_err = (int*)(b + off_err);
    double* d_zeta = (double*)(b + off_zeta);
    double* d_E = (double*)(b + off_E);
    double* d_out = (double*)(b + off_out);
    double* d_C = (double*)(b + off_C);
    const DevState& s = c->d[c->parity].s;
    int ip[10];
    double dp[15];
    do {
        rf_pack(c, g, fields[0], *fl, nd - 1, log_exp, ip, dp);
        int herr[2] = {0, 0};
        if (cuda_fail(c, cudaMemsetAsync(d_count, 0, off_zeta - off_count, c->st), "cudaMemsetAsync") ||
            sphk_rf_cells(ip, dp, s.xh, s.type, d_cell, d_count, d_err, c->st) ||
            cuda_fail(c, cudaMemcpyAsync(herr, d_err, sizeof(herr), cudaMemcpyDeviceToHost, c->st), "cudaMemcpyAsync") ||
            cuda_fail(c, cudaStreamSynchronize(c->st), "cudaStreamSynchronize")) { rc = SPHGPU_E_CUDA; break; }
        // a particle outside the cells, where the reference would index past
        // its cell array; else a cell over its 39 places (error 42)
        if (herr[0]) { rc = SPHGPU_E_ARG; break; }
        if (herr[1]) { rc = 42; break; }
        const sphgpu_kl_field* factored = nullptr;
        for (int q = 0; q < nfields && !rc; q++) {
            const sphgpu_kl_field& f = fields[q];
            rf_pack(c, g, f, *fl, depth_axis[q], log_exp, ip, dp);
            dp[13] = soil_max; dp[14] = water_max;
            if (!factored || std::memcmp(factored->rl_value, f.rl_value, sizeof(f.rl_value)) != 0) {
                if (sphk_rf_factor(ip, dp, d_C, c->st)) { rc = SPHGPU_E_CUDA; break; }
                factored = &f;
            }
            if (cuda_fail(c, cudaMemcpyAsync(d_zeta, zetas[q], 8 * T, cudaMemcpyHostToDevice, c->st),
                          "cudaMemcpyAsync") ||
                sphk_rf_assign(ip, dp, d_C, d_zeta, d_E, d_cell, s.type, d_out, c->st) ||
                cuda_fail(c, cudaMemcpyAsync(out + (size_t)q * N, d_out, 8 * (size_t)N, cudaMemcpyDeviceToHost,
                                             c->st), "cudaMemcpyAsync") ||
                cuda_fail(c, cudaStreamSynchronize(c->st), "cudaStreamSynchronize")) { rc = SPHGPU_E_CUDA; break; }
        }
    } while (0);
    cudaFree(buf);
    return rc;
}

int rf_check(const sphgpu_ctx* c, const sphgpu_kl_field* fields, int nfields)
{
    if (c->h_type.empty() || (c->h_soil.empty() && c->h_fluid.empty())) return SPHGPU_E_STATE;
    if (!c->h_inst.empty()) return SPHGPU_E_UNSUPPORTED;     // one system per context
    for (int q = 0; q < nfields; q++) {
        if (fields[q].no < 0 || fields[q].no > 5) return SPHGPU_E_ARG;
        if (fields[q].no <= 3 && c->h_soil.empty()) return SPHGPU_E_STATE;
        if (fields[q].no >= 4 && c->h_fluid.empty()) return SPHGPU_E_STATE;
    }
    return 0;
}

int rf_finish(sphgpu_ctx* c, const sphgpu_kl_field* fields, int nfields, const double* v)
{
    for (int q = 0; q < nfields; q++) kl_store(c, fields[q].no, v + (size_t)q * c->N, 0, c->N);
    return sphgpu_set_materials(c, c->h_fluid.empty() ? nullptr : c->h_fluid.data(),
                                c->h_soil.empty() ? nullptr : c->h_soil.data(), c->N);
}

// the correlation coefficient of the underlying normals and the 2 x 2 factor
// (CPP_17-5:206-225): for lognormal fields from the fields' COVs
void rf_pair_factor(const sphgpu_kl_field pair[2], double coe, double cm[4])
{
    double coefficient = coe;
    if (pair[0].type == 2) {
        const double m0 = pair[0].mean_value, s0 = pair[0].sd_value, m1 = pair[1].mean_value, s1 = pair[1].sd_value;
        coefficient = std::log(1.0 + coe * (s0 / m0) * (s1 / m1));
        coefficient = coefficient / std::sqrt(std::log(1.0 + s0 * s0 / m0 / m0) * std::log(1.0 + s1 * s1 / m1 / m1));
    }
    cm[0] = 1.0; cm[1] = coefficient; cm[2] = 0.0; cm[3] = std::sqrt(1.0 - coefficient * coefficient);
}

int rf_pair_check(const sphgpu_kl_field pair[2])
{
    // friction then cohesion of one phase
    if (!((pair[0].no == 0 && pair[1].no == 1) || (pair[0].no == 4 && pair[1].no == 5))) return SPHGPU_E_ARG;
    return 0;
}

}  // namespace

int sphgpu_rf_cells(sphgpu_ctx* c, const sphgpu_kl_domain* dom, const sphgpu_rf_flags* fl, int* ncell)
{
    if (!c || !dom || !fl || !ncell) return SPHGPU_E_ARG;
    RFGeom g;
    const int rc = rf_geom(c->P.ndim, c->P.dr, dom, fl->cell_ndx, g);
    *ncell = g.total;
    return rc;
}

int sphgpu_rf_generate(sphgpu_ctx* c, const sphgpu_kl_domain* dom, const sphgpu_kl_field* fields, int nfields,
                       const sphgpu_rf_flags* fl, const double* zeta, int ncell, double* out)
{
    if (!c || !dom || !fields || !fl || !zeta || nfields <= 0) return SPHGPU_E_ARG;
    int rc = rf_check(c, fields, nfields);
    if (rc) return rc;
    RFGeom g;
    if ((rc = rf_geom(c->P.ndim, c->P.dr, dom, fl->cell_ndx, g))) return rc;
    if (ncell != g.total) return SPHGPU_E_ARG;
    const int N = c->N;
    std::vector<double> v((size_t)nfields * N);
    std::vector<const double*> zetas(nfields);
    std::vector<int> axis(nfields, c->P.ndim - 1);
    for (int q = 0; q < nfields; q++) zetas[q] = zeta + (size_t)q * ncell;
    rc = rf_run(c, dom, fields, nfields, fl, zetas.data(), axis.data(), 0, v.data());
    if (rc) return rc;
    if (out) std::memcpy(out, v.data(), sizeof(double) * v.size());
    return rf_finish(c, fields, nfields, v.data());
}

int sphgpu_rf_generate_corr(sphgpu_ctx* c, const sphgpu_kl_domain* dom, const sphgpu_kl_field pair[2],
                            const sphgpu_rf_flags* fl, const double* u2, int ncell, double* out)
{
    if (!c || !dom || !pair || !fl || !u2) return SPHGPU_E_ARG;
    int rc = rf_pair_check(pair);
    if (rc || (rc = rf_check(c, pair, 2))) return rc;
    RFGeom g;
    if ((rc = rf_geom(c->P.ndim, c->P.dr, dom, fl->cell_ndx, g))) return rc;
    if (ncell != g.total) return SPHGPU_E_ARG;
    // zeta = u2 [1, coefficient; 0, sqrt(1 - coefficient^2)] (matrix_multi,
    // CPP_17-5:21-33, 225-227)
    double cm[4];
    rf_pair_factor(pair, fl->coe_frict_cohesion, cm);
    std::vector<double> z0(ncell), z1(ncell);
    for (int i = 0; i < ncell; i++) {
        double t0 = 0.0, t1 = 0.0;
        t0 = t0 + u2[(size_t)i * 2 + 0] * cm[0];
        t0 = t0 + u2[(size_t)i * 2 + 1] * cm[2];
        t1 = t1 + u2[(size_t)i * 2 + 0] * cm[1];
        t1 = t1 + u2[(size_t)i * 2 + 1] * cm[3];
        z0[i] = t0;
        z1[i] = t1;
    }
    // both members take the friction field's lengths and distribution type
    // (psv_temp, CPP_17-5:177-186); the fluid members of the 3-D field read
    // their depth on y (17-5:650-735)
    sphgpu_kl_field two[2] = {pair[0], pair[1]};
    for (int d = 0; d < 3; d++) two[1].rl_value[d] = pair[0].rl_value[d];
    two[1].type = pair[0].type;
    const int nd = c->P.ndim;
    const int axis[2] = {(nd == 3 && pair[0].no == 4) ? 1 : nd - 1, (nd == 3 && pair[1].no == 5) ? 1 : nd - 1};
    const double* zetas[2] = {z0.data(), z1.data()};
    const int N = c->N;
    std::vector<double> v(2 * (size_t)N);
    rc = rf_run(c, dom, two, 2, fl, zetas, axis, 1, v.data());
    if (rc) return rc;
    if (out) std::memcpy(out, v.data(), sizeof(double) * v.size());
    return rf_finish(c, pair, 2, v.data());
}

int sphgpu_rv_generate_corr(sphgpu_ctx* c, const sphgpu_kl_field pair[2], double coe_frict_cohesion,
                            const double u2[2], double out[2])
{
    if (!c || !pair || !u2) return SPHGPU_E_ARG;
    int rc = rf_pair_check(pair);
    if (rc || (rc = rf_check(c, pair, 2))) return rc;
    // the correlated pair [zeta_c, zeta_fai] (random_variable_generate,
    // CPP_17-5:738-863): friction takes the second, cohesion the first
    double cm[4];
    rf_pair_factor(pair, coe_frict_cohesion, cm);
    double t0 = 0.0, t1 = 0.0;
    t0 = t0 + u2[0] * cm[0];
    t0 = t0 + u2[1] * cm[2];
    t1 = t1 + u2[0] * cm[1];
    t1 = t1 + u2[1] * cm[3];
    const double z[2] = {t1, t0};
    double val[2];
    const int dist = pair[0].type;
    for (int k = 0; k < 2; k++) {
        double mean = pair[k].mean_value, sd = pair[k].sd_value;
        if (dist == 1) val[k] = mean + sd * z[k];
        else if (dist == 2) {
            sd = std::sqrt(std::log(1.0 + (sd / mean) * (sd / mean)));
            mean = std::log(mean) - 0.5 * sd * sd;
            val[k] = std::exp(mean + sd * z[k]);
        } else val[k] = std::nan("");
    }
    if (out) { out[0] = val[0]; out[1] = val[1]; }
    const int want = pair[0].no == 0 ? 2 : 1;
    const int N = c->N;
    std::vector<double> v(2 * (size_t)N, std::nan(""));
    for (int i = 0; i < N; i++)
        if (c->h_type[i] == want) { v[i] = val[0]; v[(size_t)N + i] = val[1]; }
    return rf_finish(c, pair, 2, v.data());
}


int sphgpu_kl_wait_check(sphgpu_ctx* c, long long budget_cycles)
{
    if (!c || budget_cycles <= 0) return SPHGPU_E_ARG;
    cudaSetDevice(c->device);
    int* d_err = nullptr;
    CK(cudaMalloc(&d_err, sizeof(int)));
    int rc = 0, err = 0;
    if (cuda_fail(c, cudaMemsetAsync(d_err, 0, sizeof(int), c->st), "cudaMemsetAsync") ||
        sphk_kl_wait_probe(budget_cycles, d_err, c->st) ||
        cuda_fail(c, cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st), "cudaMemcpyAsync") ||
        cuda_fail(c, cudaStreamSynchronize(c->st), "cudaStreamSynchronize"))
        rc = SPHGPU_E_CUDA;
    cudaFree(d_err);
    return rc ? rc : err;
}

int sphgpu_kl_synthesize(sphgpu_ctx* c, const sphgpu_kl_domain* dom, const sphgpu_kl_field* f, const double* xi,
                         int R, int K, float* d_out, double* kernel_ms)
{
    if (!c || !dom || !f || !xi || !d_out || R <= 0 || R % 16 != 0 || K < 8 || K % 8 != 0) return SPHGPU_E_ARG;
    if (f->no < 0 || f->no > 5) return SPHGPU_E_ARG;
    if (f->type != 1 && f->type != 2) return 14;
    if (c->h_type.empty()) return SPHGPU_E_STATE;
    cudaSetDevice(c->device);
    if (const int ro = to_caller_order(c)) return ro;
    const int nd = c->P.ndim, N = c->N;
    double a[3], xt[3], soil_max, water_max;
    if (kl_dom(nd, dom, a, xt, &soil_max, &water_max)) return 13;
    KLPlan plan;
    int rc = kl_plan(c, a, *f, K, plan);
    if (rc) return rc;
    // the tensor-core kernel's term record: w (FP64), alpha (FP32), parity
    struct TCTerm { double w; float alpha; int use_cos; };
    if (sphk_kl_tc_term_bytes() != sizeof(TCTerm)) return SPHGPU_E_ARG;
    std::vector<TCTerm> tc(plan.terms.size());
    for (size_t q = 0; q < tc.size(); q++)
        tc[q] = TCTerm{plan.terms[q].w, (float)plan.terms[q].alpha, plan.terms[q].use_cos};
    // the separable form: per axis the distinct 1-D eigenfunctions the terms
    // use (in order of first use) and each term's index among them
    std::vector<TCTerm> modes;
    std::vector<unsigned short> tidx((size_t)K * nd);
    int nmode[3] = {0, 0, 0};
    for (int d = 0; d < nd; d++) {
        std::vector<int> slot(K, -1);
        for (int j = 0; j < K; j++) {
            const int id = plan.ids[(size_t)j * nd + d];
            if (slot[id] < 0) {
                slot[id] = nmode[d]++;
                modes.push_back(tc[(size_t)j * nd + d]);
            }
            tidx[(size_t)j * nd + d] = (unsigned short)slot[id];
        }
    }
    const int Rc = R < 256 ? R : 256;   // realisations per launch
    const size_t off_se = 256 * ((sizeof(TCTerm) * tc.size() + 255) / 256);
    const size_t off_xi = off_se + 256 * ((8 * (size_t)K + 255) / 256);
    const size_t off_ch = off_xi + 256 * ((8 * (size_t)Rc * K + 255) / 256);
    const size_t off_cl = off_ch + 256 * ((4 * (size_t)Rc * K + 255) / 256);
    const size_t off_err = off_cl + 256 * ((4 * (size_t)Rc * K + 255) / 256);
    const size_t off_md = off_err + 256;
    const size_t off_ti = off_md + 256 * ((sizeof(TCTerm) * modes.size() + 255) / 256);
    void* buf = nullptr;
    CK(cudaMalloc(&buf, off_ti + 2 * tidx.size() + 16));
    char* b = (char*)buf;
    float total_ms = 0.f;
    do {
        if (cuda_fail(c, cudaMemcpyAsync(b, tc.data(), sizeof(TCTerm) * tc.size(), cudaMemcpyHostToDevice, c->st),
                      "cudaMemcpyAsync") ||
            cuda_fail(c, cudaMemcpyAsync(b + off_se, plan.sqrt_eig.data(), 8 * (size_t)K, cudaMemcpyHostToDevice,
                                         c->st), "cudaMemcpyAsync") ||
            cuda_fail(c, cudaMemsetAsync(b + off_err, 0, 16, c->st), "cudaMemsetAsync") ||
            cuda_fail(c, cudaMemcpyAsync(b + off_md, modes.data(), sizeof(TCTerm) * modes.size(),
                                         cudaMemcpyHostToDevice, c->st), "cudaMemcpyAsync") ||
            cuda_fail(c, cudaMemcpyAsync(b + off_ti, tidx.data(), 2 * tidx.size(), cudaMemcpyHostToDevice, c->st),
                      "cudaMemcpyAsync")) { rc = SPHGPU_E_CUDA; break; }
        const DevState& s = c->d[c->parity].s;
        for (int r0 = 0; r0 < R && !rc; r0 += Rc) {
            const int rr = (R - r0) < Rc ? (R - r0) : Rc;
            if (cuda_fail(c, cudaMemcpyAsync(b + off_xi, xi + (size_t)r0 * K, 8 * (size_t)rr * K,
                                             cudaMemcpyHostToDevice, c->st), "cudaMemcpyAsync")) { rc = SPHGPU_E_CUDA; break; }
            cudaEventRecord(c->ev0, c->st);
            if (sphk_kl_synthesize(N, nd, K, rr, f->no, f->type, xt, f->mean_value, f->sd_value, f->coe_depth,
                                   soil_max, water_max, s.xh, s.type, b, (const double*)(b + off_se),
                                   (const double*)(b + off_xi), (float*)(b + off_ch), (float*)(b + off_cl),
                                   d_out + (size_t)r0 * N, (int*)(b + off_err), c->st, b + off_md, nmode,
                                   (const unsigned short*)(b + off_ti))) {
                rc = cuda_fail(c, cudaGetLastError(), "K-L synthesis launch");
                if (!rc) rc = SPHGPU_E_ARG;
                break;
            }
            cudaEventRecord(c->ev1, c->st);
            if (cuda_fail(c, cudaStreamSynchronize(c->st), "cudaStreamSynchronize")) { rc = SPHGPU_E_CUDA; break; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, c->ev0, c->ev1);
            total_ms += ms;
            int err = 0;
            if (cuda_fail(c, cudaMemcpy(&err, b + off_err, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy")) {
                rc = SPHGPU_E_CUDA;
                break;
            }
            if (err) rc = err;
        }
    } while (0);
    cudaFree(buf);
    if (kernel_ms) *kernel_ms = total_ms;
    return rc;
}

}  // extern "C"
