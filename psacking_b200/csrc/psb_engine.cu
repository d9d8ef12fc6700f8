// psb_engine.cu — host side of the B200 placement-search engine and its C ABI.
//
// A psb_tray is the device-resident tray context (the reference's
// GPUTrayContext, spectral_packing/fft3.cu:1040-1460): tray, distance field,
// their half spectra, and per-orientation work buffers so that every
// orientation of a batch is searched by the same kernel launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include <atomic>
#include <thread>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include "../../include/psb200.h"
#include "psb_kernels2.cuh"
#include "psb_kernels3.cuh"
#include "psb_kernels4.cuh"
#include "psb_loop.cuh"
#include "psb_filter.cuh"
#include "psb_proposal.cuh"
#include "psb_voxel.cuh"
#include <nvtx3/nvToolsExt.h>

// NVTX range around a C-ABI call, so the engine's calls show on an Nsight
// Systems timeline next to their kernels; with no tool attached the range
// calls return at once.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

namespace {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess && (cudaGetLastError(), true))                                       \
            return fail(PSB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                 \
    } while (0)

#define CKL()                                                                                      \
    do {                                                                                           \
        cudaError_t e_ = cudaGetLastError();                                                       \
        if (e_ != cudaSuccess)                                                                     \
            return fail(PSB_ERR_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                 \
    } while (0)

#define TRY(x)                 \
    do {                       \
        int r_ = (x);          \
        if (r_ != PSB_OK) return r_; \
    } while (0)

constexpr double kP = 100000000.0;  // constants.h:7
constexpr int kCandCap = 1 << 18;

int ensure_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(PSB_ERR_NODEVICE, "no CUDA device visible (%s)", cudaGetErrorString(e));
    }
    return PSB_OK;
}

// ---------------------------------------------------------------------------
// per-launch CUDA-event profiler (psb_profile_*): off by default
// ---------------------------------------------------------------------------
struct ProfRec {
    const char* name;
    cudaEvent_t a, b;
};
struct Profiler {
    bool on = false;
    std::vector<std::string> only;  // when non-empty: record only these kernels
    std::vector<ProfRec> recs;
    std::vector<cudaEvent_t> pool;
    std::mutex mu;
    cudaEvent_t get() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
};
Profiler g_prof;

struct ProfScope {
    int idx = -1;
    cudaStream_t st;
    ProfScope(const char* name, cudaStream_t s) : st(s) {
        if (!g_prof.on) return;
        std::lock_guard<std::mutex> lk(g_prof.mu);
        if (!g_prof.only.empty() &&
            std::find(g_prof.only.begin(), g_prof.only.end(), std::string(name)) == g_prof.only.end())
            return;
        ProfRec r{name, g_prof.get(), g_prof.get()};
        cudaEventRecord(r.a, st);
        g_prof.recs.push_back(r);
        idx = (int)g_prof.recs.size() - 1;
    }
    ~ProfScope() {
        if (idx < 0) return;
        std::lock_guard<std::mutex> lk(g_prof.mu);
        cudaEventRecord(g_prof.recs[idx].b, st);
    }
};
#define PSB_CAT2(a, b) a##b
#define PSB_CAT(a, b) PSB_CAT2(a, b)
#define PROF(name, stream) ProfScope PSB_CAT(prof_, __LINE__)(name, stream)

// ---------------------------------------------------------------------------
// FFT plans: lengths with factors 2,3,5,7 up to PSB_MAX_FFT
// ---------------------------------------------------------------------------
bool factorize(int n, AxisPlan* p) {
    p->n = n;
    p->nstages = 0;
    int m = n;
    auto push = [&](int r) {
        if (p->nstages >= PSB_MAX_STAGES) return false;
        p->radix[p->nstages++] = r;
        m /= r;
        return true;
    };
    while (m % 8 == 0) if (!push(8)) return false;
    while (m % 4 == 0) if (!push(4)) return false;
    while (m % 2 == 0) if (!push(2)) return false;
    while (m % 3 == 0) if (!push(3)) return false;
    while (m % 5 == 0) if (!push(5)) return false;
    while (m % 7 == 0) if (!push(7)) return false;
    return m == 1;
}

int fft_len_smooth(int n) {
    for (int m = std::max(n, 1); m <= PSB_MAX_FFT; ++m) {
        AxisPlan p;
        if (factorize(m, &p)) return m;
    }
    return -1;
}

// Smallest 7-smooth length >= n, or the smallest length >= n with a
// specialised two-pass plan when that is at most 6% longer (e.g. 123 -> 128
// rather than 125: radices 16 x 8 instead of 25 x 5, fewer registers).
int fft_len(int n) {
    int s = fft_len_smooth(n);
    if (s < 0) return s;
    for (int m = s; m <= PSB_MAX_FFT && m <= s + s / 16; ++m)
        if (fast_len(m)) return m;
    return s;
}

struct Plan1D {
    AxisPlan p;
    float2* tw = nullptr;
};

std::mutex g_plan_mu;
std::map<std::pair<int, int>, Plan1D> g_plans;  // (device, n) -> plan

int get_plan(int n, Plan1D* out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_plans.find({dev, n});
    if (it != g_plans.end()) { *out = it->second; return PSB_OK; }
    Plan1D pl;
    if (!factorize(n, &pl.p)) return fail(PSB_ERR_ARG, "FFT length %d is not 7-smooth", n);
    std::vector<float2> tw(n);
    for (int i = 0; i < n; ++i) {
        double a = -2.0 * M_PI * (double)i / (double)n;
        tw[i] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    CK(cudaMalloc(&pl.tw, sizeof(float2) * n));
    CK(cudaMemcpy(pl.tw, tw.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
    g_plans[{dev, n}] = pl;
    *out = pl;
    return PSB_OK;
}

int g_smem_optin = 0;  // max dynamic shared memory per block of the current device
bool g_fast_fft = true;  // specialised two-pass kernels where a plan exists
// Tray grids (circular, F >= n) may be padded further: when every axis
// reaches a length with specialised kernels (x: 64, 100, 128, 240; y and z:
// 64, 100, 128) for at most g_pad_max times the volume, those lengths are
// taken, so the tray runs the specialised split flow (and its direct
// decisions) instead of the generic kernels.  The circular correlation stays
// exact for every translation the search scores (t + x <= n - 1 < F).
// 0 disables (PSB_PAD_MAX).  Default 3 (config-5 trays, 64 trays of sides
// 64-160: 0 -> 506, 2 -> 562, 3 -> 578 / 626 items placed/s).
double g_pad_max = 3.0;
// psb_pack stages its items in two parts when it has at least 2 x
// kStreamFirst of them: the first kStreamFirst before the loop, the rest
// while they are searched (PSB_STREAM_STAGE=0: all before the loop)
bool g_stream_stage = true;
constexpr int kStreamFirst = 32;


using XpassFn = void (*)(const OrientDesc*, SearchBufs, const float2*, const float2*, int, const float2*,
                         const unsigned char*, long long, BaseMap);
using PlaneFn = void (*)(const OrientDesc*, SearchBufs, PlaneBufs, ScoreParams, const float2*, const float2*);

// mode 0: both products, 1: collision only, 2: proximity only (gated);
// shared: the slabs come from the orientation's permutation base
XpassFn xpass2_for(int n, int mode = 0, bool shared = false) {
#define PSB_XP(N)                                                                                     \
    if (shared) return mode == 1 ? k_xpass2<N, 1, true> : (mode == 2 ? k_xpass2<N, 2, true> : k_xpass2<N, 0, true>); \
    return mode == 1 ? k_xpass2<N, 1, false> : (mode == 2 ? k_xpass2<N, 2, false> : k_xpass2<N, 0, false>)
    switch (n) {
        case 64: PSB_XP(64);
        case 100: PSB_XP(100);
        case 128: PSB_XP(128);
        case 240: PSB_XP(240);
        default: return nullptr;
    }
#undef PSB_XP
}

#define PSB_PLANE_ROW(NY)                      \
    case NY:                                   \
        switch (nz) {                          \
            case 64: return k_plane2<NY, 64>;   \
            case 100: return k_plane2<NY, 100>; \
            case 128: return k_plane2<NY, 128>; \
            default: return nullptr;           \
        }
PlaneFn plane2_for(int ny, int nz) {
    switch (ny) {
        PSB_PLANE_ROW(64)
        PSB_PLANE_ROW(100)
        PSB_PLANE_ROW(128)
        default: return nullptr;
    }
}
#undef PSB_PLANE_ROW

#define PSB_PLANE3_ROW(NY)                                                                \
    case NY:                                                                              \
        switch (nz) {                                                                     \
            case 64: return field ? k_plane3<NY, 64, 1> : k_plane3<NY, 64, 0>;             \
            case 100: return field ? k_plane3<NY, 100, 1> : k_plane3<NY, 100, 0>;          \
            case 128: return field ? k_plane3<NY, 128, 1> : k_plane3<NY, 128, 0>;          \
            default: return nullptr;                                                      \
        }
PlaneFn plane3_for(int ny, int nz, int field) {
    switch (ny) {
        PSB_PLANE3_ROW(64)
        PSB_PLANE3_ROW(100)
        PSB_PLANE3_ROW(128)
        default: return nullptr;
    }
}
#undef PSB_PLANE3_ROW

// plane-pass variant: 3 (warp-owned lines, collision and proximity in two
// launches with the flood fill between them, default) or 2 (both fields in
// one CTA-wide launch, lazy flood fill)
int g_plane_variant = 3;

// z,y slab transforms shared across the flips of a permutation
// (psb_kernels3.cuh).  Off by default: measured on the config-3 benchmark the
// x pass's per-element index map and phase cost more (+13 ms per run) than
// the 6-instead-of-24 slab transforms save (-3.4 ms: that launch is
// latency-bound, not work-bound).
bool g_share_flips = false;

// exact candidate pre-filter of the packing loop's collision searches
// (psb_filter.cuh); on by default
bool g_cand_filter = true;
// orientations left with at most this many candidates are decided directly
// (exact checks against the item's columns, exact proximity sums) instead of
// by transforms; 0 disables.  Measured on the config-3 benchmark (items
// placed/s): 1024: 1258.9, 2048: 1265.8, 4096: 1275.0 / 1277.2, 8192: 1268.1,
// 16384: 1247.3.
int g_direct_max = 4096;
// filter cut-off (k_cand_filter): a warp stops sampling when more than this
// percentage of its translations survive the first samples; 0 disables
int g_filter_cut = 50;
// the candidate filter as one CTA per x plane (and orientation group) with
// the tray's free-bit window staged in shared memory (k_cand_filter_plane),
// PSB_FILTER_PLANE=1 (or the group count).  Off: measured slower on the
// config-3 benchmark (items placed/s: off 1283.7 / 1285.2; on with 1, 2, 3,
// 4, 6 groups 1157.6, 1212.8, 1227.5, 1219.6, 1217.3): re-staging the
// ~100 KB window for every CTA costs more L2 traffic than the per-sample L1
// hits of the CTA-per-(plane, orientation) kernel.
bool g_filter_plane = false;
// (Several consecutive x planes per k_cand_filter CTA, sharing the staged
// samples, measured slower: 1, 2, 4, 8 planes 1453.8, 1423.4, 1362.8, 1270.7
// items placed/s; the kernel wants the parallelism more than the reuse.)
int g_filter_groups = 3;   // CTA rows of k_cand_filter_plane, each a third of the orientations
// CTA rows of the transform kernels when they take their orientations from
// the active list (k_active_list); 0: one row per orientation (PSB_ACTIVE_GRID)
int g_active_grid = 8;
// the flood fill and the selection kernels also loop over the searched
// orientations' list (PSB_LIST_SELECT=1).  Off: measured slower (same box,
// items placed/s: off 1243.3, on 1238.2; k_ff_union 9.4 -> 12.4 ms per run):
// those kernels hold no shared memory, so a CTA row per orientation costs
// little, and the list serialises orientations within a row.  Also measured
// with launch overlap on, and only for items the candidate filter ran on:
// lists there 1380.5 against 1405.3 without; the transform kernels with 2 /
// 3 / 4 instead of 8 CTA rows on those items 1146.5 / 1258.2 / 1286.8.
bool g_list_select = false;
// k_cand_filter variant for trays of at most 128 cells per column (tuning:
// 0 = 8-sample batches within 64 registers, 1 = 4-sample batches and 12
// CTAs per SM, 2 = 8-sample batches without a register bound, 3 = 16-sample
// batches); PSB_FILTER_VARIANT
int g_filter_variant = 0;
// bound on the flood fill's union-find retries and path steps (psb_set_uf_limit)
int g_uf_limit = PSB_UF_LIMIT;
// orientations left with at most this many ok cells after the collision pass
// skip the proximity transforms (psb_set_late_direct_max; 0 disables).  Off
// by default: measured on the config-3 benchmark (items placed/s) 0: 1208.5,
// 256: 1195.5, 1024: 1198.1, 4096: 1197.0 -- the orientations that reach the
// proximity pass hold many ok cells.
int g_late_max = 0;

// the 6 axis permutations of an orientation map, as base indices
int perm_index(const int* a) {
    static const int tab[27] = {-1, -1, -1, -1, -1, 0, -1, 1, -1, -1, -1, 2, -1, -1, -1, 3, -1, -1,
                                -1, 4, -1, 5, -1, -1, -1, -1, -1};
    return tab[a[0] * 9 + a[1] * 3 + a[2]];
}

using FwdPlaneFn = void (*)(FwdSrc, const OrientDesc*, const float2*, const float2*);
using XfwdFn = void (*)(const float2*, float2*, int, int, const int*, const float2*);

#define PSB_FWD_ROW(NY)                           \
    case NY:                                      \
        switch (nz) {                             \
            case 64: return k_fwd_plane<NY, 64>;   \
            case 100: return k_fwd_plane<NY, 100>; \
            case 128: return k_fwd_plane<NY, 128>; \
            default: return nullptr;              \
        }
FwdPlaneFn fwd_plane_for(int ny, int nz) {
    switch (ny) {
        PSB_FWD_ROW(64)
        PSB_FWD_ROW(100)
        PSB_FWD_ROW(128)
        default: return nullptr;
    }
}
#undef PSB_FWD_ROW

XfwdFn xfwd_for(int n) {
    switch (n) {
        case 64: return k_xfwd<64>;
        case 100: return k_xfwd<100>;
        case 128: return k_xfwd<128>;
        case 240: return k_xfwd<240>;
        default: return nullptr;
    }
}

// register-DFT twiddles W_R^i for R <= 32 (offset R*(R-1)/2)
int init_register_twiddles() {
    std::vector<float2> t(PSB_TWR_SIZE);
    for (int R = 1; R <= 32; ++R)
        for (int i = 0; i < R; ++i) {
            double a = -2.0 * M_PI * (double)i / (double)R;
            t[R * (R - 1) / 2 + i] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
    CK(cudaMemcpyToSymbol(c_twr, t.data(), sizeof(float2) * PSB_TWR_SIZE));
    return PSB_OK;
}

template <class K>
int set_max_dyn_smem(K func) {
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, func));
    int dyn = g_smem_optin - (int)fa.sharedSizeBytes;
    CK(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    return PSB_OK;
}

int set_smem_attrs() {
    static bool done[64] = {false};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 64 && done[dev]) return PSB_OK;
    CK(cudaDeviceGetAttribute(&g_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (const char* e = getenv("PSB_PLANE_VARIANT")) g_plane_variant = atoi(e) == 2 ? 2 : 3;
    if (const char* e = getenv("PSB_SHARE_FLIPS")) g_share_flips = atoi(e) != 0;
    if (const char* e = getenv("PSB_CAND_FILTER")) g_cand_filter = atoi(e) != 0;
    if (const char* e = getenv("PSB_DIRECT_MAX")) g_direct_max = std::max(0, atoi(e));
    if (const char* e = getenv("PSB_FILTER_CUT")) g_filter_cut = std::max(0, std::min(100, atoi(e)));
    if (const char* e = getenv("PSB_ACTIVE_GRID")) g_active_grid = std::max(0, atoi(e));
    if (const char* e = getenv("PSB_PAD_MAX")) g_pad_max = std::max(0.0, atof(e));
    if (const char* e = getenv("PSB_FAST_FFT")) g_fast_fft = atoi(e) != 0;
    if (const char* e = getenv("PSB_LIST_SELECT")) g_list_select = atoi(e) != 0;
    if (const char* e = getenv("PSB_FILTER_VARIANT")) g_filter_variant = std::max(0, std::min(3, atoi(e)));
    if (const char* e = getenv("PSB_FILTER_PLANE")) {
        g_filter_plane = atoi(e) != 0;
        if (atoi(e) > 1) g_filter_groups = atoi(e);
    }
    if (const char* e = getenv("PSB_PDL")) g_pdl = atoi(e) != 0;
    if (const char* e = getenv("PSB_STREAM_STAGE")) g_stream_stage = atoi(e) != 0;
    if (const char* e = getenv("PSB_LATE_MAX")) g_late_max = std::min(std::max(0, atoi(e)), kCandCap);
    TRY(set_max_dyn_smem(k_rfft_z));
    TRY(set_max_dyn_smem(k_irfft_z_int));
    TRY(set_max_dyn_smem(k_fft_mid<-1>));
    TRY(set_max_dyn_smem(k_fft_mid<1>));
    TRY(set_max_dyn_smem(k_xpass));
    TRY(set_max_dyn_smem(k_plane));
    TRY(set_max_dyn_smem(k_dist_axis));
    for (int n : {64, 100, 128, 240})
        for (int m = 0; m < 3; ++m) {
            TRY(set_max_dyn_smem(xpass2_for(n, m, false)));
            TRY(set_max_dyn_smem(xpass2_for(n, m, true)));
        }
    for (int a : {64, 100, 128})
        for (int b : {64, 100, 128}) {
            TRY(set_max_dyn_smem(plane2_for(a, b)));
            TRY(set_max_dyn_smem(plane3_for(a, b, 0)));
            TRY(set_max_dyn_smem(plane3_for(a, b, 1)));
            TRY(set_max_dyn_smem(fwd_plane_for(a, b)));
        }
    for (int n : {64, 100, 128, 240}) TRY(set_max_dyn_smem(xfwd_for(n)));
    TRY(set_max_dyn_smem(k_cand_filter_plane<1>));
    TRY(set_max_dyn_smem(k_cand_filter_plane<2>));
    TRY(init_register_twiddles());
    if (dev < 64) done[dev] = true;
    return PSB_OK;
}

// Device allocations.  With a stream they are stream-ordered (the tray's own
// stream), so creating and freeing trays never synchronises the whole device
// while other trays are running.
//
// Test hooks (psb_debug_fail_alloc, psb_debug_live_allocs): the n-th
// allocation from the moment the hook is armed fails as a CUDA error would,
// and the allocations made here and not yet freed are counted, so the tests
// can check that every failure path returns PSB_ERR_CUDA and frees what it
// allocated.
std::atomic<int> g_fail_alloc{0};
std::atomic<long long> g_live_allocs{0};

template <class T>
int dalloc(T** p, size_t n, cudaStream_t s = nullptr) {
    *p = nullptr;
    if (n == 0) n = 1;
    if (g_fail_alloc.load() > 0 && g_fail_alloc.fetch_sub(1) == 1)
        return fail(PSB_ERR_CUDA, "device allocation of %zu B failed (injected by psb_debug_fail_alloc)",
                    sizeof(T) * n);
    if (s) {
        CK(cudaMallocAsync((void**)p, sizeof(T) * n, s));
    } else {
        CK(cudaMalloc((void**)p, sizeof(T) * n));
    }
    g_live_allocs.fetch_add(1);
    return PSB_OK;
}

template <class T>
void dfree(T*& p, cudaStream_t s = nullptr) {
    if (p) {
        if (s) cudaFreeAsync(p, s);
        else cudaFree(p);
        g_live_allocs.fetch_sub(1);
    }
    p = nullptr;
}

int grid1d(size_t n, int block = 256) {
    size_t g = (n + block - 1) / block;
    return (int)std::max<size_t>(1, std::min<size_t>(g, 148 * 32));
}

// ---------------------------------------------------------------------------
// real 3-D transforms on an (n0,n1,n2) grid with FFT dims (F0,F1,F2)
// ---------------------------------------------------------------------------
struct Grid3 {
    int n[3];
    int F[3];
    int H;  // F2/2 + 1
    Plan1D p[3];
};

int next_special(int n, bool x_axis) {
    const int xs[4] = {64, 100, 128, 240}, yz[3] = {64, 100, 128};
    const int* set = x_axis ? xs : yz;
    const int m = x_axis ? 4 : 3;
    for (int i = 0; i < m; ++i)
        if (set[i] >= n) return set[i];
    return -1;
}

int make_grid3(int nx, int ny, int nz, bool linear, Grid3* g) {
    g->n[0] = nx; g->n[1] = ny; g->n[2] = nz;
    for (int a = 0; a < 3; ++a) {
        int want = linear ? 2 * g->n[a] - 1 : g->n[a];
        g->F[a] = fft_len(want);
        if (g->F[a] < 0)
            return fail(PSB_ERR_ARG, "axis %d of length %d needs an FFT longer than %d", a, g->n[a], PSB_MAX_FFT);
    }
    if (!linear && g_fast_fft && g_pad_max > 0.0) {
        int P[3];
        bool all = true;
        for (int a = 0; a < 3; ++a) {
            P[a] = next_special(g->n[a], a == 0);
            all = all && P[a] > 0;
        }
        if (all && !(P[0] == g->F[0] && P[1] == g->F[1] && P[2] == g->F[2])) {
            const double ratio = ((double)P[0] * P[1] * P[2]) / ((double)g->F[0] * g->F[1] * g->F[2]);
            if (ratio <= g_pad_max)
                for (int a = 0; a < 3; ++a) g->F[a] = P[a];
        }
    }
    for (int a = 0; a < 3; ++a) TRY(get_plan(g->F[a], &g->p[a]));
    g->H = g->F[2] / 2 + 1;
    return PSB_OK;
}

size_t smem_rz(int N) { return sizeof(float2) * (N + 2 * PSB_PAIRS * N); }
size_t smem_mid(int N) { return sizeof(float2) * (N + 2 * PSB_TILE * N); }

// forward with descriptors already on the device: d_rz[0] (z pass, out = w1),
// d_mid[0] (y pass w1 -> w2), d_mid[1] (x pass w2 -> spectrum).  No host copies,
// so it can be queued inside the asynchronous packing loop.
int forward3_dev(const Grid3& g, const RzDesc* d_rz, const MidDesc* d_mid, cudaStream_t st) {
    int npairs = (g.n[0] * g.n[1] + 1) / 2;
    {
        PROF("k_rfft_z", st);
        pdl(k_rfft_z, dim3((npairs + PSB_PAIRS - 1) / PSB_PAIRS, 1), PSB_THREADS, smem_rz(g.F[2]), st)(
            d_rz, nullptr, g.p[2].p, g.p[2].tw);
    }
    CKL();
    {
        PROF("k_fft_mid_fwd", st);
        pdl(k_fft_mid<-1>, dim3((g.H + PSB_TILE - 1) / PSB_TILE, g.n[0], 1), PSB_THREADS, smem_mid(g.F[1]), st)(
            d_mid, nullptr, g.p[1].p, g.p[1].tw);
    }
    CKL();
    {
        PROF("k_fft_mid_fwd", st);
        pdl(k_fft_mid<-1>, dim3((g.F[1] * g.H + PSB_TILE - 1) / PSB_TILE, 1, 1), PSB_THREADS, smem_mid(g.F[0]), st)(
            d_mid + 1, nullptr, g.p[0].p, g.p[0].tw);
    }
    CKL();
    return PSB_OK;
}

// the two MidDescs of a forward transform (w1 -> w2 -> spec)
void forward_mids(const Grid3& g, float2* w1, float2* w2, float2* spec, const int* gate, MidDesc* m) {
    // y: [n0][n1->F1][H]
    m[0] = MidDesc{w1, w2, g.n[0], g.H, g.n[1], g.F[1], (long long)g.n[1] * g.H, (long long)g.F[1] * g.H, g.H, g.H,
                   -1, 0, gate};
    // x: [1][n0->F0][F1*H]
    m[1] = MidDesc{w2, spec, 1, g.F[1] * g.H, g.n[0], g.F[0], 0, 0, g.F[1] * g.H, g.F[1] * g.H, -1, 0, gate};
}

// forward: src grid -> spectrum [F0][F1][H].  w1: [n0][n1][H], w2: [n0][F1][H]
int forward3(const Grid3& g, const RzDesc& rz_in, float2* w1, float2* w2, float2* spec, RzDesc* d_rz,
             MidDesc* d_mid, cudaStream_t st) {
    RzDesc rz = rz_in;
    rz.out = w1;
    CK(cudaMemcpyAsync(d_rz, &rz, sizeof(rz), cudaMemcpyHostToDevice, st));
    MidDesc m[2];
    forward_mids(g, w1, w2, spec, nullptr, m);
    CK(cudaMemcpyAsync(d_mid, m, sizeof(m), cudaMemcpyHostToDevice, st));
    return forward3_dev(g, d_rz, d_mid, st);
}

int inverse3_dev(const Grid3& g, float2* w1, int32_t* out, const MidDesc* d_mid, cudaStream_t st);

// inverse: spectrum [F0][F1][H] -> int32 grid (rounded, scaled by 1/(F0 F1 F2))
int inverse3_int(const Grid3& g, float2* spec, float2* w1, float2* w2, int32_t* out, MidDesc* d_mid,
                 cudaStream_t st) {
    MidDesc m[2];
    // x: [1][F0 -> n0][F1*H]   (spec -> w2 [n0][F1][H])
    m[0] = MidDesc{spec, w2, 1, g.F[1] * g.H, g.F[0], g.n[0], 0, 0, g.F[1] * g.H, g.F[1] * g.H, -1, 0};
    // y: [n0][F1 -> n1][H]     (w2 -> w1 [n0][n1][H])
    m[1] = MidDesc{w2, w1, g.n[0], g.H, g.F[1], g.n[1], (long long)g.F[1] * g.H, (long long)g.n[1] * g.H, g.H, g.H, -1, 0};
    CK(cudaMemcpyAsync(d_mid, m, sizeof(m), cudaMemcpyHostToDevice, st));
    return inverse3_dev(g, w1, out, d_mid, st);
}

// inverse with its two MidDescs already on the device (d_mid[0]: x pass
// spectrum -> w2, d_mid[1]: y pass w2 -> w1), then the z C2R from w1
int inverse3_dev(const Grid3& g, float2* w1, int32_t* out, const MidDesc* d_mid, cudaStream_t st) {
    {
        PROF("k_fft_mid_inv", st);
        pdl(k_fft_mid<1>, dim3((g.F[1] * g.H + PSB_TILE - 1) / PSB_TILE, 1, 1), PSB_THREADS, smem_mid(g.F[0]), st)(
            d_mid, nullptr, g.p[0].p, g.p[0].tw);
    }
    CKL();
    {
        PROF("k_fft_mid_inv", st);
        pdl(k_fft_mid<1>, dim3((g.H + PSB_TILE - 1) / PSB_TILE, g.n[0], 1), PSB_THREADS, smem_mid(g.F[1]), st)(
            d_mid + 1, nullptr, g.p[1].p, g.p[1].tw);
    }
    CKL();
    int nlines = g.n[0] * g.n[1];
    float scale = (float)(1.0 / ((double)g.F[0] * g.F[1] * g.F[2]));
    {
        PROF("k_irfft_z_int", st);
        pdl(k_irfft_z_int, ((nlines + 1) / 2 + PSB_PAIRS - 1) / PSB_PAIRS, PSB_THREADS, smem_rz(g.F[2]), st)(
            w1, out, nlines, g.n[2], scale, g.p[2].p, g.p[2].tw);
    }
    CKL();
    return PSB_OK;
}

int distance_on_device(const int32_t* d_grid, int32_t* d_out, int nx, int ny, int nz, cudaStream_t st,
                       const int* gate = nullptr) {
    size_t V = (size_t)nx * ny * nz;
    int far = nx + ny + nz + 10;  // fft3.cu:948
    {
        PROF("k_dist_init", st);
        pdl(k_dist_init, grid1d(V), 256, 0, st)(d_grid, d_out, V, far, gate);
    }
    CKL();
    for (int axis = 0; axis < 3; ++axis) {
        int L = axis == 0 ? nx : (axis == 1 ? ny : nz);
        long long nlines = axis == 0 ? (long long)ny * nz : (axis == 1 ? (long long)nx * nz : (long long)nx * ny);
        if (L <= 1) continue;
        long long W = std::min<long long>(256, (96 * 1024) / (4LL * L));
        if (W >= 1) {
            long long blocks = (nlines + W - 1) / W;
            {
                PROF("k_dist_axis", st);
                pdl(k_dist_axis, (unsigned)blocks, 256, (size_t)W * L * 4, st)(d_out, axis, nx, ny, nz, (int)W, gate);
            }
        } else {
            {
                PROF("k_dist_axis_global", st);
                pdl(k_dist_axis_global, (unsigned)((nlines + 255) / 256), 256, 0, st)(d_out, axis, nx, ny, nz, gate);
            }
        }
        CKL();
    }
    return PSB_OK;
}

int check_grid_args(const void* p, int nx, int ny, int nz, const char* what) {
    if (!p) return fail(PSB_ERR_ARG, "%s: null pointer", what);
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail(PSB_ERR_ARG, "%s: dims must be positive, got (%d,%d,%d)", what, nx, ny, nz);
    return PSB_OK;
}

bool has_negative(const int32_t* a, size_t n) {
    for (size_t i = 0; i < n; ++i) if (a[i] < 0) return true;
    return false;
}

// fn(begin, end) over [0, n) in chunks, on up to all host cores (the calling
// thread takes part); a single chunk runs inline.
template <typename F>
void parallel_chunks(size_t n, size_t chunk, F fn) {
    const size_t nchunks = (n + chunk - 1) / chunk;
    const int nthr = (int)std::min<size_t>(nchunks, std::max(1u, std::thread::hardware_concurrency()));
    if (nthr <= 1) {
        if (n) fn((size_t)0, n);
        return;
    }
    std::atomic<size_t> next(0);
    auto work = [&]() {
        for (size_t c = next.fetch_add(1); c < nchunks; c = next.fetch_add(1))
            fn(c * chunk, std::min(n, (c + 1) * chunk));
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < nthr; ++w) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
}

// ---------------------------------------------------------------------------
// host-side item analysis
// ---------------------------------------------------------------------------
struct ItemInfo {
    int dims[3];
    int lo[3], hi[3];          // bounds of voxels > 0; hi = -1 when none
    long long sum = 0;         // sum of values
    long long sabs = 0;        // sum of |values|
    double sumsq = 0.0;
    long long nvox = 0;        // nonzero voxels
    std::vector<int4> vox;     // their list (x, y, z, value), when asked for
    std::vector<int4> samp;    // candidate-filter samples (positive voxels, spread out)
    std::vector<int4> runs[3]; // runs of equal nonzero values along each source axis (build_runs)
};

// The item's runs along source axis s, in the layout orient_run reads
// ({u, v, r0 | r1 << 16, value}, psb_kernels.cuh): the exact proximity and
// collision sums of a translation then cost one pair of prefix-table loads
// per run instead of one load per voxel.
void build_runs(const int32_t* a, ItemInfo* info, int s) {
    std::vector<int4>& out = info->runs[s];
    out.clear();
    const int* d = info->dims;
    const int lo = s == 0 ? 1 : 0, hi = s == 2 ? 1 : 2;
    const size_t stride[3] = {(size_t)d[1] * d[2], (size_t)d[2], 1};
    const size_t sl = stride[lo], sh = stride[hi], ss = stride[s];
    const int len = d[s];
    for (int u = 0; u < d[lo]; ++u)
        for (int v = 0; v < d[hi]; ++v) {
            const int32_t* line = a + u * sl + v * sh;
            int r0 = -1, w = 0;
            for (int r = 0; r <= len; ++r) {
                const int val = r < len ? line[r * ss] : 0;
                if (r0 >= 0 && val != w) {
                    out.push_back(make_int4(u, v, r0 | ((r - 1) << 16), w));
                    r0 = -1;
                }
                if (r0 < 0 && val != 0) {
                    r0 = r;
                    w = val;
                }
            }
        }
}

// Up to PSB_FSAMP positive voxels spread over the item, for the candidate
// filter.  Pool: in each cell of a 10x10x10 split of the item's box, the
// voxel farthest from the box centre (extreme voxels are the ones that stop
// an item from fitting a gap; the first such voxel in row-major order).
// Order: farthest-point (each next sample is the pool voxel farthest from
// those taken), starting from the voxel farthest from the centre, so the
// filter's first samples already span the item.  Any subset is exact for the
// filter; the spread only makes it sharp.  Read from the item's z-runs
// (build_runs, axis 2), which list the nonzero voxels in row-major order:
// within the part of a run that falls in one split cell the squared distance
// to the centre is a convex function of z (and exact in float: sums of
// squared half-integers below 2^24), so the farthest voxel there is one of
// the part's two ends, the lower one on a tie.
void pick_samples(ItemInfo* info) {
    info->samp.clear();
    const int G = 10;
    const int* d = info->dims;
    const float cx = 0.5f * (d[0] - 1), cy = 0.5f * (d[1] - 1), cz = 0.5f * (d[2] - 1);
    auto d2 = [](const int4& a, float x, float y, float z) {
        return (a.x - x) * (a.x - x) + (a.y - y) * (a.y - y) + (a.z - z) * (a.z - z);
    };
    // the split cell of each coordinate, per axis (c * G / extent)
    std::vector<int> cell_of[3];
    for (int q = 0; q < 3; ++q) {
        cell_of[q].resize(d[q]);
        for (int c = 0; c < d[q]; ++c) cell_of[q][c] = c * G / d[q];
    }
    std::vector<int4> best(G * G * G, make_int4(0, 0, 0, 0));   // w = 0: cell empty
    std::vector<float> bd(G * G * G, 0.f);
    const std::vector<int4>& zr = info->runs[2];
    for (const int4& q : zr) {
        if (q.w <= 0) continue;
        const int i = q.x, j = q.y, z1 = q.z >> 16;
        const int cij = (cell_of[0][i] * G + cell_of[1][j]) * G;
        for (int k = q.z & 0xffff; k <= z1;) {
            const int c = cell_of[2][k];
            int e = k;
            while (e < z1 && cell_of[2][e + 1] == c) ++e;
            const int4 vk = make_int4(i, j, k, q.w), ve = make_int4(i, j, e, q.w);
            const float dk = d2(vk, cx, cy, cz), de = d2(ve, cx, cy, cz);
            const int4 v = de > dk ? ve : vk;
            const float dist = de > dk ? de : dk;
            const int cell = cij + c;
            if (best[cell].w == 0 || dist > bd[cell]) { best[cell] = v; bd[cell] = dist; }
            k = e + 1;
        }
    }
    std::vector<int4> pool;
    for (const int4& b : best)
        if (b.w != 0) pool.push_back(b);
    if (pool.empty()) return;
    size_t k = 0;
    for (size_t i = 1; i < pool.size(); ++i)
        if (d2(pool[i], cx, cy, cz) > d2(pool[k], cx, cy, cz)) k = i;
    // farthest-point order over the pool, structure of arrays; a taken entry
    // holds -1 in dmin, below every distance, so it is never picked again
    const size_t P = pool.size();
    std::vector<float> fx(P), fy(P), fz(P), dmin(P, 3.0e38f);
    for (size_t i = 0; i < P; ++i) {
        fx[i] = (float)pool[i].x;
        fy[i] = (float)pool[i].y;
        fz[i] = (float)pool[i].z;
    }
    const size_t m = std::min(P, (size_t)PSB_FSAMP);
    while (info->samp.size() < m) {
        dmin[k] = -1.f;
        info->samp.push_back(pool[k]);
        const float kx = fx[k], ky = fy[k], kz = fz[k];
        float far = -1.f;
        size_t i = 0;
#if defined(__SSE2__)
        // four lanes at a time: the same single-precision products, sums and
        // min as the scalar form below (minps(a, b) = a < b ? a : b)
        const __m128 vx = _mm_set1_ps(kx), vy = _mm_set1_ps(ky), vz = _mm_set1_ps(kz);
        __m128 vfar = _mm_set1_ps(-1.f);
        for (; i + 4 <= P; i += 4) {
            const __m128 dx = _mm_sub_ps(_mm_loadu_ps(&fx[i]), vx);
            const __m128 dy = _mm_sub_ps(_mm_loadu_ps(&fy[i]), vy);
            const __m128 dz = _mm_sub_ps(_mm_loadu_ps(&fz[i]), vz);
            const __m128 dd = _mm_add_ps(_mm_add_ps(_mm_mul_ps(dx, dx), _mm_mul_ps(dy, dy)), _mm_mul_ps(dz, dz));
            const __m128 dm = _mm_min_ps(dd, _mm_loadu_ps(&dmin[i]));
            _mm_storeu_ps(&dmin[i], dm);
            vfar = _mm_max_ps(vfar, dm);
        }
        float lanes[4];
        _mm_storeu_ps(lanes, vfar);
        far = std::max(std::max(lanes[0], lanes[1]), std::max(lanes[2], lanes[3]));
#endif
        for (; i < P; ++i) {
            const float dx = fx[i] - kx, dy = fy[i] - ky, dz = fz[i] - kz;
            dmin[i] = std::min(dmin[i], dx * dx + dy * dy + dz * dz);
            far = std::max(far, dmin[i]);
        }
        if (!(far > -1.f)) break;   // every pool voxel taken
        size_t nk = 0;
#if defined(__SSE2__)
        const __m128 vf = _mm_set1_ps(far);
        for (; nk + 4 <= P; nk += 4) {
            const int hit = _mm_movemask_ps(_mm_cmpeq_ps(_mm_loadu_ps(&dmin[nk]), vf));
            if (hit) { nk += __builtin_ctz(hit); break; }
        }
#endif
        while (dmin[nk] != far) ++nk;   // the first farthest
        k = nk;
    }
}

// analyse_item's bounds and sums from the item's z-runs (no pass over the
// dense array).  The sum of squares adds one term per voxel in row-major
// order, as analyse_item does, unless every partial sum is an integer below
// 2^53 (then any order gives the same double).
void analyse_runs(ItemInfo* info) {
    for (int k = 0; k < 3; ++k) { info->lo[k] = INT32_MAX; info->hi[k] = -1; }
    info->sum = 0;
    info->sabs = 0;
    info->sumsq = 0.0;
    info->nvox = 0;
    info->vox.clear();
    const std::vector<int4>& zr = info->runs[2];
    long long wmax = 0;
    for (const int4& q : zr) wmax = std::max(wmax, std::llabs((long long)q.w));
    long long n = 0;
    for (const int4& q : zr) n += (q.z >> 16) - (q.z & 0xffff) + 1;
    const bool exact = wmax <= 32768 && n < (1LL << 22);   // n * wmax^2 < 2^52
    long long isq = 0;
    for (const int4& q : zr) {
        const int z0 = q.z & 0xffff, z1 = q.z >> 16, len = z1 - z0 + 1;
        const long long w = q.w;
        info->nvox += len;
        info->sum += w * len;
        info->sabs += std::llabs(w) * len;
        if (exact) isq += w * w * len;
        else
            for (int k = 0; k < len; ++k) info->sumsq += (double)w * (double)w;
        if (w > 0) {
            info->lo[0] = std::min(info->lo[0], q.x); info->hi[0] = std::max(info->hi[0], q.x);
            info->lo[1] = std::min(info->lo[1], q.y); info->hi[1] = std::max(info->hi[1], q.y);
            info->lo[2] = std::min(info->lo[2], z0);  info->hi[2] = std::max(info->hi[2], z1);
        }
    }
    if (exact) info->sumsq = (double)isq;
}

void analyse_item(const int32_t* a, int ex, int ey, int ez, ItemInfo* info, bool keep_vox = true) {
    info->dims[0] = ex; info->dims[1] = ey; info->dims[2] = ez;
    for (int k = 0; k < 3; ++k) { info->lo[k] = INT32_MAX; info->hi[k] = -1; }
    info->sum = 0;
    info->sabs = 0;
    info->sumsq = 0.0;
    info->nvox = 0;
    info->vox.clear();
    for (int i = 0; i < ex; ++i)
        for (int j = 0; j < ey; ++j)
            for (int k = 0; k < ez; ++k) {
                int v = a[((size_t)i * ey + j) * ez + k];
                if (v == 0) continue;
                info->nvox += 1;
                if (keep_vox) info->vox.push_back(make_int4(i, j, k, v));
                info->sum += v;
                info->sabs += std::llabs((long long)v);
                info->sumsq += (double)v * v;
                if (v > 0) {
                    int c[3] = {i, j, k};
                    for (int q = 0; q < 3; ++q) {
                        info->lo[q] = std::min(info->lo[q], c[q]);
                        info->hi[q] = std::max(info->hi[q], c[q]);
                    }
                }
            }
}

double ulp32(double v) {
    if (v < 1.0) return 1.19209290e-07;
    int e;
    std::frexp(v, &e);  // v = m * 2^e, m in [0.5,1)
    return std::ldexp(1.0, e - 24);
}

}  // namespace

// The item's 6 axis permutations as base descriptors (no flips), and each
// orientation's base index.  A base is skipped when it does not fit the tray
// (the same for all flips of it) or no orientation uses it.  Returns false
// (no sharing possible) unless every orientation turns the same item: the
// synchronous entry points take explicit arrays, which may be different
// items described as identity maps.
bool make_bases(std::vector<OrientDesc>* ods, std::vector<OrientDesc>* bases) {
    for (auto& od : *ods)
        if (od.item != (*ods)[0].item || od.b[0] != (*ods)[0].b[0] || od.b[1] != (*ods)[0].b[1] ||
            od.b[2] != (*ods)[0].b[2])
            return false;
    bases->assign(6, OrientDesc());
    for (auto& b : *bases) {
        memset(&b, 0, sizeof(b));
        b.skip = 1;
        b.perm = -1;
    }
    std::vector<char> used(6, 0);
    for (auto& od : *ods) {
        const int p = perm_index(od.src_axis);
        od.perm = p;
        if (p < 0 || used[p]) continue;
        OrientDesc b = od;
        b.flip[0] = b.flip[1] = b.flip[2] = 0;
        b.perm = p;
        (*bases)[p] = b;
        used[p] = 1;
    }
    return true;
}

// ===========================================================================
// psb_tray: the device-resident tray context
// ===========================================================================
struct psb_tray {
    int dev = 0;
    int nx = 0, ny = 0, nz = 0;
    size_t V = 0;
    Grid3 g;
    int nzw = 0;
    cudaStream_t st = nullptr;
    bool ready = false;

    int32_t* d_tray = nullptr;
    int32_t* d_phi = nullptr;
    float2* d_Socc = nullptr;
    float2* d_Sphi = nullptr;
    float2* d_w1 = nullptr;
    float2* d_w2 = nullptr;
    float2* d_wocc = nullptr;   // z,y transforms of the occupancy's x slabs, kept between placements
    double* d_pen = nullptr;
    RzDesc* d_rz = nullptr;
    MidDesc* d_mid = nullptr;
    unsigned long long* d_stats = nullptr;
    unsigned int* d_err = nullptr;
    unsigned long long* d_first = nullptr;

    int subbatch = 0;        // orientations per x-pass/plane-pass launch pair (0: all)

    // asynchronous packing loop: device state, distance statistics and the
    // transform descriptors of the occupancy / distance spectra (uploaded once)
    LoopState* d_ls = nullptr;
    PhiStats* d_ps = nullptr;
    int* d_ostat = nullptr;    // k_occ_stats output: occupied count (8 bytes) + bounding box
    RzDesc* d_rzd = nullptr;    // [0] occ, [1] phi, [2] occ gated, [3] phi gated
    MidDesc* d_midd = nullptr;  // pairs in the same order
    OrientDesc* d_od_all = nullptr;
    size_t od_all_cap = 0;
    OrientDesc* d_base_all = nullptr;   // 6 axis-permutation bases per staged item
    size_t base_all_cap = 0;
    DecisionDev* d_dec = nullptr;
    size_t dec_cap = 0;

    int phi_mean = 0;
    double phi_norm = 0.0;
    int phi_maxabs = 0;

    // per-orientation slots
    int cap = 0;
    float2 *d_Ai = nullptr, *d_Bi = nullptr, *d_Pc = nullptr, *d_Pd = nullptr;
    float* d_Dq = nullptr;
    uint32_t *d_free = nullptr, *d_reach = nullptr;
    int *d_cnt = nullptr, *d_off = nullptr, *d_rz2 = nullptr, *d_rline = nullptr, *d_par = nullptr, *d_rflag = nullptr,
        *d_total = nullptr, *d_blk = nullptr;
    int *d_cand = nullptr, *d_ncand = nullptr;
    double* d_cscore = nullptr;
    unsigned long long *d_smin = nullptr, *d_best = nullptr, *d_bestkey = nullptr;
    unsigned long long* d_pmin = nullptr;   // per (orientation, x plane) minimum approximate score key
    int* d_needff = nullptr;                // lazy interlocking search: flood fill needed
    unsigned char* d_okplane = nullptr;     // per (orientation, x plane): holds an ok cell
    unsigned char* d_candplane = nullptr;   // per (orientation, x plane): holds a filter candidate
    bool cand_active = false;               // the current search's candidate words and planes are valid
    const PhiStats* prep_ps = nullptr;      // when set, k_cand_prep also does k_prep's work
    bool pending_apply = false;             // stage 1 of k_cand_apply still to run on the current item
    int apply_dmax = 0;
    bool direct_active = false;             // ... and direct orientations may exist
    bool late_active = false;               // the current search may hold late-direct orientations
    DecideArgs decide{nullptr, nullptr, nullptr, nullptr};   // the loop's decision, fused into the
    bool fused = false;                                      // split flow's last selection step (done)
    int *d_ccount = nullptr, *d_vcount = nullptr, *d_ncol = nullptr;   // per orientation: candidates,
                                                                      // verified free cells, item columns
    int* d_okcount = nullptr;               // per orientation: ok cells after the collision pass
    int* d_act = nullptr;                   // the search's active orientations (k_active_list), and
    int* d_nact = nullptr;                  // their count
    int* d_srch = nullptr;                  // the searched orientations (not skipped), and
    int* d_nsrch = nullptr;                 // their count
    bool act_ready = false;                 // the current search's active list is queued
    int* d_clist = nullptr;                 // per orientation: its filter candidates while few (k_cand_filter)
    size_t clist_cap = 0;
    uint4* d_icols = nullptr;               // item column masks of direct orientations, stride nx*ny
    int4* d_fsamp = nullptr;                // oriented, shift-sorted filter samples (k_cand_prep)
    int* d_fbound = nullptr;                // their bucket bounds
    uint4* d_tbits = nullptr;               // free bits of the tray (k_tray_bits), tq uint4 per column
    int tq = 0;
    unsigned long long* d_work = nullptr;   // collision-kernel work counters (SearchBufs::work)
    size_t occ = 0;                         // occupied cells of the tray, kept on the host
    OrientDesc* d_bases = nullptr;          // their descriptors (synchronous searches)
    unsigned int* d_diag = nullptr;
    unsigned int* d_errmax = nullptr;
    OrientDesc* d_od = nullptr;
    RzDesc* d_rzs = nullptr;
    MidDesc* d_mids = nullptr;
    ResultDev* d_res = nullptr;
    long long sAi = 0, sBi = 0, sP = 0, sD = 0, sBits = 0, sLine = 0, sRun = 0;

    // items of a packing run, staged once (psb_pack_stage) in one part, or
    // in two by psb_pack (the second part analysed and uploaded while the
    // first part's items are searched).  A part is one device block (runs,
    // samples, dense arrays) filled from one pinned host block.
    std::vector<ItemInfo> staged;
    struct StagedDev {
        const int32_t* item;    // the item's int32 array
        const int4* samp;       // its filter samples
        const int4* runs[3];    // its runs along each source axis
    };
    std::vector<StagedDev> sdev;
    char* d_part[2] = {nullptr, nullptr};
    size_t part_cap[2] = {0, 0};
    void* h_part[2] = {nullptr, nullptr};
    size_t h_part_cap[2] = {0, 0};
    void* h_desc = nullptr;          // pinned copy of the run's descriptors
    size_t h_desc_cap = 0;
    // item column masks of every orientation of the staged items
    // (k_item_cols_all), per part: item it at d_icp[part] + icol_off[it],
    // icol_stride[it] entries per orientation, counts in d_icn[it * n + o]
    uint4* d_icp[2] = {nullptr, nullptr};
    size_t icp_cap[2] = {0, 0};
    long long* d_icoff = nullptr;    // icol_off and icol_stride on the device
    int* d_icstr = nullptr;
    int* d_icn = nullptr;
    size_t icmeta_cap = 0, icn_cap = 0;
    void* h_icmeta = nullptr;        // pinned staging of the two tables
    std::vector<long long> icol_off;
    std::vector<int> icol_stride;
    // the current item's precomputed columns for cand_filter (null: compute)
    const uint4* cur_icols = nullptr;
    long long cur_cstride = 0;
    const int* cur_ncol = nullptr;
    cudaStream_t st_copy = nullptr;  // uploads of the second part
    cudaEvent_t ev_copy = nullptr;

    // item staging
    int32_t* d_items = nullptr;
    size_t items_cap = 0;
    int4* d_vox = nullptr;
    size_t vox_cap = 0;
    int4* d_runs = nullptr;
    size_t runs_cap = 0;

    // per-column prefix sums along z of the distance field and the occupancy
    // (k_col_prefix), for the exact sums over an item's runs
    int32_t* d_pphi = nullptr;
    int32_t* d_pocc = nullptr;

    ~psb_tray() { release(); }

    void release_slots() {
        dfree(d_Ai, st); dfree(d_Bi, st); dfree(d_Pc, st); dfree(d_Pd, st); dfree(d_Dq, st); dfree(d_free, st); dfree(d_reach, st);
        dfree(d_cnt, st); dfree(d_off, st); dfree(d_rz2, st); dfree(d_rline, st); dfree(d_par, st); dfree(d_rflag, st); dfree(d_total, st); dfree(d_blk, st);
        dfree(d_cand, st); dfree(d_ncand, st); dfree(d_cscore, st); dfree(d_smin, st); dfree(d_pmin, st); dfree(d_okplane, st); dfree(d_candplane, st); dfree(d_bases, st); dfree(d_best, st);
        dfree(d_ccount, st); d_vcount = d_ncol = d_okcount = nullptr;
        dfree(d_act, st); d_nact = d_srch = d_nsrch = nullptr; dfree(d_icols, st); dfree(d_fsamp, st); dfree(d_fbound, st);
        dfree(d_bestkey, st); dfree(d_diag, st); dfree(d_errmax, st); dfree(d_od, st); dfree(d_rzs, st); dfree(d_mids, st); dfree(d_res, st);
        cap = 0;
    }
    void release() {
        if (dev >= 0) cudaSetDevice(dev);
        release_slots();
        dfree(d_tray, st); dfree(d_phi, st); dfree(d_Socc, st); dfree(d_Sphi, st); dfree(d_w1, st); dfree(d_w2, st); dfree(d_wocc, st); dfree(d_pen, st);
        dfree(d_ostat, st);
        dfree(d_rz, st); dfree(d_mid, st); dfree(d_stats, st); dfree(d_err, st); dfree(d_first, st); dfree(d_needff, st); dfree(d_items, st); dfree(d_vox, st);
        dfree(d_runs, st); dfree(d_pphi, st); dfree(d_pocc, st);
        dfree(d_ls, st); dfree(d_ps, st); dfree(d_rzd, st); dfree(d_midd, st); dfree(d_od_all, st); dfree(d_base_all, st); dfree(d_dec, st);
        dfree(d_tbits, st); dfree(d_work, st); dfree(d_clist, st);
        for (int p = 0; p < 2; ++p) {
            dfree(d_part[p], st);
            part_cap[p] = 0;
            dfree(d_icp[p], st);
            icp_cap[p] = 0;
        }
        dfree(d_icoff, st); dfree(d_icstr, st); dfree(d_icn, st);
        icmeta_cap = icn_cap = 0;
        clist_cap = 0;
        tq = 0;
        if (st_copy) {
            cudaStreamSynchronize(st_copy);
            cudaStreamDestroy(st_copy);
        }
        st_copy = nullptr;
        if (ev_copy) cudaEventDestroy(ev_copy);
        ev_copy = nullptr;
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        st = nullptr;
        for (int p = 0; p < 2; ++p) {
            if (h_part[p]) cudaFreeHost(h_part[p]);
            h_part[p] = nullptr;
            h_part_cap[p] = 0;
        }
        if (h_desc) cudaFreeHost(h_desc);
        h_desc = nullptr;
        h_desc_cap = 0;
        if (h_icmeta) cudaFreeHost(h_icmeta);
        h_icmeta = nullptr;
    }

    int init(int x, int y, int z) {
        TRY(ensure_device());
        CK(cudaGetDevice(&dev));
        TRY(set_smem_attrs());
        nx = x; ny = y; nz = z;
        V = (size_t)nx * ny * nz;
        TRY(make_grid3(nx, ny, nz, false, &g));
        nzw = (nz + 31) / 32;
        if (const char* e = getenv("PSB_SUBBATCH")) subbatch = atoi(e);
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        size_t S = (size_t)g.F[0] * g.F[1] * g.H;
        TRY(dalloc(&d_tray, V, st)); TRY(dalloc(&d_phi, V, st));
        TRY(dalloc(&d_Socc, S, st)); TRY(dalloc(&d_Sphi, S, st));
        TRY(dalloc(&d_w1, (size_t)nx * ny * g.H, st)); TRY(dalloc(&d_w2, (size_t)nx * g.F[1] * g.H, st));
        TRY(dalloc(&d_wocc, (size_t)nx * g.F[1] * g.H, st));
        TRY(dalloc(&d_pen, 3 * (size_t)nz, st)); TRY(dalloc(&d_rz, 4, st)); TRY(dalloc(&d_mid, 4, st)); TRY(dalloc(&d_stats, 4, st));
        TRY(dalloc(&d_work, 8, st));
        CK(cudaMemsetAsync(d_work, 0, sizeof(unsigned long long) * 8, st));
        TRY(dalloc(&d_err, 1, st)); TRY(dalloc(&d_first, 1, st)); TRY(dalloc(&d_needff, 1, st));
        TRY(dalloc(&d_ls, 1, st)); TRY(dalloc(&d_ps, 1, st)); TRY(dalloc(&d_rzd, 4, st)); TRY(dalloc(&d_midd, 8, st));
        TRY(dalloc(&d_pphi, (size_t)nx * ny * (nz + 1), st)); TRY(dalloc(&d_pocc, (size_t)nx * ny * (nz + 1), st));
        CK(cudaStreamSynchronize(st));  // stream-ordered allocations complete before plain copies touch them
        CK(cudaMemset(d_err, 0, sizeof(unsigned int)));
        // SCAN-mode penalty table with the host libm pow (packing.cpp:630-631)
        // BLOCK-mode factors (fft3.cu:172-173): qz = k/nz, qa = (P*qz)*qz, both
        // single IEEE operations, identical on host and device
        std::vector<double> pen(3 * (size_t)nz);
        for (int k = 0; k < nz; ++k) {
            pen[k] = kP * std::pow((k + 0.0) / (nz + 0.0), 3.0);
            volatile double qz = (double)k / (double)nz;
            volatile double qa = (kP * qz) * qz;
            pen[nz + k] = qa;
            pen[2 * nz + k] = qz;
        }
        CK(cudaMemcpy(d_pen, pen.data(), sizeof(double) * 3 * nz, cudaMemcpyHostToDevice));
        CK(cudaMemset(d_ls, 0, sizeof(LoopState)));
        CK(cudaMemset(d_ps, 0, sizeof(PhiStats)));
        const int* mean_p = (const int*)((const char*)d_ps + offsetof(PhiStats, mean));
        const int* placed_now = (const int*)((const char*)d_ls + offsetof(LoopState, placed_now));
        const int* need_phi = (const int*)((const char*)d_ls + offsetof(LoopState, need_phi));
        RzDesc rz[4] = {RzDesc{SRC_GRID_OCC, d_tray, nx, ny, nz, 0, -1, d_w1, nullptr, nullptr},
                        RzDesc{SRC_GRID_SUB, d_phi, nx, ny, nz, 0, -1, d_w1, nullptr, mean_p},
                        RzDesc{SRC_GRID_OCC, d_tray, nx, ny, nz, 0, -1, d_w1, placed_now, nullptr},
                        RzDesc{SRC_GRID_SUB, d_phi, nx, ny, nz, 0, -1, d_w1, need_phi, mean_p}};
        MidDesc md[8];
        forward_mids(g, d_w1, d_w2, d_Socc, nullptr, md + 0);
        forward_mids(g, d_w1, d_w2, d_Sphi, nullptr, md + 2);
        forward_mids(g, d_w1, d_w2, d_Socc, placed_now, md + 4);
        forward_mids(g, d_w1, d_w2, d_Sphi, need_phi, md + 6);
        CK(cudaMemcpy(d_rzd, rz, sizeof(rz), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_midd, md, sizeof(md), cudaMemcpyHostToDevice));
        return PSB_OK;
    }

    int ensure_slots(int n) {
        if (n <= cap) return PSB_OK;
        release_slots();
        int c = std::max(n, 1);
        sAi = (long long)nx * ny * g.H;
        sBi = (long long)nx * g.F[1] * g.H;
        sP = (long long)nx * g.F[1] * g.H;
        sD = (long long)V;
        sBits = (long long)nx * ny * nzw;
        sLine = (long long)nx * ny;
        sRun = (long long)nx * ny * ((nz + 1) / 2);
        TRY(dalloc(&d_Ai, sAi * c, st)); TRY(dalloc(&d_Bi, sBi * c, st));
        TRY(dalloc(&d_Pc, sP * c, st)); TRY(dalloc(&d_Pd, sP * c, st));
        TRY(dalloc(&d_Dq, sD * c, st));
        TRY(dalloc(&d_free, sBits * c, st)); TRY(dalloc(&d_reach, sBits * c, st));
        TRY(dalloc(&d_cnt, sLine * c, st)); TRY(dalloc(&d_off, sLine * c, st));
        TRY(dalloc(&d_rz2, sRun * c, st)); TRY(dalloc(&d_rline, sRun * c, st)); TRY(dalloc(&d_par, sRun * c, st));
        TRY(dalloc(&d_rflag, sRun * c, st)); TRY(dalloc(&d_total, c, st));
        TRY(dalloc(&d_blk, (size_t)((nx * ny + 255) / 256) * c, st));
        TRY(dalloc(&d_cand, (size_t)kCandCap * c, st)); TRY(dalloc(&d_ncand, c, st));
        TRY(dalloc(&d_cscore, (size_t)kCandCap * c, st));
        TRY(dalloc(&d_smin, c, st)); TRY(dalloc(&d_pmin, (size_t)nx * c, st)); TRY(dalloc(&d_okplane, (size_t)nx * c, st));
        TRY(dalloc(&d_candplane, (size_t)nx * c, st));
        TRY(dalloc(&d_act, 2 * (size_t)c + 2, st));
        d_nact = d_act + c;
        d_srch = d_act + c + 1;
        d_nsrch = d_srch + c;
        TRY(dalloc(&d_ccount, 4 * (size_t)c, st));
        d_vcount = d_ccount + c;
        d_ncol = d_ccount + 2 * c;
        d_okcount = d_ccount + 3 * c;
        TRY(dalloc(&d_icols, (size_t)nx * ny * c, st));
        TRY(dalloc(&d_fsamp, (size_t)PSB_FSAMP * c, st));
        TRY(dalloc(&d_fbound, (size_t)PSB_FBOUND * c, st));
        TRY(dalloc(&d_bases, 6, st)); TRY(dalloc(&d_best, c, st)); TRY(dalloc(&d_bestkey, c, st));
        TRY(dalloc(&d_diag, c, st)); TRY(dalloc(&d_errmax, c, st)); TRY(dalloc(&d_od, c, st)); TRY(dalloc(&d_rzs, c, st)); TRY(dalloc(&d_mids, c, st));
        TRY(dalloc(&d_res, c, st));
        // item transform descriptors of each slot (orientation-relative)
        std::vector<RzDesc> rz(c);
        std::vector<MidDesc> md(c);
        for (int o = 0; o < c; ++o) {
            rz[o] = RzDesc{SRC_ITEM, nullptr, 0, 0, 0, 0, o, d_Ai + (size_t)o * sAi, nullptr, nullptr};
            md[o] = MidDesc{d_Ai + (size_t)o * sAi, d_Bi + (size_t)o * sBi, 0, g.H, 0, g.F[1], 0,
                            (long long)g.F[1] * g.H, g.H, g.H, o, 0, nullptr};
        }
        CK(cudaStreamSynchronize(st));  // stream-ordered allocations complete
        CK(cudaMemcpy(d_rzs, rz.data(), sizeof(RzDesc) * c, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_mids, md.data(), sizeof(MidDesc) * c, cudaMemcpyHostToDevice));
        cap = c;
        return PSB_OK;
    }

    int ensure_runs(size_t n) {
        if (n > runs_cap) {
            dfree(d_runs, st);
            runs_cap = std::max(n, (size_t)1 << 14);
            TRY(dalloc(&d_runs, runs_cap, st));
        }
        return PSB_OK;
    }

    // prefix tables of the distance field (gated when gate is set) and of
    // the occupancy
    int prefix_phi(const int* gate) {
        const int ncols = nx * ny;
        pdl(k_col_prefix<0>, (ncols + 7) / 8, 256, 0, st)(d_phi, d_pphi, ncols, nz, gate);
        CKL();
        return PSB_OK;
    }
    int prefix_occ() {
        const int ncols = nx * ny;
        pdl(k_col_prefix<1>, (ncols + 7) / 8, 256, 0, st)(d_tray, d_pocc, ncols, nz, nullptr);
        CKL();
        return PSB_OK;
    }

    int ensure_staging(size_t n_items, size_t n_vox) {
        if (n_items > items_cap) {
            dfree(d_items, st);
            items_cap = std::max(n_items, (size_t)1 << 16);
            TRY(dalloc(&d_items, items_cap, st));
        }
        if (n_vox > vox_cap) {
            dfree(d_vox, st);
            vox_cap = std::max(n_vox, (size_t)1 << 14);
            TRY(dalloc(&d_vox, vox_cap, st));
        }
        return PSB_OK;
    }

    // spectrum of the occupancy (phi = false) or of phi - mean (phi = true);
    // gated: only when *gate != 0 at run time.  Specialised kernels when the
    // FFT lengths have plans, the generic descriptor path otherwise.
    //
    // The occupancy's z,y slab transforms are kept (d_wocc): after a
    // placement (slabs = the placed item's x extent at most, x0p = its x
    // origin on the device) only the slabs under the item are transformed
    // again, then the x pass runs over every column.
    int tray_forward(bool phi, const int* gate, int slabs = 0, const int* x0p = nullptr) {
        FwdPlaneFn ff = g_fast_fft ? fwd_plane_for(g.F[1], g.F[2]) : nullptr;
        XfwdFn xf = g_fast_fft ? xfwd_for(g.F[0]) : nullptr;
        const size_t smf = fwd_plane_smem(g.F[1], g.F[2], ny) + 64;
        if (ff && xf && smf <= (size_t)g_smem_optin && xfwd_smem(g.F[0]) + 64 <= (size_t)g_smem_optin) {
            const int* mean_p = (const int*)((const char*)d_ps + offsetof(PhiStats, mean));
            float2* w = phi ? d_w2 : d_wocc;
            const bool part = !phi && x0p && slabs > 0 && slabs < nx;
            FwdSrc src{phi ? (int)SRC_GRID_SUB : (int)SRC_GRID_OCC, phi ? d_phi : d_tray, nx, ny, nz, mean_p, gate,
                       w, 0, part ? x0p : nullptr};
            {
                PROF("k_fwd_plane", st);
                pdl(ff, dim3(part ? slabs : nx, 1), 256, smf, st)(src, nullptr, g.p[1].tw, g.p[2].tw);
            }
            CKL();
            {
                PROF("k_xfwd", st);
                const int ncols = g.F[1] * g.H;
                pdl(xf, (ncols + PSB_XCOLS - 1) / PSB_XCOLS, 256, xfwd_smem(g.F[0]), st)(
                    w, phi ? d_Sphi : d_Socc, nx, ncols, gate, g.p[0].tw);
            }
            CKL();
            return PSB_OK;
        }
        const int idx = (phi ? 1 : 0) + (gate ? 2 : 0);
        return forward3_dev(g, d_rzd + idx, d_midd + 2 * idx, st);
    }

    // occupancy spectrum from the device tray
    int rebuild_occ() { return tray_forward(false, nullptr); }
    // ... only when the current item of the asynchronous loop was placed,
    // and then only the slabs under it (at most `slabs` of them from its x
    // origin ls->px)
    int rebuild_occ_gated(int slabs) {
        return tray_forward(false, (const int*)((const char*)d_ls + offsetof(LoopState, placed_now)), slabs,
                            (const int*)((const char*)d_ls + offsetof(LoopState, px)));
    }

    // mean, norm and max deviation of the distance field, on the device
    int phi_stats(const int* gate) {
        unsigned long long* raw = (unsigned long long*)((char*)d_ps + offsetof(PhiStats, raw));
        const int* mean_p = (const int*)((const char*)d_ps + offsetof(PhiStats, mean));
        CK(cudaMemsetAsync(raw, 0, sizeof(unsigned long long) * 4, st));
        {
            PROF("k_stats", st);
            pdl(k_stats_g, grid1d(V), 256, 0, st)(d_phi, V, nullptr, raw, gate);
        }
        CKL();
        pdl(k_phi_mean, 1, 1, 0, st)(d_ps, (unsigned long long)V, gate);
        CKL();
        {
            PROF("k_stats", st);
            pdl(k_stats_g, grid1d(V), 256, 0, st)(d_phi, V, mean_p, raw, gate);
        }
        CKL();
        pdl(k_phi_norm, 1, 1, 0, st)(d_ps, gate);
        CKL();
        return PSB_OK;
    }

    // distance spectrum (mean-subtracted) from the device distance field
    int rebuild_phi_spectrum() {
        TRY(phi_stats(nullptr));
        TRY(tray_forward(true, nullptr));
        PhiStats h;
        CK(cudaMemcpyAsync(&h, d_ps, sizeof(h), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        phi_mean = h.mean;
        phi_norm = h.norm;
        phi_maxabs = h.maxabs;
        return PSB_OK;
    }

    // distance field, its statistics and spectrum, only when the current item
    // of the asynchronous loop wrote voxels equal to 1
    int rebuild_phi_gated() {
        const int* need_phi = (const int*)((const char*)d_ls + offsetof(LoopState, need_phi));
        TRY(distance_on_device(d_tray, d_phi, nx, ny, nz, st, need_phi));
        TRY(prefix_phi(need_phi));
        TRY(phi_stats(need_phi));
        return tray_forward(true, need_phi);
    }

    int set(const int32_t* tray, const int32_t* phi) {
        CK(cudaSetDevice(dev));
        // negative values and occupied cells, one pass over the host cores
        std::atomic<int> neg(0);
        std::atomic<size_t> nocc(0);
        parallel_chunks(V, (size_t)1 << 20, [&](size_t b, size_t e) {
            size_t c = 0;
            int ng = 0;
            for (size_t i = b; i < e; ++i) {
                c += tray[i] != 0;
                ng |= tray[i] < 0;
            }
            nocc += c;
            if (ng) neg = 1;
        });
        if (neg) return fail(PSB_ERR_ARG, "tray holds negative values; item ids must be >= 0");
        occ = nocc;
        CK(cudaMemcpyAsync(d_tray, tray, sizeof(int32_t) * V, cudaMemcpyHostToDevice, st));
        if (phi) {
            CK(cudaMemcpyAsync(d_phi, phi, sizeof(int32_t) * V, cudaMemcpyHostToDevice, st));
        } else {
            TRY(distance_on_device(d_tray, d_phi, nx, ny, nz, st));
        }
        TRY(prefix_occ());
        TRY(prefix_phi(nullptr));
        TRY(rebuild_occ());
        TRY(rebuild_phi_spectrum());
        CK(cudaStreamSynchronize(st));
        ready = true;
        return PSB_OK;
    }

    // Fill an OrientDesc from an item's analysis and a signed permutation.
    void describe(const ItemInfo& info, const int* src_axis, const int* flip, const int32_t* d_item,
                  const int4* d_vx, const int4* const* d_rn, OrientDesc* od) const {
        int n[3] = {nx, ny, nz};
        for (int a = 0; a < 3; ++a) {
            od->src_axis[a] = src_axis[a];
            od->flip[a] = flip[a];
            od->b[a] = info.dims[a];
            od->e[a] = info.dims[src_axis[a]];
        }
        bool empty = info.hi[0] < 0;
        od->skip = 0;
        for (int a = 0; a < 3; ++a) {
            int s = src_axis[a];
            od->hi[a] = empty ? -1 : (flip[a] ? od->e[a] - 1 - info.lo[s] : info.hi[s]);
            if (od->e[a] > n[a]) od->skip = 1;
            // t + hi <= n - 1 ; an empty item (reference hi = -INF) leaves every t valid
            od->valid[a] = empty ? n[a] : std::max(0, n[a] - od->hi[a]);
        }
        od->sumI = info.sum;
        od->base = (double)phi_mean * (double)info.sum;
        const long long sabs = info.sabs;  // |D'| <= sum|I| * max|phi - m|
        double maxD = (double)sabs * (double)phi_maxabs;
        const double eps = 1.1920928955078125e-07;
        od->delta = 2.0 * eps * std::sqrt(info.sumsq) * phi_norm + 0.5 * ulp32(maxD) + 1e-3;
        od->exact = (od->delta >= 0.4 || maxD >= 8388608.0) ? 1 : 0;
        od->item = d_item;
        od->vox = d_vx;
        od->nvox = (int)info.nvox;
        od->perm = -1;
        od->sumsq = info.sumsq;
        od->sabs = sabs;
        od->samp = nullptr;
        od->nsamp = 0;
        od->direct = 0;
        od->runs = d_rn[src_axis[2]];
        od->nruns = (int)info.runs[src_axis[2]].size();
    }

    // Free bits of the tray for the candidate filter, all columns.
    int tray_bits() {
        if (!d_tbits) {
            tq = (nzw + 3) / 4;
            TRY(dalloc(&d_tbits, (size_t)nx * ny * tq, st));
        }
        {
            PROF("k_tray_bits", st);
            pdl(k_tray_bits, (unsigned)(((size_t)nx * ny + 7) / 8), 256, 0, st)(d_tray, nx, ny, nz, tq, d_tbits);
        }
        CKL();
        return PSB_OK;
    }

    // whether search_async takes the split flow (search_split) with the
    // specialised x pass for this tray: only its kernels know direct
    // orientations
    bool split_flow() const {
        if (!g_fast_fft || g_plane_variant != 3) return false;
        if (!xpass2_for(g.F[0]) || xpass2_smem(g.F[0]) + 64 > (size_t)g_smem_optin) return false;
        if (!plane3_for(g.F[1], g.F[2], 0) || !plane3_for(g.F[1], g.F[2], 1)) return false;
        return plane3_smem(g.F[1], g.F[2], ny) + 64 <= (size_t)g_smem_optin;
    }

    // Candidate filter of one item's orientations (psb_filter.cuh): candidate
    // words into the free-bit slots, plane flags, orientations without a
    // candidate skipped; orientations with few candidates verified directly.
    // The next search refines the other candidates.
    int cand_filter(OrientDesc* d_odb, const std::vector<OrientDesc>& ods, bool interlock) {
        int xmax = 0, emax = 0;
        for (auto& o : ods)
            if (!o.skip && o.nsamp > 0) {
                xmax = std::max(xmax, o.valid[0]);
                emax = std::max(emax, o.e[0]);
            }
        const int n = (int)ods.size();
        const int dmax = split_flow() ? g_direct_max : 0;
        // candidate lists for the direct checks: dmax entries per orientation
        const int ccap = std::max(dmax, 1);
        if ((size_t)ccap * cap > clist_cap) {
            dfree(d_clist, st);
            clist_cap = (size_t)ccap * cap;
            TRY(dalloc(&d_clist, clist_cap, st));
        }
        if (xmax > 0) {
            const dim3 grid(xmax, n);
            // (k_cand_prep zeroes the counters d_ccount, d_vcount, d_ncol)
            const size_t smw = sizeof(uint4) * (size_t)emax * ny * tq + (size_t)n;
            if (g_filter_plane && smw <= (size_t)g_smem_optin) {
                PROF("k_cand_filter", st);
                if (tq == 1) {
                    pdl(k_cand_prep<1>, n, 32, 0, st)(d_odb, d_fsamp, d_fbound, d_ccount, (int)cap, prep_ps);
                    pdl(k_cand_filter_plane<1>, dim3(xmax, g_filter_groups), PSB_FILT_PLANE_THREADS, smw, st)(
                        d_odb, n, d_tbits, nx, ny, nzw, emax, d_free, sBits, d_candplane, (long long)nx, d_ccount,
                        d_fsamp, d_fbound, g_filter_cut, d_clist, ccap, nz);
                } else {
                    pdl(k_cand_prep<2>, n, 32, 0, st)(d_odb, d_fsamp, d_fbound, d_ccount, (int)cap, prep_ps);
                    pdl(k_cand_filter_plane<2>, dim3(xmax, g_filter_groups), PSB_FILT_PLANE_THREADS, smw, st)(
                        d_odb, n, d_tbits, nx, ny, nzw, emax, d_free, sBits, d_candplane, (long long)nx, d_ccount,
                        d_fsamp, d_fbound, g_filter_cut, d_clist, ccap, nz);
                }
            } else {
                PROF("k_cand_filter", st);
                if (tq == 1) {
                    pdl(k_cand_prep<1>, n, 32, 0, st)(d_odb, d_fsamp, d_fbound, d_ccount, (int)cap, prep_ps);
                    // the variant (sample batch, CTAs per SM bound) is a tuning switch
                    auto kf = g_filter_variant == 1 ? k_cand_filter<1, 4, 12>
                            : g_filter_variant == 2 ? k_cand_filter<1, 8, 1>
                            : g_filter_variant == 3 ? k_cand_filter<1, 16, 1> : k_cand_filter<1>;
                    pdl(kf, grid, PSB_FILT_THREADS, 0, st)(d_odb, d_tbits, ny, nzw, d_free, sBits, d_candplane,
                                                          (long long)nx, d_ccount, d_fsamp, d_fbound, g_filter_cut,
                                                          d_clist, ccap, nz);
                } else {
                    pdl(k_cand_prep<2>, n, 32, 0, st)(d_odb, d_fsamp, d_fbound, d_ccount, (int)cap, prep_ps);
                    pdl(k_cand_filter<2>, grid, PSB_FILT_THREADS, 0, st)(d_odb, d_tbits, ny, nzw, d_free, sBits,
                                                                        d_candplane, (long long)nx, d_ccount,
                                                                        d_fsamp, d_fbound, g_filter_cut, d_clist,
                                                                        ccap, nz);
                }
            }
            CKL();
            // with direct decisions the okplane flags of the free cells
            // (non-interlocking mode) are set by the verification for direct
            // orientations, so k_cand_apply clears them first
            pdl(k_cand_apply, (n + 127) / 128, 128, 0, st)(d_odb, n, d_ccount, 0, dmax, dmax > 0 ? d_okplane : nullptr,
                                                           (long long)nx, nx);
            CKL();
            if (dmax > 0) {
                {
                    PROF("k_cand_verify", st);
                    const uint4* cols = cur_icols;
                    long long cstride = cur_cstride;
                    const int* ncol = cur_ncol;
                    if (!cols) {
                        pdl(k_item_cols, dim3(emax, n), 64, 0, st)(d_odb, d_icols, (long long)nx * ny, d_ncol);
                        CKL();
                        cols = d_icols;
                        cstride = (long long)nx * ny;
                        ncol = d_ncol;
                    }
                    pdl(k_cand_verify_list, 148 * 4, 256, sizeof(int) * (n + 1), st)(
                        d_odb, n, d_tbits, ny, nz, nzw, tq, d_free, sBits, d_clist, ccap, d_ccount, cols,
                        cstride, ncol, d_vcount, d_okplane, (long long)nx, interlock ? 0 : 1);
                }
                CKL();
                // stage 1 of k_cand_apply: done by the search's k_active_list
                // when it launches one, else by flush_apply
                pending_apply = true;
                apply_dmax = dmax;
            }
        }
        if (xmax <= 0 && prep_ps) {
            // no filter kernels ran: the error bounds the caller left to k_cand_prep
            pdl(k_prep, (n + 63) / 64, 64, 0, st)(d_odb, n, prep_ps);
            CKL();
        }
        cand_active = true;
        direct_active = dmax > 0 && xmax > 0;   // the okplane flags were cleared above
        return PSB_OK;
    }

    // the candidate filter's verification outcome (stage 1 of k_cand_apply),
    // when no k_active_list has taken it over
    int flush_apply(OrientDesc* d_odb, int n) {
        if (!pending_apply) return PSB_OK;
        pending_apply = false;
        pdl(k_cand_apply, (n + 127) / 128, 128, 0, st)(d_odb, n, d_vcount, 1, apply_dmax, nullptr, 0LL, 0);
        CKL();
        return PSB_OK;
    }

    ScoreParams score_params(int mode) const {
        ScoreParams sp;
        sp.nx = nx; sp.ny = ny; sp.nz = nz;
        sp.mode = mode;
        sp.pen = d_pen;
        sp.qa = d_pen + nz;
        sp.qz = d_pen + 2 * nz;
        sp.scale = (float)(1.0 / ((double)g.F[0] * g.F[1] * g.F[2]));
        sp.nzw = nzw;
        return sp;
    }

    // Reset of the search state before a search's kernels (k_search_reset);
    // split: the split flow, whose plane flags are cleared here unless the
    // candidate filter has done so for its direct orientations
    int search_reset(int n, bool split) {
        SearchReset a{d_smin, d_best, d_bestkey, d_diag, d_errmax, d_ncand, d_total, d_err,
                      split && !direct_active ? d_okplane : nullptr, (long long)nx * n, n};
        pdl(k_search_reset, 4, 256, 0, st)(a);
        CKL();
        return PSB_OK;
    }

    // Flood fill (Algorithm 3) of every orientation's free bits into its
    // reach bits.  okplane, when set, receives the planes that hold a
    // reachable cell; gate, when set, makes every launch conditional.
    int flood_fill(const OrientDesc* d_odb, int n, const ScoreParams& sp, const int* gate, unsigned char* okplane,
                   int* okcount = nullptr) {
        const bool lists = act_ready && g_list_select;
        FloodBufs fb{d_free, d_reach, sBits, d_cnt, d_off,   sLine, d_rz2,    d_rline,
                     d_par,  d_rflag, sRun,  d_total, d_err, gate,  okplane, (long long)nx, g_uf_limit, okcount,
                     lists ? d_srch : nullptr, lists ? d_nsrch : nullptr};
        const int rows = lists ? std::min(n, g_active_grid) : n;
        const int lines = nx * ny;
        const int nblk = (lines + 255) / 256;
        const dim3 gl(nblk, rows);
        // (the run counters d_total were zeroed by search_reset)
        {
            PROF("k_ff_runs", st);
            pdl(k_ff_runs, gl, 256, 0, st)(d_odb, fb, sp);
        }
        CKL();
        {
            PROF("k_ff_union", st);
            pdl(k_ff_union, gl, 256, 0, st)(d_odb, fb, sp);
        }
        CKL();
        {
            PROF("k_ff_seed", st);
            pdl(k_ff_seed, dim3(296, rows), 256, 0, st)(d_odb, fb);
        }
        CKL();
        {
            PROF("k_ff_reach", st);
            pdl(k_ff_reach, gl, 256, 0, st)(d_odb, fb, sp);
        }
        CKL();
        return PSB_OK;
    }

    // The default search for the specialised FFT lengths: collision plane
    // pass (free bits) -> flood fill (interlocking mode) -> proximity plane
    // pass only on the planes that hold an ok cell (free, or reachable) ->
    // selection over the ok cells.  An item that fits nowhere costs no
    // proximity transform, and every orientation's own result is exact.
    int search_split(const OrientDesc* d_odb, int n, const ScoreParams& sp, bool interlock, XpassFn xf, PlaneFn p0,
                     PlaneFn p1, size_t smem, ResultDev* d_out, bool spec) {
        SearchBufs sb{d_Bi, d_Pc, d_Pd, sBi, sP, d_work, act_ready ? d_act : nullptr, act_ready ? d_nact : nullptr};
        const int rows = act_ready ? std::min(n, g_active_grid) : n;
        // (the plane flags were cleared by search_reset, or, with direct
        // orientations, by the candidate filter, which set those of its
        // verified planes already)
        const int ncols = g.F[1] * g.H;
        XpassFn xf1 = xf ? xpass2_for(g.F[0], 1, spec) : nullptr, xf2 = xf ? xpass2_for(g.F[0], 2, spec) : nullptr;
        const BaseMap bm{g.F[1], g.H, g.F[2], g.p[1].tw, g.p[2].tw};
        if (xf) {
            PROF("k_xpass_coll", st);
            // with the filter's plane flags, only rows of planes holding a
            // candidate are stored (the plane pass skips the others)
            pdl(xf1, dim3((ncols + PSB_XCOLS - 1) / PSB_XCOLS, rows), 256, xpass2_smem(g.F[0]), st)(
                d_odb, sb, d_Socc, d_Sphi, ncols, g.p[0].tw, cand_active ? d_candplane : nullptr, (long long)nx, bm);
        } else {
            PROF("k_xpass_coll", st);
            const size_t smx = sizeof(float2) * (g.F[0] + 4 * PSB_TILE * g.F[0]);
            pdl(k_xpass, dim3((g.H + PSB_TILE - 1) / PSB_TILE, g.F[1], n), PSB_THREADS, smx, st)(
                d_odb, sb, d_Socc, d_Sphi, g.F[1], g.H, g.p[0].p, g.p[0].tw);
        }
        CKL();
        const uint32_t* ok = interlock ? d_reach : d_free;
        // orientations left with few ok cells skip the proximity transforms
        // (k_late_direct): count the ok cells of every orientation
        const bool late = g_late_max > 0;
        if (late) CK(cudaMemsetAsync(d_okcount, 0, sizeof(int) * n, st));
        PlaneBufs pb{d_free, d_Dq,      d_smin,         d_diag, sBits, sD, d_pmin, (long long)nx, ok, d_okplane,
                     interlock ? 0 : 1, cand_active ? d_candplane : nullptr, late ? d_okcount : nullptr};
        {
            PROF("k_plane_coll", st);
            pdl(p0, dim3(nx, rows), PSB_PLANE3_THREADS, smem, st)(d_odb, sb, pb, sp, g.p[1].tw, g.p[2].tw);
        }
        CKL();
        if (interlock) TRY(flood_fill(d_odb, n, sp, nullptr, d_okplane, late ? d_okcount : nullptr));
        if (late) {
            pdl(k_late_direct, (n + 127) / 128, 128, 0, st)(const_cast<OrientDesc*>(d_odb), n, d_okcount, g_late_max);
            CKL();
            late_active = true;
        }
        if (xf) {
            PROF("k_xpass_prox", st);
            pdl(xf2, dim3((ncols + PSB_XCOLS - 1) / PSB_XCOLS, rows), 256, xpass2_smem(g.F[0]), st)(
                d_odb, sb, d_Socc, d_Sphi, ncols, g.p[0].tw, d_okplane, (long long)nx, bm);
        }
        CKL();
        {
            PROF("k_plane_prox", st);
            pdl(p1, dim3(nx, rows), PSB_PLANE3_THREADS, smem, st)(d_odb, sb, pb, sp, g.p[1].tw, g.p[2].tw);
        }
        CKL();
        return select_over(d_odb, n, sp, ok, nullptr, d_out, d_okplane, decide.ls != nullptr);
    }

    // Selection over the ok cells from the plane minima: candidates in the
    // window of each orientation's minimum, exact re-score, tie rule, result.
    // okplane (may be null): the planes that hold an ok cell (the split flow
    // keeps them for every orientation)
    int select_over(const OrientDesc* d_odb, int n, const ScoreParams& sp, const uint32_t* ok, const int* gate,
                    ResultDev* d_out, const unsigned char* okplane = nullptr, bool fuse = false) {
        const bool lists = act_ready && g_list_select;
        SelectBufs sel{ok,        sBits,  d_Dq,     sD,       d_smin, d_cand,        d_ncand, d_cscore, d_best,
                       d_bestkey, d_diag, d_errmax, kCandCap, d_pmin, (long long)nx, gate, okplane,
                       lists ? d_srch : nullptr, lists ? d_nsrch : nullptr};
        const int rows = lists ? std::min(n, g_active_grid) : n;
        {
            PROF("k_collect", st);
            pdl(k_collect_plane, dim3(nx, rows), 256, 0, st)(d_odb, sel, sp);
        }
        CKL();
        {
            PROF("k_rescore", st);
            pdl(k_rescore, dim3(148, rows), 256, 0, st)(d_odb, sel, sp, d_pocc, d_pphi);
        }
        CKL();
        if (direct_active || late_active) {
            PROF("k_direct_score", st);
            pdl(k_direct_score, dim3(64, rows), 256, 0, st)(d_odb, sel, sp, d_pphi);
            CKL();
        }
        {
            PROF("k_tiebreak", st);
            pdl(k_tiebreak, dim3(64, rows), 256, 0, st)(d_odb, sel, sp);
        }
        CKL();
        if (fuse && !gate) {
            // the packing loop's decision in the same launch
            PROF("k_finalize", st);
            pdl(k_finalize_decide, 1, 128, 0, st)(d_odb, sel, sp, d_out, n, decide);
            fused = true;
        } else {
            PROF("k_finalize", st);
            pdl(k_finalize, (n + 127) / 128, 128, 0, st)(d_odb, sel, sp, d_out, n);
        }
        CKL();
        return PSB_OK;
    }

    // Queue the search of the n orientations whose descriptors are at d_odb
    // (device item data already there); each orientation's result goes to
    // d_out[o].  ods is the host copy (dims for the launch shapes).  No host
    // copy or synchronisation happens here.
    //
    // Interlocking-free searches run lazily unless every orientation's own
    // result is wanted (lazy = false): the selection first runs over the free
    // cells; when the overall winner has a straight free run to a seed face it
    // is reachable, hence also the winner over the reachable cells, and the
    // flood fill is skipped (k_line_check).  Otherwise the flood fill and a
    // second selection over the reachable cells run, gated on the device flag
    // d_needff, so the host never waits.
    //
    // With bases (d_bases / hbases: the item's 6 axis permutations, each
    // orientation's OrientDesc::perm set), the split flow transforms only the
    // bases and the x passes read their slabs (k_xpass2 SHARED).
    int search_async(const OrientDesc* d_odb, const std::vector<OrientDesc>& ods, int mode, bool interlock,
                     ResultDev* d_out, bool lazy = true, const OrientDesc* d_bases_in = nullptr,
                     const std::vector<OrientDesc>* hbases = nullptr) {
        const int n = (int)ods.size();
        act_ready = false;
        // the caller reserves the slots (ensure_slots) before taking slot
        // pointers such as d_out: growing them here would free those
        if (cap < std::max(n, 6)) return fail(PSB_ERR_STATE, "search slots not reserved (%d < %d)", cap, std::max(n, 6));
        XpassFn xf = g_fast_fft ? xpass2_for(g.F[0]) : nullptr;
        if (xf && xpass2_smem(g.F[0]) + 64 > (size_t)g_smem_optin) xf = nullptr;
        PlaneFn p0 = nullptr, p1 = nullptr;
        size_t sm3 = 0;
        if (g_fast_fft && g_plane_variant == 3) {
            p0 = plane3_for(g.F[1], g.F[2], 0);
            p1 = plane3_for(g.F[1], g.F[2], 1);
            if (p0 && p1) sm3 = plane3_smem(g.F[1], g.F[2], ny) + 64;
            if (!p0 || !p1 || sm3 > (size_t)g_smem_optin) p0 = p1 = nullptr;
        }
        FwdPlaneFn ffb = g_fast_fft ? fwd_plane_for(g.F[1], g.F[2]) : nullptr;
        const bool spec = g_share_flips && d_bases_in && hbases && p0 && xf && ffb;
        if (spec) {
            TRY(flush_apply(const_cast<OrientDesc*>(d_odb), n));
            // the bases' z,y forward into slab slots 0..5; the x passes read them
            int bx = 1, by = 1;
            for (auto& b : *hbases)
                if (!b.skip) { bx = std::max(bx, b.e[0]); by = std::max(by, b.e[1]); }
            const size_t smf = fwd_plane_smem(g.F[1], g.F[2], by) + 64;
            if (smf <= (size_t)g_smem_optin) {
                FwdSrc src{SRC_ITEM, nullptr, 0, 0, 0, nullptr, nullptr, d_Bi, sBi};
                {
                    PROF("k_fwd_plane", st);
                    pdl(ffb, dim3(bx, 6), 256, smf, st)(src, d_bases_in, g.p[1].tw, g.p[2].tw);
                }
                CKL();
                TRY(search_reset(n, true));
                return search_split(d_odb, n, score_params(mode), interlock, xf, p0, p1, sm3, d_out, true);
            }
        }
        int exmax = 1, maxpairs = 1;
        for (auto& o : ods)
            if (!o.skip) {
                exmax = std::max(exmax, o.e[0]);
                maxpairs = std::max(maxpairs, (o.e[0] * o.e[1] + 1) / 2);
            }
        int eymax = 1;
        for (auto& o : ods)
            if (!o.skip) eymax = std::max(eymax, o.e[1]);
        FwdPlaneFn ff = g_fast_fft ? fwd_plane_for(g.F[1], g.F[2]) : nullptr;
        const size_t smf = fwd_plane_smem(g.F[1], g.F[2], eymax) + 64;
        act_ready = false;
        if (!(ff && smf <= (size_t)g_smem_optin && g_active_grid > 0))
            TRY(flush_apply(const_cast<OrientDesc*>(d_odb), n));
        if (ff && smf <= (size_t)g_smem_optin) {
            // the transforms take the active orientations from a list: a few
            // CTA rows loop over them instead of a row per orientation
            const int rows = g_active_grid > 0 ? std::min(n, g_active_grid) : n;
            if (g_active_grid > 0) {
                pdl(k_active_list, 1, 32, 0, st)(const_cast<OrientDesc*>(d_odb), n, d_act, d_nact, d_srch, d_nsrch,
                                                 pending_apply ? d_vcount : nullptr);
                CKL();
                pending_apply = false;
                act_ready = true;
            }
            FwdSrc src{SRC_ITEM, nullptr, 0, 0, 0, nullptr, nullptr, d_Bi, sBi, nullptr,
                       act_ready ? d_act : nullptr, act_ready ? d_nact : nullptr};
            PROF("k_fwd_plane", st);
            pdl(ff, dim3(exmax, rows), 256, smf, st)(src, d_odb, g.p[1].tw, g.p[2].tw);
        } else {
            {
                PROF("k_rfft_z", st);
                pdl(k_rfft_z, dim3((maxpairs + PSB_PAIRS - 1) / PSB_PAIRS, n), PSB_THREADS, smem_rz(g.F[2]), st)(
                    d_rzs, d_odb, g.p[2].p, g.p[2].tw);
            }
            CKL();
            {
                PROF("k_fft_mid_fwd", st);
                pdl(k_fft_mid<-1>, dim3((g.H + PSB_TILE - 1) / PSB_TILE, exmax, n), PSB_THREADS, smem_mid(g.F[1]), st)(
                    d_mids, d_odb, g.p[1].p, g.p[1].tw);
            }
        }
        CKL();
        TRY(search_reset(n, p0 != nullptr));
        ScoreParams sp = score_params(mode);
        if (p0) return search_split(d_odb, n, sp, interlock, xf, p0, p1, sm3, d_out, false);
        PlaneFn pf = nullptr;
        size_t sm2 = 0;
        const int pthreads = PSB_PLANE_THREADS;
        if (g_fast_fft) {
            pf = plane2_for(g.F[1], g.F[2]);
            sm2 = plane2_smem(g.F[1], g.F[2], ny, nzw) + 64;
            if (pf && sm2 > (size_t)g_smem_optin) pf = nullptr;
        }
        const int wsz = std::max(PSB_TILE * g.F[1], PSB_PAIRS * g.F[2]);
        const size_t smp = sizeof(float2) * ((size_t)g.F[1] + g.F[2] + (size_t)ny * g.H + 2 * (size_t)wsz) +
                           sizeof(uint32_t) * (size_t)ny * nzw;
        if (!pf && smp + 64 > (size_t)g_smem_optin)
            return fail(PSB_ERR_ARG, "tray too large for the plane kernel (%zu B smem)", smp);
        // x pass then plane pass per sub-batch of orientations, so a
        // sub-batch's products can still be in L2 when the plane pass reads them
        const int sub = subbatch > 0 ? std::min(subbatch, n) : n;
        for (int o0 = 0; o0 < n; o0 += sub) {
            const int m = std::min(sub, n - o0);
            SearchBufs sbo{d_Bi + (size_t)o0 * sBi, d_Pc + (size_t)o0 * sP, d_Pd + (size_t)o0 * sP, sBi, sP};
            PlaneBufs pbo{d_free + (size_t)o0 * sBits, d_Dq + (size_t)o0 * sD, d_smin + o0, d_diag + o0, sBits, sD,
                          d_pmin + (size_t)o0 * nx, (long long)nx, nullptr, nullptr, 0};
            const OrientDesc* odo = d_odb + o0;
            if (xf) {
                PROF("k_xpass", st);
                int ncols = g.F[1] * g.H;
                pdl(xf, dim3((ncols + PSB_XCOLS - 1) / PSB_XCOLS, m), 256, xpass2_smem(g.F[0]), st)(
                    odo, sbo, d_Socc, d_Sphi, ncols, g.p[0].tw, nullptr, 0, BaseMap{0, 0, 0, nullptr, nullptr});
            } else {
                PROF("k_xpass", st);
                size_t smx = sizeof(float2) * (g.F[0] + 4 * PSB_TILE * g.F[0]);
                pdl(k_xpass, dim3((g.H + PSB_TILE - 1) / PSB_TILE, g.F[1], m), PSB_THREADS, smx, st)(
                    odo, sbo, d_Socc, d_Sphi, g.F[1], g.H, g.p[0].p, g.p[0].tw);
            }
            CKL();
            if (pf) {
                PROF("k_plane", st);
                pdl(pf, dim3(nx, m), pthreads, sm2, st)(odo, sbo, pbo, sp, g.p[1].tw, g.p[2].tw);
            } else {
                PROF("k_plane", st);
                pdl(k_plane, dim3(nx, m), PSB_THREADS, smp, st)(odo, sbo, pbo, sp, g.F[1], g.F[2], g.p[1].p,
                                                                g.p[2].p, g.p[1].tw, g.p[2].tw);
            }
            CKL();
        }
        auto select = [&](const uint32_t* ok, const int* gate) -> int {
            return select_over(d_odb, n, sp, ok, gate, d_out);
        };
        // flood fill over the free bits, then a selection over the reachable cells
        auto reach_select = [&](const int* gate) -> int {
            TRY(flood_fill(d_odb, n, sp, gate, nullptr));
            SelectBufs sel{d_reach,   sBits,  d_Dq,     sD,       d_smin, d_cand,        d_ncand, d_cscore, d_best,
                           d_bestkey, d_diag, d_errmax, kCandCap, d_pmin, (long long)nx, gate};
            pdl(k_sel_reset, 1, 128, 0, st)(sel, n);
            CKL();
            {
                PROF("k_plane_min", st);
                pdl(k_plane_min, dim3(nx, n), PSB_PMIN_THREADS, 0, st)(d_odb, sel, sp);
            }
            CKL();
            return select(d_reach, gate);
        };
        // plane minima over the free cells (k_plane3 and the generic k_plane
        // write them themselves)
        if (pf && (!interlock || lazy)) {
            SelectBufs sel{d_free,    sBits,  d_Dq,     sD,       d_smin, d_cand,        d_ncand, d_cscore, d_best,
                           d_bestkey, d_diag, d_errmax, kCandCap, d_pmin, (long long)nx, nullptr};
            PROF("k_plane_min", st);
            pdl(k_plane_min, dim3(nx, n), PSB_PMIN_THREADS, 0, st)(d_odb, sel, sp);
            CKL();
        }
        if (!interlock) {
            TRY(select(d_free, nullptr));
        } else if (!lazy) {
            TRY(reach_select(nullptr));
        } else {
            TRY(select(d_free, nullptr));
            {
                PROF("k_line_check", st);
                pdl(k_line_check, 1, 192, 0, st)(d_odb, d_out, n, d_free, sBits, sp, d_needff);
            }
            CKL();
            TRY(reach_select(d_needff));
        }
        return PSB_OK;
    }

    // Synchronous search (the drop-in entry points): upload, queue, wait, check.
    int search(const std::vector<OrientDesc>& ods, int mode, bool interlock, std::vector<ResultDev>* res,
               bool lazy = true) {
        const int n = (int)ods.size();
        TRY(ensure_slots(std::max(n, 6)));
        std::vector<OrientDesc> od2(ods), bases;
        const bool share = make_bases(&od2, &bases);
        CK(cudaMemcpyAsync(d_od, od2.data(), sizeof(OrientDesc) * n, cudaMemcpyHostToDevice, st));
        if (share) CK(cudaMemcpyAsync(d_bases, bases.data(), sizeof(OrientDesc) * 6, cudaMemcpyHostToDevice, st));
        const int sst = search_async(d_od, od2, mode, interlock, d_res, lazy, share ? d_bases : nullptr,
                                     share ? &bases : nullptr);
        late_active = false;
        TRY(sst);
        res->resize(n);
        unsigned int herr = 0;
        CK(cudaMemcpyAsync(res->data(), d_res, sizeof(ResultDev) * n, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&herr, d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (herr) return fail(PSB_ERR_LIMIT, "flood fill union-find hit its iteration limit");
        for (int o = 0; o < n; ++o)
            if ((*res)[o].diag & 0x100u)
                return fail(PSB_ERR_LIMIT, "orientation %d: %d tie-guard candidates exceed the capacity %d", o,
                            (*res)[o].ncand, kCandCap);
        return PSB_OK;
    }

    // device placement of an item described by od (slot 0 of d_od is overwritten)
    int place(const OrientDesc& od, int px, int py, int pz, int32_t id, int32_t* overlap_ijk) {
        TRY(ensure_slots(1));
        CK(cudaMemcpyAsync(d_od, &od, sizeof(OrientDesc), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(d_first, 0xff, sizeof(unsigned long long), st));
        int blocks = std::max(1, std::min(1024, (od.nvox + 255) / 256));
        pdl(k_place_check, blocks, 256, 0, st)(d_od, d_tray, nx, ny, nz, px, py, pz, d_first);
        CKL();
        unsigned long long first = 0;
        CK(cudaMemcpyAsync(&first, d_first, sizeof(first), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (first != 0xffffffffffffffffULL) {
            int k = (int)(first % nz), j = (int)((first / nz) % ny), i = (int)(first / ((size_t)ny * nz));
            if (overlap_ijk) { overlap_ijk[0] = i; overlap_ijk[1] = j; overlap_ijk[2] = k; }
            return fail(PSB_ERR_OVERLAP,
                        "(place_in_tray): Item to be placed intersects with contents of tray at position (%d, %d, %d)",
                        i, j, k);
        }
        pdl(k_place_write, blocks, 256, 0, st)(d_od, d_tray, nx, ny, nz, px, py, pz, id);
        CKL();
        TRY(prefix_occ());
        TRY(rebuild_occ());
        if (id == 1 && od.nvox > 0) {  // only voxels equal to 1 are distance sources (fft3.cu:948)
            TRY(distance_on_device(d_tray, d_phi, nx, ny, nz, st));
            TRY(prefix_phi(nullptr));
            TRY(rebuild_phi_spectrum());
        }
        CK(cudaStreamSynchronize(st));
        return PSB_OK;
    }
};

namespace {

const int kIdentity[3] = {0, 1, 2};
const int kNoFlip[3] = {0, 0, 0};

void to_result(const ResultDev& r, int orient, psb_result* out) {
    out->x = r.found ? r.x : -1;
    out->y = r.found ? r.y : -1;
    out->z = r.found ? r.z : -1;
    out->found = r.found;
    out->score = r.found ? r.score : 0.0;
    out->orientation = r.found ? orient : -1;
    out->diag = r.diag;
    out->n_candidates = r.ncand;
    out->err_ratio = r.err_ratio;
}

// Upload a set of explicit orientation arrays and describe them.
int stage_arrays(psb_tray* t, const int32_t* const* items, const int32_t* dims, int n, std::vector<OrientDesc>* ods) {
    std::vector<ItemInfo> infos(n);
    size_t tot = 0, totv = 0, totr = 0;
    for (int o = 0; o < n; ++o) {
        int ex = dims[3 * o], ey = dims[3 * o + 1], ez = dims[3 * o + 2];
        if (!items[o] || ex <= 0 || ey <= 0 || ez <= 0)
            return fail(PSB_ERR_ARG, "orientation %d: bad array (dims %d,%d,%d)", o, ex, ey, ez);
        size_t m = (size_t)ex * ey * ez;
        if (has_negative(items[o], m)) return fail(PSB_ERR_ARG, "orientation %d holds negative values", o);
        analyse_item(items[o], ex, ey, ez, &infos[o]);
        build_runs(items[o], &infos[o], 2);   // identity orientations: z-runs along the item's own z
        tot += m;
        totv += infos[o].vox.size();
        totr += infos[o].runs[2].size();
    }
    TRY(t->ensure_staging(tot, totv));
    TRY(t->ensure_runs(totr));
    size_t off = 0, offv = 0, offr = 0;
    ods->resize(n);
    for (int o = 0; o < n; ++o) {
        size_t m = (size_t)infos[o].dims[0] * infos[o].dims[1] * infos[o].dims[2];
        CK(cudaMemcpyAsync(t->d_items + off, items[o], sizeof(int32_t) * m, cudaMemcpyHostToDevice, t->st));
        if (!infos[o].vox.empty())
            CK(cudaMemcpyAsync(t->d_vox + offv, infos[o].vox.data(), sizeof(int4) * infos[o].vox.size(),
                               cudaMemcpyHostToDevice, t->st));
        if (!infos[o].runs[2].empty())
            CK(cudaMemcpyAsync(t->d_runs + offr, infos[o].runs[2].data(), sizeof(int4) * infos[o].runs[2].size(),
                               cudaMemcpyHostToDevice, t->st));
        const int4* rn[3] = {nullptr, nullptr, t->d_runs + offr};
        t->describe(infos[o], kIdentity, kNoFlip, t->d_items + off, t->d_vox + offv, rn, &(*ods)[o]);
        off += m;
        offv += infos[o].vox.size();
        offr += infos[o].runs[2].size();
    }
    CK(cudaStreamSynchronize(t->st));  // host vectors die at return
    return PSB_OK;
}

// cached contexts for the stateless entry points, keyed by dims.  A caller
// holds g_util_call_mu for its whole call (UtilCall), so a cached context is
// used by one call at a time and is never dropped while another call uses it.
std::mutex g_util_mu;
std::map<std::tuple<int, int, int, int>, std::unique_ptr<psb_tray>> g_util;
std::recursive_mutex g_util_call_mu;
typedef std::lock_guard<std::recursive_mutex> UtilCall;

int util_tray(int nx, int ny, int nz, psb_tray** out) {
    TRY(ensure_device());
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_util_mu);
    auto key = std::make_tuple(dev, nx, ny, nz);
    auto it = g_util.find(key);
    if (it != g_util.end()) { *out = it->second.get(); return PSB_OK; }
    if (g_util.size() >= 4) g_util.clear();
    std::unique_ptr<psb_tray> t(new psb_tray());
    TRY(t->init(nx, ny, nz));
    *out = t.get();
    g_util[key] = std::move(t);
    return PSB_OK;
}

// scratch arena for the stateless transforms
struct Arena {
    void* p = nullptr;
    size_t n = 0;
    int dev = -1;
};
thread_local Arena g_arena;

int arena(size_t bytes, void** out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (g_arena.n < bytes || g_arena.dev != dev) {
        if (g_arena.p && g_arena.dev == dev) cudaFree(g_arena.p);
        g_arena.p = nullptr;
        CK(cudaMalloc(&g_arena.p, bytes));
        g_arena.n = bytes;
        g_arena.dev = dev;
    }
    *out = g_arena.p;
    return PSB_OK;
}

// corr (conj_b=1): out[t] = sum_x b[x] a[t+x] ; conv (conj_b=0): linear conv
int linear_transform_product(const int32_t* a, const int32_t* b, int nx, int ny, int nz, int conj_b, int32_t* out) {
    TRY(ensure_device());
    TRY(set_smem_attrs());
    Grid3 g;
    TRY(make_grid3(nx, ny, nz, true, &g));
    size_t V = (size_t)nx * ny * nz;
    size_t S = (size_t)g.F[0] * g.F[1] * g.H;
    size_t w1 = (size_t)nx * ny * g.H, w2 = (size_t)nx * g.F[1] * g.H;
    size_t bytes = sizeof(float2) * (2 * S + w1 + w2) + sizeof(int32_t) * 2 * V + 4096;
    void* base = nullptr;
    TRY(arena(bytes, &base));
    char* p = (char*)base;
    auto take = [&](size_t n) { char* r = p; p += (n + 255) / 256 * 256; return r; };
    float2* Sa = (float2*)take(sizeof(float2) * S);
    float2* Sb = (float2*)take(sizeof(float2) * S);
    float2* W1 = (float2*)take(sizeof(float2) * w1);
    float2* W2 = (float2*)take(sizeof(float2) * w2);
    int32_t* da = (int32_t*)take(sizeof(int32_t) * V);
    int32_t* db = (int32_t*)take(sizeof(int32_t) * V);
    RzDesc* d_rz = (RzDesc*)take(sizeof(RzDesc) * 2);
    MidDesc* d_mid = (MidDesc*)take(sizeof(MidDesc) * 2);
    cudaStream_t st = 0;
    CK(cudaMemcpyAsync(da, a, sizeof(int32_t) * V, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(db, b, sizeof(int32_t) * V, cudaMemcpyHostToDevice, st));
    RzDesc ra{SRC_GRID_RAW, da, nx, ny, nz, 0, -1, nullptr};
    RzDesc rb{SRC_GRID_RAW, db, nx, ny, nz, 0, -1, nullptr};
    TRY(forward3(g, ra, W1, W2, Sa, d_rz, d_mid, st));
    CK(cudaStreamSynchronize(st));
    TRY(forward3(g, rb, W1, W2, Sb, d_rz + 1, d_mid, st));
    {
        PROF("k_spec_mul", st);
        pdl(k_spec_mul, grid1d(S), 256, 0, st)(Sa, Sb, Sa, S, conj_b);
    }
    CKL();
    CK(cudaStreamSynchronize(st));
    TRY(inverse3_int(g, Sa, W1, W2, da, d_mid, st));
    CK(cudaMemcpyAsync(out, da, sizeof(int32_t) * V, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return PSB_OK;
}

}  // namespace

// ===========================================================================
// psb_proposal: the learned orientation proposal (network in psb_proposal.cuh)
// ===========================================================================
namespace {
// flat parameter layout (the same order as the oracle's LAYERS)
struct PropLayer {
    size_t w, b;     // offsets of weight and bias
    size_t nw, nb;
};
struct PropLayout {
    PropLayer c[4], f1, f2, h1, h2;
    size_t n = 0;
    PropLayout() {
        const int ci[4] = {1, 16, 32, 64}, co[4] = {16, 32, 64, 64};
        auto add = [&](PropLayer& L, size_t nw, size_t nb) {
            L.w = n; L.nw = nw; n += nw;
            L.b = n; L.nb = nb; n += nb;
        };
        for (int i = 0; i < 4; ++i) add(c[i], (size_t)co[i] * ci[i] * 27, co[i]);
        add(f1, 64 * 512, 64);
        add(f2, 64 * PSB_PH * PSB_PH, 64);
        add(h1, 64 * 128, 64);
        add(h2, 64, 1);
    }
};
const PropLayout kProp;
}  // namespace

struct psb_proposal {
    int dev = 0;
    cudaStream_t st = nullptr;     // own stream for training; the packing loop passes the tray's
    float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;
    uint16_t* P16 = nullptr;
    unsigned char* isw = nullptr;
    long long step = 0;
    int capS = 0, capB = 0;
    float *a0 = nullptr, *a1 = nullptr, *a2 = nullptr, *a3 = nullptr, *a4 = nullptr, *f1 = nullptr, *t = nullptr,
          *hin = nullptr, *h1 = nullptr, *logit = nullptr, *dlogit = nullptr, *hm = nullptr;
    float *da1 = nullptr, *da2 = nullptr, *da3 = nullptr, *da4 = nullptr, *df1 = nullptr, *dt = nullptr,
          *dhin = nullptr, *dh1 = nullptr, *loss = nullptr;
    int* stats = nullptr;          // gating: items seen, fallbacks

    ~psb_proposal() { release(); }
    void free_acts() {
        for (float** q : {&a0, &a1, &a2, &a3, &a4, &f1, &t, &hin, &h1, &logit, &dlogit, &hm, &da1, &da2, &da3, &da4,
                          &df1, &dt, &dhin, &dh1})
            dfree(*q);
        capS = capB = 0;
    }
    void release() {
        cudaSetDevice(dev);
        free_acts();
        dfree(P); dfree(G); dfree(M); dfree(V); dfree(P16); dfree(isw); dfree(loss); dfree(stats);
        if (st) cudaStreamDestroy(st);
        st = nullptr;
    }
    int init() {
        TRY(ensure_device());
        CK(cudaGetDevice(&dev));
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        const size_t n = kProp.n;
        TRY(dalloc(&P, n)); TRY(dalloc(&G, n)); TRY(dalloc(&M, n)); TRY(dalloc(&V, n));
        TRY(dalloc(&P16, n)); TRY(dalloc(&isw, n)); TRY(dalloc(&loss, 1)); TRY(dalloc(&stats, 2));
        std::vector<unsigned char> w(n, 0);
        auto mark = [&](const PropLayer& L) { memset(w.data() + L.w, 1, L.nw); };
        for (int i = 0; i < 4; ++i) mark(kProp.c[i]);
        mark(kProp.f1); mark(kProp.f2); mark(kProp.h1); mark(kProp.h2);
        CK(cudaMemcpy(isw, w.data(), n, cudaMemcpyHostToDevice));
        CK(cudaMemset(P, 0, sizeof(float) * n));
        CK(cudaMemset(M, 0, sizeof(float) * n));
        CK(cudaMemset(V, 0, sizeof(float) * n));
        CK(cudaMemset(P16, 0, sizeof(uint16_t) * n));
        CK(cudaMemset(stats, 0, sizeof(int) * 2));
        return PSB_OK;
    }
    int ensure(int S, int B) {
        if (S <= capS && B <= capB) return PSB_OK;
        free_acts();
        S = std::max(S, capS);
        B = std::max(B, capB);
        const size_t s = (size_t)S;
        TRY(dalloc(&a0, s * PSB_PG3)); TRY(dalloc(&a1, s * 16 * 4096)); TRY(dalloc(&a2, s * 32 * 512));
        TRY(dalloc(&a3, s * 64 * 64)); TRY(dalloc(&a4, s * 512)); TRY(dalloc(&f1, s * 64));
        TRY(dalloc(&t, (size_t)B * 64)); TRY(dalloc(&hin, s * 128)); TRY(dalloc(&h1, s * 64));
        TRY(dalloc(&logit, s)); TRY(dalloc(&dlogit, s)); TRY(dalloc(&hm, (size_t)B * PSB_PH * PSB_PH));
        TRY(dalloc(&da1, s * 16 * 4096)); TRY(dalloc(&da2, s * 32 * 512)); TRY(dalloc(&da3, s * 64 * 64));
        TRY(dalloc(&da4, s * 512)); TRY(dalloc(&df1, s * 64)); TRY(dalloc(&dt, (size_t)B * 64));
        TRY(dalloc(&dhin, s * 128)); TRY(dalloc(&dh1, s * 64));
        capS = S;
        capB = B;
        return PSB_OK;
    }

    // forward over B items of no orientations: grids [B*no][32^3], hmaps
    // [B][1024] (device) -> this->logit [B*no]
    int forward(const float* grids, const float* hmaps, int B, int no, cudaStream_t s) {
        const int S = B * no;
        auto g1 = [](long long n) { return (unsigned)((n + 255) / 256); };
        const int ci[4] = {1, 16, 32, 64}, co[4] = {16, 32, 64, 64}, D[4] = {32, 16, 8, 4};
        const float* in[4] = {grids, a1, a2, a3};
        float* out[4] = {a1, a2, a3, a4};
        for (int i = 0; i < 4; ++i) {
            const long long n = (long long)S * (D[i] / 2) * (D[i] / 2) * (D[i] / 2);
            PROF("k_prop_conv", s);
            pdl(k_conv_fwd, dim3(g1(n), co[i] / PSB_CPT), 256, sizeof(float) * PSB_CPT * ci[i] * 27, s)(
                in[i], S, ci[i], D[i], P16 + kProp.c[i].w, P + kProp.c[i].b, out[i], co[i]);
            CKL();
        }
        PROF("k_prop_head", s);
        pdl(k_lin_fwd, g1((long long)S * 64), 256, 0, s)(a4, S, 512, P16 + kProp.f1.w, P + kProp.f1.b, 64, 1, f1);
        CKL();
        pdl(k_lin_fwd, g1((long long)B * 64), 256, 0, s)(hmaps, B, PSB_PH * PSB_PH, P16 + kProp.f2.w, P + kProp.f2.b,
                                                        64, 1, t);
        CKL();
        pdl(k_concat, g1((long long)S * 128), 256, 0, s)(f1, t, S, no, hin);
        CKL();
        pdl(k_lin_fwd, g1((long long)S * 64), 256, 0, s)(hin, S, 128, P16 + kProp.h1.w, P + kProp.h1.b, 64, 1, h1);
        CKL();
        pdl(k_lin_fwd, g1(S), 256, 0, s)(h1, S, 64, P16 + kProp.h2.w, P + kProp.h2.b, 1, 0, logit);
        CKL();
        return PSB_OK;
    }

    // item branch only (conv stack + f1) for B items of no orientations
    // whose grids are at `grids`; f1 left in this->f1 [B*no][64]
    int item_features(const float* grids, int B, int no, cudaStream_t s) {
        const int S = B * no;
        auto g1 = [](long long n) { return (unsigned)((n + 255) / 256); };
        const int ci[4] = {1, 16, 32, 64}, co[4] = {16, 32, 64, 64}, D[4] = {32, 16, 8, 4};
        const float* in[4] = {grids, a1, a2, a3};
        float* out[4] = {a1, a2, a3, a4};
        for (int i = 0; i < 4; ++i) {
            const long long n = (long long)S * (D[i] / 2) * (D[i] / 2) * (D[i] / 2);
            PROF("k_prop_conv", s);
            pdl(k_conv_fwd, dim3(g1(n), co[i] / PSB_CPT), 256, sizeof(float) * PSB_CPT * ci[i] * 27, s)(
                in[i], S, ci[i], D[i], P16 + kProp.c[i].w, P + kProp.c[i].b, out[i], co[i]);
            CKL();
        }
        pdl(k_lin_fwd, g1((long long)S * 64), 256, 0, s)(a4, S, 512, P16 + kProp.f1.w, P + kProp.f1.b, 64, 1, f1);
        CKL();
        return PSB_OK;
    }

    // loss and every parameter gradient (into G) after forward()
    int backward(const float* grids, const float* hmaps, const float* target, const float* mask, int B, int no,
                 cudaStream_t s) {
        const int S = B * no;
        auto g1 = [](long long n) { return (unsigned)((n + 255) / 256); };
        CK(cudaMemsetAsync(G, 0, sizeof(float) * kProp.n, s));
        CK(cudaMemsetAsync(loss, 0, sizeof(float), s));
        pdl(k_softmax_ce, (B + 7) / 8, 256, 0, s)(logit, target, mask, B, no, dlogit, loss);
        CKL();
        pdl(k_lin_bwd_weight, dim3(g1(64), 1), 256, 0, s)(dlogit, h1, S, 1, 64, G + kProp.h2.w, G + kProp.h2.b);
        CKL();
        pdl(k_lin_bwd_data, g1((long long)S * 64), 256, 0, s)(dlogit, S, 1, P16 + kProp.h2.w, 64, h1, dh1);
        CKL();
        pdl(k_lin_bwd_weight, dim3(g1(128), 64), 256, 0, s)(dh1, hin, S, 64, 128, G + kProp.h1.w, G + kProp.h1.b);
        CKL();
        pdl(k_lin_bwd_data, g1((long long)S * 128), 256, 0, s)(dh1, S, 64, P16 + kProp.h1.w, 128, nullptr, dhin);
        CKL();
        pdl(k_split_item, g1((long long)S * 64), 256, 0, s)(dhin, f1, S, df1);
        CKL();
        pdl(k_split_tray, g1((long long)B * 64), 256, 0, s)(dhin, t, B, no, dt);
        CKL();
        pdl(k_lin_bwd_weight, dim3(g1(PSB_PH * PSB_PH), 64), 256, 0, s)(dt, hmaps, B, 64, PSB_PH * PSB_PH,
                                                                       G + kProp.f2.w, G + kProp.f2.b);
        CKL();
        pdl(k_lin_bwd_weight, dim3(g1(512), 64), 256, 0, s)(df1, a4, S, 64, 512, G + kProp.f1.w, G + kProp.f1.b);
        CKL();
        pdl(k_lin_bwd_data, g1((long long)S * 512), 256, 0, s)(df1, S, 64, P16 + kProp.f1.w, 512, a4, da4);
        CKL();
        const int ci[4] = {1, 16, 32, 64}, co[4] = {16, 32, 64, 64}, D[4] = {32, 16, 8, 4};
        const float* in[4] = {grids, a1, a2, a3};
        float* dout[4] = {da1, da2, da3, da4};
        for (int i = 3; i >= 0; --i) {
            // enough CTAs: about 2048 (ci, co, chunk) triples
            const int nch_goal = std::max(1, 2048 / (ci[i] * co[i]));
            const int chunk = std::max(1, (S + nch_goal - 1) / nch_goal);
            const int nch = (S + chunk - 1) / chunk;
            {
                PROF("k_prop_bwd_weight", s);
                pdl(k_conv_bwd_weight, dim3(ci[i], co[i], nch), 256, 0, s)(dout[i], in[i], S, ci[i], D[i], co[i], chunk,
                                                                          G + kProp.c[i].w, G + kProp.c[i].b);
            }
            CKL();
            if (i > 0) {
                const long long n = (long long)S * D[i] * D[i] * D[i];
                PROF("k_prop_bwd_data", s);
                pdl(k_conv_bwd_data, dim3(g1(n), ci[i]), 256, sizeof(float) * co[i] * 27, s)(
                    dout[i], S, ci[i], D[i], P16 + kProp.c[i].w, co[i], in[i], 1, dout[i - 1]);
                CKL();
            }
        }
        return PSB_OK;
    }
};

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* psb_version(void) { return "psacking_b200 0.1.0 (sm_100a)"; }

int psb_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return PSB_ERR_ARG;
    snprintf(buf, len, "%s", g_err.c_str());
    return PSB_OK;
}

int psb_device_count(int* n) {
    if (!n) return fail(PSB_ERR_ARG, "null pointer");
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) { cudaGetLastError(); c = 0; }
    *n = c;
    return PSB_OK;
}

int psb_dft_conv3(const int32_t* a, const int32_t* b, int nx, int ny, int nz, int32_t* out) {
    NvtxRange nvtx_range("psb_dft_conv3");
    TRY(check_grid_args(a, nx, ny, nz, "dft_conv3"));
    TRY(check_grid_args(b, nx, ny, nz, "dft_conv3"));
    if (!out) return fail(PSB_ERR_ARG, "dft_conv3: null output");
    return linear_transform_product(a, b, nx, ny, nz, 0, out);
}

int psb_dft_corr3(const int32_t* a, const int32_t* b, int nx, int ny, int nz, int32_t* out) {
    NvtxRange nvtx_range("psb_dft_corr3");
    TRY(check_grid_args(a, nx, ny, nz, "dft_corr3"));
    TRY(check_grid_args(b, nx, ny, nz, "dft_corr3"));
    if (!out) return fail(PSB_ERR_ARG, "dft_corr3: null output");
    return linear_transform_product(a, b, nx, ny, nz, 1, out);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// dft_corr3 for callers that cannot allocate device memory
// ---------------------------------------------------------------------------
// Everything psb_dft_corr3 would allocate (two spectra, two transform work
// buffers, the twiddle tables and the launch descriptors) lives in this fixed
// array instead.  It is created when the library's device code is loaded on a
// GPU and stays there until the process exits, on every GPU that loads it.
namespace {
constexpr int kNoAllocMaxSide = 32;                         // every axis <= 32 voxels
constexpr size_t kNoAllocScratchBytes = (size_t)3 << 20;   // 3 MiB per GPU
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {nullptr};  // device address of the array, per device

// The descriptors and twiddle tables of one call, passed by value to
// k_noalloc_setup, which writes them into the array in stream order (no
// host-to-device copy, so the call never waits for the GPU).
struct NoAllocSetup {
    RzDesc rz[2];          // z passes of a and b
    MidDesc mid[6];        // y, x passes of a; of b; x, y passes of the inverse
    RzDesc* d_rz;
    MidDesc* d_mid;
    float2* tw[3];         // twiddle tables, F[a] entries each
    int F[3];
};

__global__ void k_noalloc_setup(NoAllocSetup s) {
    pdl_enter();
    if (blockIdx.x == 0 && threadIdx.x < 2) s.d_rz[threadIdx.x] = s.rz[threadIdx.x];
    if (blockIdx.x == 0 && threadIdx.x < 6) s.d_mid[threadIdx.x] = s.mid[threadIdx.x];
    // tw[a][i] = exp(-2 pi i / F), in double precision, rounded to float
    for (int a = 0; a < 3; ++a)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.F[a]; i += gridDim.x * blockDim.x) {
            double sn, cs;
            sincospi(-2.0 * (double)i / (double)s.F[a], &sn, &cs);
            s.tw[a][i] = make_float2((float)cs, (float)sn);
        }
}
}  // namespace

extern "C" {

int psb_dft_corr3_noalloc(const int32_t* d_a, const int32_t* d_b, int nx, int ny, int nz, int32_t* d_out,
                          void* stream) {
    if (!d_a || !d_b || !d_out) return fail(PSB_ERR_ARG, "dft_corr3_noalloc: null device pointer");
    if (nx <= 0 || ny <= 0 || nz <= 0)
        return fail(PSB_ERR_ARG, "dft_corr3_noalloc: dims must be positive, got (%d,%d,%d)", nx, ny, nz);
    if (nx > kNoAllocMaxSide || ny > kNoAllocMaxSide || nz > kNoAllocMaxSide)
        return fail(PSB_ERR_LIMIT,
                    "dft_corr3_noalloc: grid (%d,%d,%d) exceeds the fixed scratch limit of %d voxels per axis; "
                    "use psb_dft_corr3", nx, ny, nz, kNoAllocMaxSide);
    TRY(ensure_device());
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(PSB_ERR_ARG, "dft_corr3_noalloc: device index %d out of range", dev);
    void* scratch = nullptr;
    {
        // once per device, with that device current: the array's device address
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            g_noalloc_ptr[dev] = p;
        }
        scratch = g_noalloc_ptr[dev];
    }
    Grid3 g;
    g.n[0] = nx; g.n[1] = ny; g.n[2] = nz;
    for (int a = 0; a < 3; ++a) {
        g.F[a] = fft_len(2 * g.n[a] - 1);
        if (g.F[a] < 0 || !factorize(g.F[a], &g.p[a].p))
            return fail(PSB_ERR_ARG, "dft_corr3_noalloc: no FFT length for axis %d", a);
    }
    g.H = g.F[2] / 2 + 1;
    const size_t S = (size_t)g.F[0] * g.F[1] * g.H;
    const size_t w1 = (size_t)nx * ny * g.H, w2 = (size_t)nx * g.F[1] * g.H;
    char* p = (char*)scratch;
    size_t used = 0;
    auto take = [&](size_t n) {
        char* r = p + used;
        used += (n + 255) / 256 * 256;
        return r;
    };
    NoAllocSetup su;
    for (int a = 0; a < 3; ++a) {
        su.tw[a] = (float2*)take(sizeof(float2) * g.F[a]);
        su.F[a] = g.F[a];
        g.p[a].tw = su.tw[a];
    }
    su.d_rz = (RzDesc*)take(sizeof(RzDesc) * 2);
    su.d_mid = (MidDesc*)take(sizeof(MidDesc) * 6);
    float2* Sa = (float2*)take(sizeof(float2) * S);
    float2* Sb = (float2*)take(sizeof(float2) * S);
    float2* W1 = (float2*)take(sizeof(float2) * w1);
    float2* W2 = (float2*)take(sizeof(float2) * w2);
    if (used > kNoAllocScratchBytes)
        return fail(PSB_ERR_LIMIT, "dft_corr3_noalloc: grid (%d,%d,%d) needs %zu B of scratch, the fixed array has %zu B",
                    nx, ny, nz, used, kNoAllocScratchBytes);
    cudaStream_t st = (cudaStream_t)stream;
    su.rz[0] = RzDesc{SRC_GRID_RAW, d_a, nx, ny, nz, 0, -1, W1, nullptr, nullptr};
    su.rz[1] = RzDesc{SRC_GRID_RAW, d_b, nx, ny, nz, 0, -1, W1, nullptr, nullptr};
    forward_mids(g, W1, W2, Sa, nullptr, su.mid + 0);
    forward_mids(g, W1, W2, Sb, nullptr, su.mid + 2);
    // inverse: x [1][F0 -> n0][F1*H] (Sa -> W2), then y [n0][F1 -> n1][H] (W2 -> W1)
    su.mid[4] = MidDesc{Sa, W2, 1, g.F[1] * g.H, g.F[0], g.n[0], 0, 0, g.F[1] * g.H, g.F[1] * g.H, -1, 0, nullptr};
    su.mid[5] = MidDesc{W2, W1, g.n[0], g.H, g.F[1], g.n[1], (long long)g.F[1] * g.H, (long long)g.n[1] * g.H, g.H,
                        g.H, -1, 0, nullptr};
    // every byte the transforms read is written first in stream order, so
    // nothing in the array needs clearing
    pdl(k_noalloc_setup, 4, 256, 0, st)(su);
    CKL();
    TRY(forward3_dev(g, su.d_rz + 0, su.d_mid + 0, st));
    TRY(forward3_dev(g, su.d_rz + 1, su.d_mid + 2, st));
    pdl(k_spec_mul, grid1d(S), 256, 0, st)(Sa, Sb, Sa, S, 1);
    CKL();
    TRY(inverse3_dev(g, W1, d_out, su.d_mid + 4, st));
    return PSB_OK;
}

int psb_collision_grid(const int32_t* tray, int nx, int ny, int nz, const int32_t* item, int ex, int ey, int ez,
                       int32_t* out) {
    NvtxRange nvtx_range("psb_collision_grid");
    TRY(check_grid_args(tray, nx, ny, nz, "collision_grid"));
    TRY(check_grid_args(item, ex, ey, ez, "collision_grid"));
    if (ex > nx || ey > ny || ez > nz)
        return fail(PSB_ERR_ARG, "collision_grid: item (%d,%d,%d) larger than tray (%d,%d,%d)", ex, ey, ez, nx, ny, nz);
    size_t V = (size_t)nx * ny * nz;
    std::vector<int32_t> padded(V, 0);
    ItemInfo info;
    for (int i = 0; i < ex; ++i)
        for (int j = 0; j < ey; ++j)
            memcpy(&padded[((size_t)i * ny + j) * nz], &item[((size_t)i * ey + j) * ez], sizeof(int32_t) * ez);
    analyse_item(item, ex, ey, ez, &info);
    TRY(linear_transform_product(tray, padded.data(), nx, ny, nz, 1, out));
    // bounds of the padded item (voxelGrid.cpp:279-299); empty -> -INF
    int hx = info.hi[0] < 0 ? -1000000000 : info.hi[0];
    int hy = info.hi[0] < 0 ? -1000000000 : info.hi[1];
    int hz = info.hi[0] < 0 ? -1000000000 : info.hi[2];
    void* base = nullptr;
    TRY(arena(sizeof(int32_t) * V + 256, &base));
    int32_t* d = (int32_t*)base;
    CK(cudaMemcpy(d, out, sizeof(int32_t) * V, cudaMemcpyHostToDevice));
    k_oob_raise<<<grid1d(V), 256>>>(d, nx, ny, nz, hx, hy, hz);
    CKL();
    CK(cudaMemcpy(out, d, sizeof(int32_t) * V, cudaMemcpyDeviceToHost));
    return PSB_OK;
}

int psb_calculate_distance(const int32_t* grid, int nx, int ny, int nz, int32_t* out) {
    NvtxRange nvtx_range("psb_calculate_distance");
    TRY(check_grid_args(grid, nx, ny, nz, "calculate_distance"));
    if (!out) return fail(PSB_ERR_ARG, "calculate_distance: null output");
    TRY(ensure_device());
    TRY(set_smem_attrs());
    size_t V = (size_t)nx * ny * nz;
    void* base = nullptr;
    TRY(arena(sizeof(int32_t) * 2 * V + 512, &base));
    int32_t* dg = (int32_t*)base;
    int32_t* dd = dg + ((V + 63) / 64) * 64;
    CK(cudaMemcpy(dg, grid, sizeof(int32_t) * V, cudaMemcpyHostToDevice));
    TRY(distance_on_device(dg, dd, nx, ny, nz, 0));
    CK(cudaMemcpy(out, dd, sizeof(int32_t) * V, cudaMemcpyDeviceToHost));
    return PSB_OK;
}

int psb_interlocking_free_positions(const int32_t* tray, int nx, int ny, int nz, const int32_t* obj, int ex, int ey,
                                    int ez, int32_t* out) {
    NvtxRange nvtx_range("psb_interlocking_free_positions");
    TRY(check_grid_args(tray, nx, ny, nz, "interlocking_free_positions"));
    TRY(check_grid_args(obj, ex, ey, ez, "interlocking_free_positions"));
    if (ex > nx || ey > ny || ez > nz)
        return fail(PSB_ERR_ARG, "interlocking_free_positions: object larger than tray");
    // obj_max from voxels != 0, 0 when none (bindings.cpp:585-597)
    int om[3] = {0, 0, 0};
    for (int i = 0; i < ex; ++i)
        for (int j = 0; j < ey; ++j)
            for (int k = 0; k < ez; ++k)
                if (obj[((size_t)i * ey + j) * ez + k] != 0) {
                    om[0] = std::max(om[0], i); om[1] = std::max(om[1], j); om[2] = std::max(om[2], k);
                }
    size_t V = (size_t)nx * ny * nz;
    std::vector<int32_t> coll(V);
    TRY(psb_collision_grid(tray, nx, ny, nz, obj, ex, ey, ez, coll.data()));
    UtilCall serial(g_util_call_mu);
    psb_tray* t = nullptr;
    TRY(util_tray(nx, ny, nz, &t));
    TRY(t->ensure_slots(1));
    OrientDesc od;
    memset(&od, 0, sizeof(od));
    int n[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a) {
        od.e[a] = n[a];
        od.hi[a] = om[a];
        od.valid[a] = std::max(0, n[a] - om[a]);
    }
    int32_t* dcoll = (int32_t*)t->d_Dq;  // slot 0 proximity buffer reused as int32 scratch
    CK(cudaMemcpyAsync(dcoll, coll.data(), sizeof(int32_t) * V, cudaMemcpyHostToDevice, t->st));
    CK(cudaMemcpyAsync(t->d_od, &od, sizeof(od), cudaMemcpyHostToDevice, t->st));
    pdl(k_bits_from_coll, grid1d((size_t)nx * ny), 256, 0, t->st)(dcoll, t->d_free, nx, ny, nz, t->nzw, od.valid[0],
                                                                   od.valid[1], od.valid[2]);
    CKL();
    CK(cudaMemsetAsync(t->d_err, 0, sizeof(unsigned int), t->st));
    ScoreParams sp = t->score_params(1);
    FloodBufs fb{t->d_free, t->d_reach, t->sBits, t->d_cnt, t->d_off, t->sLine, t->d_rz2, t->d_rline, t->d_par,
                 t->d_rflag, t->sRun, t->d_total, t->d_err, nullptr, nullptr, 0, g_uf_limit};
    int lines = nx * ny;
    const int nblk = (lines + 255) / 256;
    dim3 gl(nblk, 1);
    CK(cudaMemsetAsync(t->d_total, 0, sizeof(int), t->st));
    {
        PROF("k_ff_runs", t->st);
        pdl(k_ff_runs, gl, 256, 0, t->st)(t->d_od, fb, sp);
    }
    {
        PROF("k_ff_union", t->st);
        pdl(k_ff_union, gl, 256, 0, t->st)(t->d_od, fb, sp);
    }
    {
        PROF("k_ff_seed", t->st);
        pdl(k_ff_seed, dim3(296, 1), 256, 0, t->st)(t->d_od, fb);
    }
    {
        PROF("k_ff_reach", t->st);
        pdl(k_ff_reach, gl, 256, 0, t->st)(t->d_od, fb, sp);
    }
    pdl(k_bits_to_mask, grid1d(V), 256, 0, t->st)(t->d_reach, dcoll, nx, ny, nz, t->nzw);
    CKL();
    unsigned int herr = 0;
    CK(cudaMemcpyAsync(out, dcoll, sizeof(int32_t) * V, cudaMemcpyDeviceToHost, t->st));
    CK(cudaMemcpyAsync(&herr, t->d_err, sizeof(herr), cudaMemcpyDeviceToHost, t->st));
    CK(cudaStreamSynchronize(t->st));
    if (herr) return fail(PSB_ERR_LIMIT, "flood fill union-find hit its iteration limit");
    return PSB_OK;
}

int psb_fft_search_placement(const int32_t* item, int ex, int ey, int ez, const int32_t* tray, int nx, int ny, int nz,
                             psb_result* out) {
    NvtxRange nvtx_range("psb_fft_search_placement");
    TRY(check_grid_args(item, ex, ey, ez, "fft_search_placement"));
    TRY(check_grid_args(tray, nx, ny, nz, "fft_search_placement"));
    if (!out) return fail(PSB_ERR_ARG, "fft_search_placement: null result");
    psb_result none{-1, -1, -1, 0, 0.0, -1, 0, 0, 0.f};
    *out = none;
    if (ex > nx || ey > ny || ez > nz) return PSB_OK;  // bindings.cpp:189-194
    UtilCall serial(g_util_call_mu);
    psb_tray* t = nullptr;
    TRY(util_tray(nx, ny, nz, &t));
    TRY(t->set(tray, nullptr));
    const int32_t* items[1] = {item};
    int32_t dims[3] = {ex, ey, ez};
    return psb_tray_search(t, items, dims, 1, PSB_MODE_SCAN, out, nullptr);
}

int psb_place_in_tray(const int32_t* item, int ex, int ey, int ez, const int32_t* tray, int nx, int ny, int nz, int px,
                      int py, int pz, int32_t item_id, int32_t* out_tray, int32_t* overlap_ijk) {
    NvtxRange nvtx_range("psb_place_in_tray");
    TRY(check_grid_args(item, ex, ey, ez, "place_in_tray"));
    TRY(check_grid_args(tray, nx, ny, nz, "place_in_tray"));
    if (!out_tray) return fail(PSB_ERR_ARG, "place_in_tray: null output");
    TRY(ensure_device());
    size_t V = (size_t)nx * ny * nz;
    if (out_tray != tray) memcpy(out_tray, tray, sizeof(int32_t) * V);
    // the clipped box of tray cells the item covers
    int i0 = std::max(px, 0), j0 = std::max(py, 0), k0 = std::max(pz, 0);
    int i1 = std::min(nx, px + ex), j1 = std::min(ny, py + ey), k1 = std::min(nz, pz + ez);
    if (i0 >= i1 || j0 >= j1 || k0 >= k1) return PSB_OK;
    int bx = i1 - i0, by = j1 - j0, bz = k1 - k0;
    size_t B = (size_t)bx * by * bz;
    std::vector<int32_t> box(B);
    for (int i = 0; i < bx; ++i)
        for (int j = 0; j < by; ++j)
            memcpy(&box[((size_t)i * by + j) * bz], &tray[((size_t)(i0 + i) * ny + (j0 + j)) * nz + k0],
                   sizeof(int32_t) * bz);
    ItemInfo info;
    analyse_item(item, ex, ey, ez, &info);
    size_t I = (size_t)ex * ey * ez;
    void* base = nullptr;
    size_t need = sizeof(int32_t) * (B + I) + sizeof(int4) * (info.vox.size() + 1) + sizeof(OrientDesc) + 2048;
    TRY(arena(need, &base));
    char* p = (char*)base;
    auto take = [&](size_t n) { char* r = p; p += (n + 255) / 256 * 256; return r; };
    int32_t* dbox = (int32_t*)take(sizeof(int32_t) * B);
    int32_t* ditem = (int32_t*)take(sizeof(int32_t) * I);
    int4* dvox = (int4*)take(sizeof(int4) * (info.vox.size() + 1));
    OrientDesc* dod = (OrientDesc*)take(sizeof(OrientDesc));
    unsigned long long* dfirst = (unsigned long long*)take(sizeof(unsigned long long));
    OrientDesc od;
    memset(&od, 0, sizeof(od));
    for (int a = 0; a < 3; ++a) { od.src_axis[a] = a; od.flip[a] = 0; od.e[a] = info.dims[a]; od.b[a] = info.dims[a]; }
    od.item = ditem;
    od.vox = dvox;
    od.nvox = (int)info.vox.size();
    CK(cudaMemcpy(dbox, box.data(), sizeof(int32_t) * B, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ditem, item, sizeof(int32_t) * I, cudaMemcpyHostToDevice));
    if (!info.vox.empty()) CK(cudaMemcpy(dvox, info.vox.data(), sizeof(int4) * info.vox.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dod, &od, sizeof(od), cudaMemcpyHostToDevice));
    CK(cudaMemset(dfirst, 0xff, sizeof(unsigned long long)));
    int blocks = std::max(1, std::min(1024, (od.nvox + 255) / 256));
    // the box is a small tray: position relative to the box origin
    k_place_check<<<blocks, 256>>>(dod, dbox, bx, by, bz, px - i0, py - j0, pz - k0, dfirst);
    CKL();
    unsigned long long first = 0;
    CK(cudaMemcpy(&first, dfirst, sizeof(first), cudaMemcpyDeviceToHost));
    if (first != 0xffffffffffffffffULL) {
        int k = (int)(first % bz), j = (int)((first / bz) % by), i = (int)(first / ((size_t)by * bz));
        i += i0; j += j0; k += k0;
        // row-major order of the box agrees with the tray's row-major order
        if (overlap_ijk) { overlap_ijk[0] = i; overlap_ijk[1] = j; overlap_ijk[2] = k; }
        if (out_tray != tray) memcpy(out_tray, tray, sizeof(int32_t) * V);
        return fail(PSB_ERR_OVERLAP,
                    "(place_in_tray): Item to be placed intersects with contents of tray at position (%d, %d, %d)", i,
                    j, k);
    }
    k_place_write<<<blocks, 256>>>(dod, dbox, bx, by, bz, px - i0, py - j0, pz - k0, item_id);
    CKL();
    CK(cudaMemcpy(box.data(), dbox, sizeof(int32_t) * B, cudaMemcpyDeviceToHost));
    for (int i = 0; i < bx; ++i)
        for (int j = 0; j < by; ++j)
            memcpy(&out_tray[((size_t)(i0 + i) * ny + (j0 + j)) * nz + k0], &box[((size_t)i * by + j) * bz],
                   sizeof(int32_t) * bz);
    return PSB_OK;
}

int psb_tray_create(int nx, int ny, int nz, psb_tray** out) {
    if (!out) return fail(PSB_ERR_ARG, "null output");
    *out = nullptr;
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail(PSB_ERR_ARG, "tray dims must be positive");
    std::unique_ptr<psb_tray> t(new psb_tray());
    TRY(t->init(nx, ny, nz));
    *out = t.release();
    return PSB_OK;
}

int psb_tray_destroy(psb_tray* t) {
    delete t;
    return PSB_OK;
}

int psb_tray_dims(const psb_tray* t, int* nx, int* ny, int* nz) {
    if (!t || !nx || !ny || !nz) return fail(PSB_ERR_ARG, "null pointer");
    *nx = t->nx; *ny = t->ny; *nz = t->nz;
    return PSB_OK;
}

int psb_tray_set(psb_tray* t, const int32_t* tray, const int32_t* phi) {
    NvtxRange nvtx_range("psb_tray_set");
    if (!t || !tray) return fail(PSB_ERR_ARG, "null pointer");
    return t->set(tray, phi);
}

int psb_tray_get(psb_tray* t, int32_t* tray, int32_t* phi) {
    if (!t) return fail(PSB_ERR_ARG, "null tray");
    CK(cudaSetDevice(t->dev));
    if (tray) CK(cudaMemcpyAsync(tray, t->d_tray, sizeof(int32_t) * t->V, cudaMemcpyDeviceToHost, t->st));
    if (phi) CK(cudaMemcpyAsync(phi, t->d_phi, sizeof(int32_t) * t->V, cudaMemcpyDeviceToHost, t->st));
    CK(cudaStreamSynchronize(t->st));
    return PSB_OK;
}

int psb_tray_stats(psb_tray* t, long long* occupied, int32_t* lo, int32_t* hi) {
    if (!t || !occupied || !lo || !hi) return fail(PSB_ERR_ARG, "null pointer");
    if (!t->ready) return fail(PSB_ERR_STATE, "tray not initialised");
    CK(cudaSetDevice(t->dev));
    if (!t->d_ostat) TRY(dalloc(&t->d_ostat, 8, t->st));
    struct {
        unsigned long long count;
        int box[6];
    } h = {0ULL, {INT_MAX, INT_MAX, INT_MAX, -1, -1, -1}};
    CK(cudaMemcpyAsync(t->d_ostat, &h, sizeof(h), cudaMemcpyHostToDevice, t->st));
    pdl(k_occ_stats, 148 * 4, 256, 0, t->st)(t->d_tray, t->nx, t->ny, t->nz, (unsigned long long*)t->d_ostat,
                                             t->d_ostat + 2);
    CKL();
    CK(cudaMemcpyAsync(&h, t->d_ostat, sizeof(h), cudaMemcpyDeviceToHost, t->st));
    CK(cudaStreamSynchronize(t->st));
    *occupied = (long long)h.count;
    for (int a = 0; a < 3; ++a) {
        lo[a] = h.count ? h.box[a] : -1;
        hi[a] = h.count ? h.box[3 + a] : -1;
    }
    return PSB_OK;
}

int psb_tray_search(psb_tray* t, const int32_t* const* items, const int32_t* dims, int n, int mode_flags,
                    psb_result* out, psb_result* per_orient) {
    NvtxRange nvtx_range("psb_tray_search");
    if (!t || !items || !dims || !out || n < 0) return fail(PSB_ERR_ARG, "null pointer");
    if (!t->ready) return fail(PSB_ERR_STATE, "GPU tray context not initialized. Call gpu_tray_init() first.");
    CK(cudaSetDevice(t->dev));
    psb_result none{-1, -1, -1, 0, 0.0, -1, 0, 0, 0.f};
    *out = none;
    if (n == 0) return PSB_OK;
    std::vector<OrientDesc> ods;
    TRY(stage_arrays(t, items, dims, n, &ods));
    std::vector<ResultDev> res;
    int mode = mode_flags & 0xf;
    // every orientation's own result is exact only without the lazy flood fill
    TRY(t->search(ods, mode, (mode_flags & PSB_FLAG_INTERLOCK) != 0, &res, per_orient == nullptr));
    double best = 1e300;
    for (int o = 0; o < n; ++o) {
        psb_result r;
        to_result(res[o], o, &r);
        if (ods[o].skip) r.diag |= 0x200u;
        if (per_orient) per_orient[o] = r;
        if (r.found && r.score < best) { best = r.score; *out = r; }  // strict <: first best wins
    }
    return PSB_OK;
}

int psb_tray_place(psb_tray* t, const int32_t* item, int ex, int ey, int ez, int px, int py, int pz, int32_t item_id) {
    NvtxRange nvtx_range("psb_tray_place");
    if (!t || !item) return fail(PSB_ERR_ARG, "null pointer");
    if (!t->ready) return fail(PSB_ERR_STATE, "tray not initialised");
    CK(cudaSetDevice(t->dev));
    const int32_t* items[1] = {item};
    int32_t dims[3] = {ex, ey, ez};
    std::vector<OrientDesc> ods;
    TRY(stage_arrays(t, items, dims, 1, &ods));
    TRY(t->place(ods[0], px, py, pz, item_id, nullptr));
    t->occ += (size_t)std::max(0, ods[0].nvox);
    return PSB_OK;
}

}  // extern "C"

namespace {
// Staging of a packing run's items (psb_pack_stage, psb_pack).

// Null arrays, bad dims and negative values, checked for every item before
// anything is staged (items spread over the host cores).
int stage_check(const int32_t* const* items, const int32_t* dims, int n_items) {
    for (int it = 0; it < n_items; ++it) {
        const int ex = dims[3 * it], ey = dims[3 * it + 1], ez = dims[3 * it + 2];
        if (!items[it] || ex <= 0 || ey <= 0 || ez <= 0) return fail(PSB_ERR_ARG, "item %d: bad array", it);
    }
    std::vector<char> neg(n_items, 0);
    parallel_chunks((size_t)n_items, 4, [&](size_t b, size_t e) {
        for (size_t it = b; it < e; ++it) {
            const size_t m = (size_t)dims[3 * it] * dims[3 * it + 1] * dims[3 * it + 2];
            neg[it] = has_negative(items[it], m) ? 1 : 0;
        }
    });
    for (int it = 0; it < n_items; ++it)
        if (neg[it]) return fail(PSB_ERR_ARG, "item %d holds negative values", it);
    return PSB_OK;
}

// Runs, bounds, sums and filter samples of items [i0, i1) into t->staged
// (host only; the packing loop places items by their runs, so no voxel list
// is built).
void stage_analyse(psb_tray* t, const int32_t* const* items, const int32_t* dims, int i0, int i1) {
    parallel_chunks((size_t)(i1 - i0), 1, [&](size_t b, size_t e) {
        for (size_t k = b; k < e; ++k) {
            const int it = i0 + (int)k;
            ItemInfo& inf = t->staged[it];
            for (int a = 0; a < 3; ++a) inf.dims[a] = dims[3 * it + a];
            for (int a = 0; a < 3; ++a) build_runs(items[it], &inf, a);
            analyse_runs(&inf);
            pick_samples(&inf);
        }
    });
}

// Items [i0, i1) as one part: the part's device block holds their runs,
// samples and int32 arrays, filled from the part's pinned host block by one
// copy on stream s (no synchronisation); t->sdev gets their device pointers.
int stage_upload(psb_tray* t, const int32_t* const* items, int i0, int i1, int part, cudaStream_t s) {
    size_t n4 = 0, n1 = 0;   // int4 entries (runs, samples), int32 cells
    for (int it = i0; it < i1; ++it) {
        const ItemInfo& inf = t->staged[it];
        for (int a = 0; a < 3; ++a) n4 += inf.runs[a].size();
        n4 += inf.samp.size();
        n1 += (size_t)inf.dims[0] * inf.dims[1] * inf.dims[2];
    }
    const size_t bytes = sizeof(int4) * n4 + sizeof(int32_t) * n1;
    if (bytes > t->part_cap[part]) {
        dfree(t->d_part[part], t->st);
        t->part_cap[part] = 0;
        TRY(dalloc(&t->d_part[part], bytes, s));
        t->part_cap[part] = bytes;
    }
    if (bytes > t->h_part_cap[part]) {
        if (t->h_part[part]) cudaFreeHost(t->h_part[part]);
        t->h_part[part] = nullptr;
        t->h_part_cap[part] = 0;
        CK(cudaMallocHost(&t->h_part[part], bytes));
        t->h_part_cap[part] = bytes;
    }
    // offsets: every item's runs and samples, then the int32 arrays
    std::vector<size_t> o4(i1 - i0), o1(i1 - i0);
    size_t a4 = 0, a1 = 0;
    for (int it = i0; it < i1; ++it) {
        const ItemInfo& inf = t->staged[it];
        o4[it - i0] = a4;
        o1[it - i0] = a1;
        for (int a = 0; a < 3; ++a) a4 += inf.runs[a].size();
        a4 += inf.samp.size();
        a1 += (size_t)inf.dims[0] * inf.dims[1] * inf.dims[2];
    }
    int4* h4 = (int4*)t->h_part[part];
    int32_t* h1 = (int32_t*)(h4 + n4);
    const int4* d4 = (const int4*)t->d_part[part];
    const int32_t* d1 = (const int32_t*)(d4 + n4);
    parallel_chunks((size_t)(i1 - i0), 1, [&](size_t b, size_t e) {
        for (size_t k = b; k < e; ++k) {
            const int it = i0 + (int)k;
            const ItemInfo& inf = t->staged[it];
            psb_tray::StagedDev& sd = t->sdev[it];
            size_t q = o4[k];
            for (int a = 0; a < 3; ++a) {
                if (!inf.runs[a].empty()) memcpy(h4 + q, inf.runs[a].data(), sizeof(int4) * inf.runs[a].size());
                sd.runs[a] = d4 + q;
                q += inf.runs[a].size();
            }
            if (!inf.samp.empty()) memcpy(h4 + q, inf.samp.data(), sizeof(int4) * inf.samp.size());
            sd.samp = d4 + q;
            const size_t m = (size_t)inf.dims[0] * inf.dims[1] * inf.dims[2];
            memcpy(h1 + o1[k], items[it], sizeof(int32_t) * m);
            sd.item = d1 + o1[k];
        }
    });
    if (bytes) CK(cudaMemcpyAsync(t->d_part[part], t->h_part[part], bytes, cudaMemcpyHostToDevice, s));
    return PSB_OK;
}
}  // namespace

extern "C" {

int psb_pack_stage(psb_tray* t, const int32_t* const* items, const int32_t* dims, int n_items) {
    NvtxRange nvtx_range("psb_pack_stage");
    if (!t || (!items && n_items > 0) || !dims || n_items < 0) return fail(PSB_ERR_ARG, "null pointer");
    CK(cudaSetDevice(t->dev));
    t->staged.clear();
    t->sdev.clear();
    TRY(stage_check(items, dims, n_items));
    t->staged.resize(n_items);
    t->sdev.resize(n_items);
    stage_analyse(t, items, dims, 0, n_items);
    TRY(stage_upload(t, items, 0, n_items, 0, t->st));
    CK(cudaStreamSynchronize(t->st));
    return PSB_OK;
}

}  // extern "C"

namespace {
// Options of the packing loop beyond the plain form.
struct PackOpts {
    psb_proposal* prop = nullptr;   // learned proposal: gate each item's orientations
    int topk = 4;
    float margin = 0.f;
    psb_result* per_orient = nullptr;   // n_items x n_orient results of every orientation
    float* hmaps = nullptr;             // n_items x 1024 pooled height maps before each item
    int32_t* gate_stats = nullptr;      // [items gated, fallbacks to the full sweep]
    // orientation sharding (psb_pack_staged_sharded): this rank searches the
    // orientations o with o % world == rank; per item its decision goes to
    // d_local, exchange(ctx) gathers every rank's into d_all, and the merged
    // winner is placed
    int rank = 0, world = 1;
    // staging in two parts (psb_pack): items from feed_at on are staged by
    // feed() when the loop reaches them, uploaded on the tray's copy stream
    std::function<int()> feed;
    int feed_at = 0;
    void* d_local = nullptr;
    void* d_all = nullptr;
    psb_exchange_fn exchange = nullptr;
    void* ctx = nullptr;
};
int pack_staged_impl(psb_tray* t, const int32_t* orient_maps, int n_orient, int interlock, int32_t id_offset,
                     psb_result* out_placements, int32_t* final_tray, const PackOpts& opt);
}  // namespace

extern "C" {

int psb_pack_staged(psb_tray* t, const int32_t* orient_maps, int n_orient, int interlock, int32_t id_offset,
                    psb_result* out_placements, int32_t* final_tray) {
    NvtxRange nvtx_range("psb_pack_staged");
    return pack_staged_impl(t, orient_maps, n_orient, interlock, id_offset, out_placements, final_tray, PackOpts());
}

int psb_pack_staged_detail(psb_tray* t, const int32_t* orient_maps, int n_orient, int interlock, int32_t id_offset,
                           psb_result* out_placements, int32_t* final_tray, psb_result* per_orient, float* hmaps) {
    NvtxRange nvtx_range("psb_pack_staged_detail");
    PackOpts o;
    o.per_orient = per_orient;
    o.hmaps = hmaps;
    return pack_staged_impl(t, orient_maps, n_orient, interlock, id_offset, out_placements, final_tray, o);
}

int psb_pack_staged_sharded(psb_tray* t, const int32_t* orient_maps, int n_orient, int interlock, int32_t id_offset,
                            int rank, int world, void* d_local, void* d_all, psb_exchange_fn exchange, void* ctx,
                            psb_result* out_placements, int32_t* final_tray) {
    NvtxRange nvtx_range("psb_pack_staged_sharded");
    if (world < 1 || rank < 0 || rank >= world) return fail(PSB_ERR_ARG, "bad rank %d of world %d", rank, world);
    if (!d_local || !d_all) return fail(PSB_ERR_ARG, "sharded packing needs the decision buffers");
    if (world > 1 && !exchange) return fail(PSB_ERR_ARG, "sharded packing over %d ranks needs an exchange", world);
    PackOpts o;
    o.rank = rank;
    o.world = world;
    o.d_local = d_local;
    o.d_all = d_all;
    o.exchange = exchange;
    o.ctx = ctx;
    return pack_staged_impl(t, orient_maps, n_orient, interlock, id_offset, out_placements, final_tray, o);
}

int psb_pack_staged_prop(psb_tray* t, psb_proposal* prop, const int32_t* orient_maps, int n_orient, int interlock,
                         int32_t id_offset, int topk, float margin, psb_result* out_placements, int32_t* final_tray,
                         int32_t* gate_stats) {
    NvtxRange nvtx_range("psb_pack_staged_prop");
    if (!prop) return fail(PSB_ERR_ARG, "pack_staged_prop: null proposal");
    if (n_orient != PSB_PNO) return fail(PSB_ERR_ARG, "the proposal network ranks exactly %d orientations", PSB_PNO);
    if (topk < 1) return fail(PSB_ERR_ARG, "topk must be >= 1");
    PackOpts o;
    o.prop = prop;
    o.topk = topk;
    o.margin = margin;
    o.gate_stats = gate_stats;
    return pack_staged_impl(t, orient_maps, n_orient, interlock, id_offset, out_placements, final_tray, o);
}

}  // extern "C"

namespace {
int pack_staged_impl(psb_tray* t, const int32_t* orient_maps, int n_orient, int interlock, int32_t id_offset,
                     psb_result* out_placements, int32_t* final_tray, const PackOpts& opt) {
    if (!t || !orient_maps || n_orient <= 0 || !out_placements)
        return fail(PSB_ERR_ARG, "null pointer or bad orientation count");
    if (!t->ready) return fail(PSB_ERR_STATE, "tray not initialised");
    CK(cudaSetDevice(t->dev));
    for (int o = 0; o < n_orient; ++o) {
        const int32_t* m = orient_maps + 6 * o;
        int seen = 0;
        for (int a = 0; a < 3; ++a) {
            if (m[a] < 0 || m[a] > 2) return fail(PSB_ERR_ARG, "orientation %d: bad axis map", o);
            seen |= 1 << m[a];
        }
        if (seen != 7) return fail(PSB_ERR_ARG, "orientation %d: axis map is not a permutation", o);
    }
    const int mode = (interlock || n_orient > 1) ? PSB_MODE_BLOCK : PSB_MODE_SCAN;
    const int n_items = (int)t->staged.size();
    if (n_items == 0) {
        if (final_tray) TRY(psb_tray_get(t, final_tray, nullptr));
        return PSB_OK;
    }
    // slots for the orientations and the item's 6 permutation bases; reserved
    // here, before any slot pointer (d_res ...) is handed to a search
    TRY(t->ensure_slots(std::max(n_orient, 6)));
    // every orientation of every item, described once (bounds, maps, sizes);
    // the error bounds are filled on the device by k_prep from the current
    // distance statistics.  Items [i0, i1) at a time: with a feed (psb_pack)
    // the items from opt.feed_at on are described when the loop reaches them.
    std::vector<OrientDesc> all((size_t)n_items * n_orient);
    std::vector<OrientDesc> allb((size_t)n_items * 6);   // each item's 6 axis permutations
    // candidate-filter samples (tray columns of at most 256 cells)
    const bool filt = g_cand_filter && t->nzw <= 8;
    if (all.size() > t->od_all_cap) {
        dfree(t->d_od_all, t->st);
        t->od_all_cap = all.size();
        TRY(dalloc(&t->d_od_all, t->od_all_cap, t->st));
    }
    if (allb.size() > t->base_all_cap) {
        dfree(t->d_base_all, t->st);
        t->base_all_cap = allb.size();
        TRY(dalloc(&t->d_base_all, t->base_all_cap, t->st));
    }
    if ((size_t)n_items > t->dec_cap) {
        dfree(t->d_dec, t->st);
        t->dec_cap = n_items;
        TRY(dalloc(&t->d_dec, t->dec_cap, t->st));
    }
    // descriptors go to the device from pinned memory, so an upload queued
    // while the loop runs does not wait for the stream
    const size_t dbytes = sizeof(OrientDesc) * (all.size() + allb.size());
    if (dbytes > t->h_desc_cap) {
        if (t->h_desc) cudaFreeHost(t->h_desc);
        t->h_desc = nullptr;
        t->h_desc_cap = 0;
        CK(cudaMallocHost(&t->h_desc, dbytes));
        t->h_desc_cap = dbytes;
    }
    OrientDesc* hd_all = (OrientDesc*)t->h_desc;
    OrientDesc* hd_base = hd_all + all.size();
    // item columns of the direct checks, for every item up front (they do not
    // depend on the tray): one k_item_cols_all per described range
    const bool icols_pre = filt && t->split_flow() && g_direct_max > 0;
    if (icols_pre) {
        t->icol_off.assign(n_items, 0);
        t->icol_stride.assign(n_items, 0);
        if ((size_t)n_items > t->icmeta_cap) {
            dfree(t->d_icoff, t->st);
            dfree(t->d_icstr, t->st);
            t->icmeta_cap = 0;
            TRY(dalloc(&t->d_icoff, (size_t)n_items, t->st));
            TRY(dalloc(&t->d_icstr, (size_t)n_items, t->st));
            if (t->h_icmeta) cudaFreeHost(t->h_icmeta);
            t->h_icmeta = nullptr;
            CK(cudaMallocHost(&t->h_icmeta, (size_t)n_items * (sizeof(long long) + sizeof(int))));
            t->icmeta_cap = n_items;
        }
        if ((size_t)n_items * n_orient > t->icn_cap) {
            dfree(t->d_icn, t->st);
            t->icn_cap = 0;
            TRY(dalloc(&t->d_icn, (size_t)n_items * n_orient, t->st));
            t->icn_cap = (size_t)n_items * n_orient;
        }
    }
    auto item_cols_range = [&](int i0, int i1, cudaStream_t s) -> int {
        const int part = i0 == 0 ? 0 : 1;
        long long acc = 0;
        int emax = 1;
        for (int it = i0; it < i1; ++it) {
            const int* d = t->staged[it].dims;
            const int str = std::max(std::max(d[0] * d[1], d[0] * d[2]), d[1] * d[2]);
            t->icol_off[it] = acc;
            t->icol_stride[it] = str;
            acc += (long long)n_orient * str;
            emax = std::max(emax, std::max(d[0], std::max(d[1], d[2])));
        }
        if ((size_t)acc > t->icp_cap[part]) {
            dfree(t->d_icp[part], t->st);
            t->icp_cap[part] = 0;
            TRY(dalloc(&t->d_icp[part], (size_t)acc, s));
            t->icp_cap[part] = (size_t)acc;
        }
        long long* hoff = (long long*)t->h_icmeta;
        int* hstr = (int*)(hoff + t->icmeta_cap);
        memcpy(hoff + i0, t->icol_off.data() + i0, sizeof(long long) * (i1 - i0));
        memcpy(hstr + i0, t->icol_stride.data() + i0, sizeof(int) * (i1 - i0));
        CK(cudaMemcpyAsync(t->d_icoff + i0, hoff + i0, sizeof(long long) * (i1 - i0), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(t->d_icstr + i0, hstr + i0, sizeof(int) * (i1 - i0), cudaMemcpyHostToDevice, s));
        CK(cudaMemsetAsync(t->d_icn + (size_t)i0 * n_orient, 0, sizeof(int) * (size_t)(i1 - i0) * n_orient, s));
        pdl(k_item_cols_all, dim3(emax, n_orient, i1 - i0), 64, 0, s)(t->d_od_all, n_orient, i0, t->d_icp[part],
                                                                     t->d_icoff, t->d_icstr, t->d_icn);
        CKL();
        return PSB_OK;
    };
    auto describe_range = [&](int i0, int i1, cudaStream_t s) -> int {
        for (int it = i0; it < i1; ++it) {
            const psb_tray::StagedDev& sd = t->sdev[it];
            for (int o = 0; o < n_orient; ++o) {
                OrientDesc& od = all[(size_t)it * n_orient + o];
                t->describe(t->staged[it], orient_maps + 6 * o, orient_maps + 6 * o + 3, sd.item, nullptr, sd.runs,
                            &od);
                // orientation sharding: the other ranks' orientations are not searched here
                if (opt.world > 1 && o % opt.world != opt.rank) od.skip = 1;
                if (filt) {
                    od.samp = sd.samp;
                    od.nsamp = (int)t->staged[it].samp.size();
                }
            }
            // the flips of one axis permutation share its spectrum
            std::vector<OrientDesc> slice(all.begin() + (size_t)it * n_orient,
                                          all.begin() + (size_t)(it + 1) * n_orient);
            std::vector<OrientDesc> b;
            if (!make_bases(&slice, &b)) return fail(PSB_ERR_STATE, "item %d: orientations of different items", it);
            std::copy(slice.begin(), slice.end(), all.begin() + (size_t)it * n_orient);
            std::copy(b.begin(), b.end(), allb.begin() + (size_t)it * 6);
        }
        const size_t a0 = (size_t)i0 * n_orient, na = (size_t)(i1 - i0) * n_orient;
        const size_t b0 = (size_t)i0 * 6, nb = (size_t)(i1 - i0) * 6;
        memcpy(hd_all + a0, all.data() + a0, sizeof(OrientDesc) * na);
        memcpy(hd_base + b0, allb.data() + b0, sizeof(OrientDesc) * nb);
        CK(cudaMemcpyAsync(t->d_od_all + a0, hd_all + a0, sizeof(OrientDesc) * na, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(t->d_base_all + b0, hd_base + b0, sizeof(OrientDesc) * nb, cudaMemcpyHostToDevice, s));
        if (icols_pre) TRY(item_cols_range(i0, i1, s));
        return PSB_OK;
    };
    if (opt.feed && (opt.prop || opt.feed_at <= 0 || opt.feed_at >= n_items))
        return fail(PSB_ERR_STATE, "a staged feed needs 0 < feed_at < n_items and no proposal");
    TRY(describe_range(0, opt.feed ? opt.feed_at : n_items, t->st));
    LoopState ls0;
    memset(&ls0, 0, sizeof(ls0));
    ls0.id_offset = id_offset;
    CK(cudaMemcpyAsync(t->d_ls, &ls0, sizeof(ls0), cudaMemcpyHostToDevice, t->st));
    // optional outputs and the proposal's inputs
    ResultDev* d_per = nullptr;
    float* d_hm = nullptr;
    float* d_pgrid = nullptr;  // base grids of the staged items (proposal)
    int* d_pG = nullptr;       // their scaled extents
    int* d_pmaps = nullptr;
    struct Cleanup {
        psb_tray* t;
        ResultDev** per;
        float** hm;
        float** pg;
        int** pG;
        int** pm;
        ~Cleanup() { dfree(*per, t->st); dfree(*hm, t->st); dfree(*pg, t->st); dfree(*pG, t->st); dfree(*pm, t->st); }
    } cleanup{t, &d_per, &d_hm, &d_pgrid, &d_pG, &d_pmaps};
    if (opt.per_orient) TRY(dalloc(&d_per, (size_t)n_items * n_orient, t->st));
    if (opt.hmaps || opt.prop) TRY(dalloc(&d_hm, (size_t)n_items * PSB_PH * PSB_PH, t->st));
    float* d_feat = nullptr;   // item features of every orientation of every item [n_items][24][64]
    struct FeatCleanup {
        psb_tray* t;
        float** f;
        ~FeatCleanup() { dfree(*f, t->st); }
    } feat_cleanup{t, &d_feat};
    const int kChunk = 32;      // items per batched item-branch pass
    if (opt.prop) {
        TRY(opt.prop->ensure(n_orient * std::min(kChunk, n_items), 1));
        TRY(dalloc(&d_feat, (size_t)n_items * n_orient * 64, t->st));
        TRY(dalloc(&d_pgrid, (size_t)n_items * PSB_PG3, t->st));
        TRY(dalloc(&d_pG, (size_t)n_items * 3, t->st));
        TRY(dalloc(&d_pmaps, (size_t)n_orient * 6, t->st));
        CK(cudaMemsetAsync(d_pgrid, 0, sizeof(float) * n_items * PSB_PG3, t->st));
        std::vector<int> G(3 * (size_t)n_items);
        for (int it = 0; it < n_items; ++it) {
            const ItemInfo& inf = t->staged[it];
            const int sc = std::max(1, (std::max(inf.dims[0], std::max(inf.dims[1], inf.dims[2])) + PSB_PG - 1) / PSB_PG);
            for (int a = 0; a < 3; ++a) G[3 * it + a] = (inf.dims[a] + sc - 1) / sc;
            const int nr = (int)inf.runs[2].size();
            if (nr > 0)
                pdl(k_base_grid_runs, (nr + 255) / 256, 256, 0, t->st)(t->sdev[it].runs[2], nr, sc,
                                                                      d_pgrid + (size_t)it * PSB_PG3);
            CKL();
        }
        CK(cudaMemcpyAsync(d_pG, G.data(), sizeof(int) * G.size(), cudaMemcpyHostToDevice, t->st));
        CK(cudaMemcpyAsync(d_pmaps, orient_maps, sizeof(int) * 6 * n_orient, cudaMemcpyHostToDevice, t->st));
        CK(cudaMemsetAsync(opt.prop->stats, 0, sizeof(int) * 2, t->st));
        // the item branch does not depend on the tray: all items, in chunks
        psb_proposal* pr = opt.prop;
        for (int i0 = 0; i0 < n_items; i0 += kChunk) {
            const int m = std::min(kChunk, n_items - i0);
            {
                PROF("k_prop_inputs", t->st);
                pdl(k_orient_grids, dim3(PSB_PG3 / 256, n_orient, m), 256, 0, t->st)(
                    d_pgrid + (size_t)i0 * PSB_PG3, d_pG + 3 * i0, d_pmaps, n_orient, pr->a0);
            }
            CKL();
            TRY(pr->item_features(pr->a0, m, n_orient, t->st));
            CK(cudaMemcpyAsync(d_feat + (size_t)i0 * n_orient * 64, pr->f1, sizeof(float) * m * n_orient * 64,
                               cudaMemcpyDeviceToDevice, t->st));
        }
    }
    CK(cudaStreamSynchronize(t->st));
    // While no item is placed yet and ids start at 1, the next placement writes
    // distance sources (voxels == 1); the host waits on those few items and
    // queues the gated distance rebuild.  After that ids are >= 2, the
    // distance field is final and the rest of the run is queued without waits.
    bool first_pending = (id_offset == 0);
    if (filt) TRY(t->tray_bits());
    // The filter rules translations out only where occupied cells block
    // them: while the tray's cells plus every item searched so far (placed
    // or not: an upper bound of the occupancy) fill less than a quarter of
    // the tray it rarely skips anything and only costs its kernels, so it
    // starts after that.  Its results are exact either way.
    size_t occ_est = t->occ;
    std::vector<OrientDesc> host_ods(n_orient);
    for (int it = 0; it < n_items; ++it) {
        if (opt.feed && it == opt.feed_at) {
            // the rest of the items, staged by the caller while the first
            // part was searched: uploaded on the copy stream, which the
            // loop's stream then waits for
            TRY(opt.feed());
            TRY(describe_range(opt.feed_at, n_items, t->st_copy));
            CK(cudaEventRecord(t->ev_copy, t->st_copy));
            CK(cudaStreamWaitEvent(t->st, t->ev_copy, 0));
        }
        OrientDesc* d_odb = t->d_od_all + (size_t)it * n_orient;
        for (int o = 0; o < n_orient; ++o) host_ods[o] = all[(size_t)it * n_orient + o];
        // with the filter, k_cand_prep fills the error bounds (k_prep's work)
        const bool filter_now = filt && occ_est * 4 >= t->V;
        const bool fold_prep = filter_now && !opt.prop && !d_hm;
        if (!fold_prep) {
            pdl(k_prep, (n_orient + 63) / 64, 64, 0, t->st)(d_odb, n_orient, t->d_ps);
            CKL();
        }
        if (d_hm) {
            pdl(k_height_map, PSB_PH * PSB_PH, 256, 0, t->st)(t->d_tray, t->nx, t->ny, t->nz,
                                                             d_hm + (size_t)it * PSB_PH * PSB_PH);
            CKL();
        }
        if (opt.prop) {
            psb_proposal* pr = opt.prop;
            {
                PROF("k_prop_head", t->st);
                pdl(k_prop_tray_feat, 64, 256, 0, t->st)(d_hm + (size_t)it * PSB_PH * PSB_PH, pr->P16 + kProp.f2.w,
                                                        pr->P + kProp.f2.b, pr->t);
                CKL();
                pdl(k_prop_item_head, n_orient, 64, 0, t->st)(d_feat + (size_t)it * n_orient * 64, pr->t,
                                                             pr->P16 + kProp.h1.w, pr->P + kProp.h1.b,
                                                             pr->P16 + kProp.h2.w, pr->P + kProp.h2.b, pr->logit);
            }
            CKL();
            {
                PROF("k_gate", t->st);
                pdl(k_gate<OrientDesc>, 1, 32, 0, t->st)(pr->logit, d_odb, n_orient, opt.topk, opt.margin, pr->stats);
            }
            CKL();
        }
        std::vector<OrientDesc> hb(allb.begin() + (size_t)it * 6, allb.begin() + (size_t)(it + 1) * 6);
        if (filter_now) {
            t->prep_ps = fold_prep ? t->d_ps : nullptr;
            if (icols_pre) {
                const int part = (opt.feed && it >= opt.feed_at) ? 1 : 0;
                t->cur_icols = t->d_icp[part] + t->icol_off[it];
                t->cur_cstride = t->icol_stride[it];
                t->cur_ncol = t->d_icn + (size_t)it * n_orient;
            }
            const int fst = t->cand_filter(d_odb, host_ods, interlock != 0);
            t->prep_ps = nullptr;
            t->cur_icols = nullptr;
            t->cur_ncol = nullptr;
            TRY(fst);
        }
        occ_est += (size_t)t->staged[it].nvox;
        ShardRecord* rec = opt.world > 1 || opt.d_local ? (ShardRecord*)opt.d_local : nullptr;
        // the decision below may be fused into the search's last launch
        t->decide = DecideArgs{t->d_ls, t->d_dec + it, t->d_err, rec};
        t->fused = false;
        const int sst = t->search_async(d_odb, host_ods, mode, interlock != 0, t->d_res, true,
                                        t->d_base_all + (size_t)it * 6, &hb);
        t->cand_active = t->direct_active = t->late_active = t->pending_apply = false;
        t->decide = DecideArgs{nullptr, nullptr, nullptr, nullptr};
        TRY(sst);
        if (d_per)
            CK(cudaMemcpyAsync(d_per + (size_t)it * n_orient, t->d_res, sizeof(ResultDev) * n_orient,
                               cudaMemcpyDeviceToDevice, t->st));
        if (!t->fused) {
            pdl(k_decide, 1, 32, 0, t->st)(d_odb, t->d_res, n_orient, t->d_ls, t->d_dec + it, t->d_err, rec);
            CKL();
        }
        t->fused = false;
        if (rec) {
            // the exchange queues the gathering of every rank's record on the
            // tray's stream; the merge then decides for all ranks alike
            if (opt.exchange) {
                if (opt.exchange(opt.ctx) != 0) return fail(PSB_ERR_STATE, "decision exchange failed at item %d", it);
            } else {
                CK(cudaMemcpyAsync(opt.d_all, opt.d_local, sizeof(ShardRecord), cudaMemcpyDeviceToDevice, t->st));
            }
            pdl(k_decide_merge, 1, 1, 0, t->st)((const ShardRecord*)opt.d_all, opt.world, t->d_ls, t->d_dec + it);
            CKL();
        }
        {
            PROF("k_place", t->st);
            pdl(k_place_item, 1, 1024, 0, t->st)(d_odb, t->d_ls, t->d_tray, t->nx, t->ny, t->nz, t->d_dec + it,
                                                 t->d_pocc);
        }
        CKL();
        {
            // the placed item's columns: occupancy prefix sums and the
            // filter's free bits (gated on the placement)
            size_t box = 1;
            for (auto& o : host_ods) box = std::max(box, (size_t)o.e[0] * o.e[1]);
            PROF("k_box_refresh", t->st);
            pdl(k_box_refresh, (unsigned)((box + 7) / 8), 256, 0, t->st)(t->d_tray, t->d_pocc, filt ? t->d_tbits : nullptr,
                                                                         t->tq, t->nx, t->ny, t->nz, t->d_ls, d_odb);
        }
        CKL();
        {
            int slabs = 1;
            for (auto& o : host_ods) slabs = std::max(slabs, o.e[0]);
            TRY(t->rebuild_occ_gated(slabs));
        }
        if (first_pending) {
            TRY(t->rebuild_phi_gated());
            LoopState h;
            CK(cudaMemcpyAsync(&h, t->d_ls, sizeof(h), cudaMemcpyDeviceToHost, t->st));
            CK(cudaStreamSynchronize(t->st));
            if (h.placed > 0) first_pending = false;
        }
    }
    std::vector<DecisionDev> dec(n_items);
    LoopState h;
    CK(cudaMemcpyAsync(dec.data(), t->d_dec, sizeof(DecisionDev) * n_items, cudaMemcpyDeviceToHost, t->st));
    CK(cudaMemcpyAsync(&h, t->d_ls, sizeof(h), cudaMemcpyDeviceToHost, t->st));
    std::vector<ResultDev> per;
    if (d_per) {
        per.resize((size_t)n_items * n_orient);
        CK(cudaMemcpyAsync(per.data(), d_per, sizeof(ResultDev) * per.size(), cudaMemcpyDeviceToHost, t->st));
    }
    if (opt.hmaps)
        CK(cudaMemcpyAsync(opt.hmaps, d_hm, sizeof(float) * n_items * PSB_PH * PSB_PH, cudaMemcpyDeviceToHost,
                           t->st));
    int gst[2] = {0, 0};
    if (opt.prop) CK(cudaMemcpyAsync(gst, opt.prop->stats, sizeof(gst), cudaMemcpyDeviceToHost, t->st));
    CK(cudaStreamSynchronize(t->st));
    if (opt.gate_stats) { opt.gate_stats[0] = gst[0]; opt.gate_stats[1] = gst[1]; }
    for (size_t i = 0; i < per.size(); ++i) {
        const int o = (int)(i % n_orient);
        to_result(per[i], o, &opt.per_orient[i]);
        if (all[i].skip) opt.per_orient[i].diag |= 0x200u;
    }
    for (int it = 0; it < n_items; ++it) {
        psb_result r;
        r.x = dec[it].x; r.y = dec[it].y; r.z = dec[it].z;
        r.found = dec[it].found;
        r.score = dec[it].score;
        r.orientation = dec[it].orientation;
        r.diag = dec[it].diag;
        r.n_candidates = dec[it].ncand;
        r.err_ratio = dec[it].err_ratio;
        out_placements[it] = r;
        if (r.found) t->occ += (size_t)t->staged[it].nvox;   // a placement writes every item voxel
    }
    if (h.err & 1u) return fail(PSB_ERR_LIMIT, "flood fill union-find hit its iteration limit");
    if (h.err & 2u) return fail(PSB_ERR_LIMIT, "tie-guard candidates exceeded the capacity %d", kCandCap);
    if (h.err & 4u)
        return fail(PSB_ERR_OVERLAP, "(place_in_tray): a searched position overlapped the tray on exact re-check");
    // host copies of the distance statistics for later synchronous searches
    PhiStats ps;
    CK(cudaMemcpy(&ps, t->d_ps, sizeof(ps), cudaMemcpyDeviceToHost));
    t->phi_mean = ps.mean;
    t->phi_norm = ps.norm;
    t->phi_maxabs = ps.maxabs;
    if (final_tray) TRY(psb_tray_get(t, final_tray, nullptr));
    return PSB_OK;
}

}  // namespace

extern "C" {

int psb_pack(psb_tray* t, const int32_t* const* items, const int32_t* dims, int n_items, const int32_t* orient_maps,
             int n_orient, int interlock, int32_t id_offset, psb_result* out_placements, int32_t* final_tray) {
    NvtxRange nvtx_range("psb_pack");
    const int first = kStreamFirst;
    if (!g_stream_stage || n_items < 2 * first || !t || !items || !dims || !t->ready) {
        TRY(psb_pack_stage(t, items, dims, n_items));
        return psb_pack_staged(t, orient_maps, n_orient, interlock, id_offset, out_placements, final_tray);
    }
    // Staged in two parts: the first items are analysed and uploaded before
    // the loop starts, the rest is analysed on the host cores while the
    // first part is searched and uploaded on the copy stream when the loop
    // reaches it.  Every item is checked before anything is staged.
    CK(cudaSetDevice(t->dev));
    t->staged.clear();
    t->sdev.clear();
    TRY(stage_check(items, dims, n_items));
    t->staged.resize(n_items);
    t->sdev.resize(n_items);
    if (!t->st_copy) CK(cudaStreamCreateWithFlags(&t->st_copy, cudaStreamNonBlocking));
    if (!t->ev_copy) CK(cudaEventCreateWithFlags(&t->ev_copy, cudaEventDisableTiming));
    stage_analyse(t, items, dims, 0, first);
    TRY(stage_upload(t, items, 0, first, 0, t->st));
    std::thread rest([=] { stage_analyse(t, items, dims, first, n_items); });
    struct Join {
        std::thread& th;
        ~Join() {
            if (th.joinable()) th.join();
        }
    } join{rest};
    PackOpts o;
    o.feed_at = first;
    o.feed = [&]() -> int {
        rest.join();
        return stage_upload(t, items, first, n_items, 1, t->st_copy);
    };
    return pack_staged_impl(t, orient_maps, n_orient, interlock, id_offset, out_placements, final_tray, o);
}

int psb_pack_many(int n_trays, const int32_t* tray_dims, const int32_t* const* items, const int32_t* item_dims,
                  const int32_t* items_per_tray, const int32_t* orient_maps, int n_orient, int interlock,
                  int concurrency, psb_result* out_placements, int32_t* const* final_trays) {
    NvtxRange nvtx_range("psb_pack_many");
    if (n_trays < 0 || !tray_dims || !items_per_tray || !orient_maps || !out_placements)
        return fail(PSB_ERR_ARG, "pack_many: null pointer");
    TRY(ensure_device());
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::vector<size_t> first(n_trays + 1, 0);
    for (int i = 0; i < n_trays; ++i) {
        if (items_per_tray[i] < 0) return fail(PSB_ERR_ARG, "pack_many: tray %d has a negative item count", i);
        first[i + 1] = first[i] + (size_t)items_per_tray[i];
    }
    const int workers = std::max(1, std::min(concurrency > 0 ? concurrency : 8, std::max(1, n_trays)));
    std::atomic<int> next(0);
    std::vector<int> status(n_trays, PSB_OK);
    std::vector<std::string> messages(n_trays);
    auto work = [&]() {
        cudaSetDevice(dev);
        for (int i = next.fetch_add(1); i < n_trays; i = next.fetch_add(1)) {
            const int nx = tray_dims[3 * i], ny = tray_dims[3 * i + 1], nz = tray_dims[3 * i + 2];
            psb_tray* t = nullptr;
            int st = psb_tray_create(nx, ny, nz, &t);
            std::vector<int32_t> empty;
            if (st == PSB_OK) {
                empty.assign((size_t)nx * ny * nz, 0);
                st = psb_tray_set(t, empty.data(), nullptr);
            }
            if (st == PSB_OK)
                st = psb_pack(t, items + first[i], item_dims + 3 * first[i], items_per_tray[i], orient_maps, n_orient,
                              interlock, 0, out_placements + first[i], final_trays ? final_trays[i] : nullptr);
            if (st != PSB_OK) {
                status[i] = st;
                messages[i] = g_err;
            }
            if (t) psb_tray_destroy(t);
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < workers; ++w) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    for (int i = 0; i < n_trays; ++i)
        if (status[i] != PSB_OK) return fail(status[i], "pack_many: tray %d: %s", i, messages[i].c_str());
    return PSB_OK;
}

// ---------------------------------------------------------------------------
// learned orientation proposal
// ---------------------------------------------------------------------------
int psb_prop_create(psb_proposal** out) {
    if (!out) return fail(PSB_ERR_ARG, "null pointer");
    std::unique_ptr<psb_proposal> p(new psb_proposal());
    TRY(p->init());
    *out = p.release();
    return PSB_OK;
}

int psb_prop_destroy(psb_proposal* p) {
    delete p;
    return PSB_OK;
}

int psb_prop_num_params(size_t* n) {
    if (!n) return fail(PSB_ERR_ARG, "null pointer");
    *n = kProp.n;
    return PSB_OK;
}

int psb_prop_set_params(psb_proposal* p, const float* params, size_t n) {
    if (!p || !params) return fail(PSB_ERR_ARG, "null pointer");
    if (n != kProp.n) return fail(PSB_ERR_ARG, "expected %zu parameters, got %zu", kProp.n, n);
    CK(cudaSetDevice(p->dev));
    std::vector<uint16_t> h16(n);
    for (size_t i = 0; i < n; ++i) h16[i] = bf16_bits(params[i]);
    CK(cudaMemcpy(p->P, params, sizeof(float) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(p->P16, h16.data(), sizeof(uint16_t) * n, cudaMemcpyHostToDevice));
    CK(cudaMemset(p->M, 0, sizeof(float) * n));
    CK(cudaMemset(p->V, 0, sizeof(float) * n));
    p->step = 0;
    return PSB_OK;
}

int psb_prop_get_params(psb_proposal* p, float* params, size_t n) {
    if (!p || !params) return fail(PSB_ERR_ARG, "null pointer");
    if (n != kProp.n) return fail(PSB_ERR_ARG, "expected %zu parameters, got %zu", kProp.n, n);
    CK(cudaSetDevice(p->dev));
    CK(cudaStreamSynchronize(p->st));
    CK(cudaMemcpy(params, p->P, sizeof(float) * n, cudaMemcpyDeviceToHost));
    return PSB_OK;
}

int psb_prop_get_grads(psb_proposal* p, float* grads, size_t n) {
    if (!p || !grads) return fail(PSB_ERR_ARG, "null pointer");
    if (n != kProp.n) return fail(PSB_ERR_ARG, "expected %zu parameters, got %zu", kProp.n, n);
    CK(cudaSetDevice(p->dev));
    CK(cudaStreamSynchronize(p->st));
    CK(cudaMemcpy(grads, p->G, sizeof(float) * n, cudaMemcpyDeviceToHost));
    return PSB_OK;
}

int psb_prop_forward_backward(psb_proposal* p, const float* d_grids, const float* d_hmaps, const float* d_mask,
                              const float* d_target, int n_items, float* d_logits, float* h_loss) {
    if (!p || !d_grids || !d_hmaps || n_items <= 0) return fail(PSB_ERR_ARG, "null pointer or empty batch");
    if (d_target && !d_mask) return fail(PSB_ERR_ARG, "a target needs a mask");
    CK(cudaSetDevice(p->dev));
    const int S = n_items * PSB_PNO;
    TRY(p->ensure(S, n_items));
    TRY(p->forward(d_grids, d_hmaps, n_items, PSB_PNO, p->st));
    if (d_target) TRY(p->backward(d_grids, d_hmaps, d_target, d_mask, n_items, PSB_PNO, p->st));
    if (d_logits) CK(cudaMemcpyAsync(d_logits, p->logit, sizeof(float) * S, cudaMemcpyDeviceToDevice, p->st));
    if (h_loss) {
        float l = 0.f;
        if (d_target) CK(cudaMemcpyAsync(&l, p->loss, sizeof(float), cudaMemcpyDeviceToHost, p->st));
        CK(cudaStreamSynchronize(p->st));
        *h_loss = l;
    }
    CK(cudaStreamSynchronize(p->st));
    return PSB_OK;
}

int psb_prop_adam_step(psb_proposal* p, float lr, float beta1, float beta2, float eps) {
    if (!p) return fail(PSB_ERR_ARG, "null pointer");
    CK(cudaSetDevice(p->dev));
    p->step += 1;
    const float c1 = 1.f - std::pow(beta1, (float)p->step), c2 = 1.f - std::pow(beta2, (float)p->step);
    const long long n = (long long)kProp.n;
    pdl(k_adam, (unsigned)((n + 255) / 256), 256, 0, p->st)(p->P, p->G, p->M, p->V, p->P16, p->isw, n, lr, beta1,
                                                            beta2, eps, c1, c2);
    CKL();
    CK(cudaStreamSynchronize(p->st));
    return PSB_OK;
}

int psb_prop_item_grids(const int32_t* const* items, const int32_t* dims, int n_items, const int32_t* orient_maps,
                        int n_orient, float* d_out) {
    if (!items || !dims || !orient_maps || !d_out || n_items < 0 || n_orient <= 0)
        return fail(PSB_ERR_ARG, "null pointer or bad count");
    TRY(ensure_device());
    if (n_items == 0) return PSB_OK;
    std::vector<ItemInfo> infos(n_items);
    std::vector<int> G(3 * (size_t)n_items), S(n_items);
    size_t totv = 0;
    for (int i = 0; i < n_items; ++i) {
        const int ex = dims[3 * i], ey = dims[3 * i + 1], ez = dims[3 * i + 2];
        if (!items[i] || ex <= 0 || ey <= 0 || ez <= 0) return fail(PSB_ERR_ARG, "item %d: bad array", i);
        analyse_item(items[i], ex, ey, ez, &infos[i]);
        S[i] = std::max(1, (std::max(ex, std::max(ey, ez)) + PSB_PG - 1) / PSB_PG);
        for (int a = 0; a < 3; ++a) G[3 * i + a] = (infos[i].dims[a] + S[i] - 1) / S[i];
        totv += infos[i].vox.size();
    }
    float* base = nullptr;
    int4* vox = nullptr;
    int *dG = nullptr, *dm = nullptr;
    TRY(dalloc(&base, (size_t)n_items * PSB_PG3));
    TRY(dalloc(&vox, std::max<size_t>(totv, 1)));
    TRY(dalloc(&dG, G.size()));
    TRY(dalloc(&dm, (size_t)6 * n_orient));
    int rc = PSB_OK;
    do {
        if (cudaMemset(base, 0, sizeof(float) * n_items * PSB_PG3) != cudaSuccess) { rc = fail(PSB_ERR_CUDA, "memset"); break; }
        size_t off = 0;
        for (int i = 0; i < n_items && rc == PSB_OK; ++i) {
            const size_t nv = infos[i].vox.size();
            if (nv == 0) continue;
            if (cudaMemcpy(vox + off, infos[i].vox.data(), sizeof(int4) * nv, cudaMemcpyHostToDevice) != cudaSuccess)
                rc = fail(PSB_ERR_CUDA, "copy");
            k_base_grid<<<(unsigned)((nv + 255) / 256), 256>>>(vox + off, (int)nv, S[i], base + (size_t)i * PSB_PG3);
            off += nv;
        }
        if (rc != PSB_OK) break;
        if (cudaMemcpy(dG, G.data(), sizeof(int) * G.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(dm, orient_maps, sizeof(int) * 6 * n_orient, cudaMemcpyHostToDevice) != cudaSuccess) {
            rc = fail(PSB_ERR_CUDA, "copy");
            break;
        }
        k_orient_grids<<<dim3(PSB_PG3 / 256, n_orient, n_items), 256>>>(base, dG, dm, n_orient, d_out);
        if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess)
            rc = fail(PSB_ERR_CUDA, "item grids: %s", cudaGetErrorString(cudaGetLastError()));
    } while (0);
    dfree(base); dfree(vox); dfree(dG); dfree(dm);
    return rc;
}

int psb_height_map(const int32_t* d_tray, int nx, int ny, int nz, float* d_out) {
    if (!d_tray || !d_out || nx <= 0 || ny <= 0 || nz <= 0) return fail(PSB_ERR_ARG, "bad arguments");
    TRY(ensure_device());
    k_height_map<<<PSB_PH * PSB_PH, 256>>>(d_tray, nx, ny, nz, d_out);
    CKL();
    CK(cudaDeviceSynchronize());
    return PSB_OK;
}

// ---------------------------------------------------------------------------
// mesh voxelizer (voxelize_stl: bindings.cpp:285-302, packing.cpp:540-588)
// ---------------------------------------------------------------------------
int psb_voxelize_mesh(const float* tris, int ntri, int resolution, int32_t* out, int32_t* dims_out) {
    NvtxRange nvtx_range("psb_voxelize_mesh");
    if (!tris || !out || !dims_out || ntri <= 0 || resolution <= 0)
        return fail(PSB_ERR_ARG, "voxelize: null pointer, no triangles or bad resolution");
    TRY(ensure_device());
    // mergeVerticesExact (LibSL Mesh.cpp:350-392): the new index of a vertex
    // is the rank of its position in lexicographic order
    const int nv = 3 * ntri;
    std::vector<std::pair<std::array<float, 3>, int>> all(nv);
    for (int v = 0; v < nv; ++v) all[v] = {{tris[3 * v], tris[3 * v + 1], tris[3 * v + 2]}, v};
    std::sort(all.begin(), all.end());
    std::vector<int> newidx(nv);
    std::vector<std::array<float, 3>> pos;
    for (int v = 0; v < nv; ++v) {
        if (pos.empty() || all[v].first != pos.back()) pos.push_back(all[v].first);
        newidx[all[v].second] = (int)pos.size() - 1;
    }
    // box transform in float, composed and applied as LibSL's Matrix4x4 does
    // (products accumulated from zero in index order; no fused multiply-add)
    float lo[3], hi[3], ext[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = hi[a] = pos[0][a];
        for (auto& p : pos) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
        ext[a] = hi[a] - lo[a];
    }
    const float emax = std::max(ext[0], std::max(ext[1], ext[2]));
    if (!(emax > 0.f)) return fail(PSB_ERR_ARG, "voxelize: the mesh has no extent");
    typedef std::array<std::array<float, 4>, 4> M4;
    auto ident = []() { M4 m{}; for (int i = 0; i < 4; ++i) m[i][i] = 1.f; return m; };
    auto scale = [&](float s) { M4 m = ident(); for (int i = 0; i < 3; ++i) m[i][i] = s; return m; };
    auto trans = [&](const float* t) { M4 m = ident(); for (int i = 0; i < 3; ++i) m[i][3] = t[i]; return m; };
    auto mul = [](const M4& a, const M4& b) {
        M4 r{};
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) {
                volatile float acc = 0.f;
                for (int k = 0; k < 4; ++k) {
                    volatile float prod = a[i][k] * b[k][j];
                    acc = acc + prod;
                }
                r[i][j] = acc;
            }
        return r;
    };
    const float factor = 0.95f;
    float t1[3], t2[3];
    for (int a = 0; a < 3; ++a) {
        volatile float h = (1.f - factor) * 0.5f;
        t1[a] = h * ext[a];
        t2[a] = -lo[a];
    }
    volatile float inv = 1.f / emax;
    const M4 box = mul(mul(mul(mul(scale((float)resolution * (float)PSB_FP_SCALE), scale(inv)), trans(t1)),
                           scale(factor)),
                       trans(t2));
    const float top = (float)resolution * (float)PSB_FP_SCALE - 1.f;
    std::vector<int> pts(3 * pos.size());
    for (size_t p = 0; p < pos.size(); ++p)
        for (int i = 0; i < 3; ++i) {
            volatile float acc = 0.f;
            for (int k = 0; k < 3; ++k) {
                volatile float prod = box[i][k] * pos[p][k];
                acc = acc + prod;
            }
            acc = acc + box[i][3];
            float r = ::roundf(acc);
            r = std::min(std::max(r, 0.f), top);
            pts[3 * p + i] = (int)r;
        }
    int dims[3];
    for (int a = 0; a < 3; ++a) {
        volatile float q = ext[a] / emax;
        volatile float d = q * (float)resolution;
        dims[a] = (int)(unsigned int)d;
    }
    const size_t V = (size_t)dims[0] * dims[1] * dims[2];
    std::vector<int> tri(3 * (size_t)ntri);
    for (int v = 0; v < nv; ++v) tri[v] = newidx[v];
    std::vector<unsigned int> hv(V, 0u);
    if (V > 0) {
        int *dp = nullptr, *dt = nullptr;
        unsigned int* dv = nullptr;
        TRY(dalloc(&dp, pts.size()));
        TRY(dalloc(&dt, tri.size()));
        TRY(dalloc(&dv, V));
        int rc = PSB_OK;
        if (cudaMemcpy(dp, pts.data(), sizeof(int) * pts.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(dt, tri.data(), sizeof(int) * tri.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(dv, 0, sizeof(unsigned int) * V) != cudaSuccess) {
            rc = fail(PSB_ERR_CUDA, "voxelize: upload failed");
        } else {
            const long long warps = 3LL * ntri;
            PROF("k_voxel_raster", nullptr);
            k_voxel_raster<<<(unsigned)((warps + 7) / 8), 256>>>(dp, dt, ntri, dims[0], dims[1], dims[2], dv);
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaMemcpy(hv.data(), dv, sizeof(unsigned int) * V, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) rc = fail(PSB_ERR_CUDA, "voxelize: %s", cudaGetErrorString(e));
        }
        dfree(dp); dfree(dt); dfree(dv);
        TRY(rc);
    }
    // occupied = any axis bit; then the tight bounding box (make_voxel_grid_tight)
    int lo3[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi3[3] = {-1, -1, -1};
    for (int i = 0; i < dims[0]; ++i)
        for (int j = 0; j < dims[1]; ++j)
            for (int k = 0; k < dims[2]; ++k)
                if (hv[((size_t)i * dims[1] + j) * dims[2] + k]) {
                    const int c[3] = {i, j, k};
                    for (int a = 0; a < 3; ++a) { lo3[a] = std::min(lo3[a], c[a]); hi3[a] = std::max(hi3[a], c[a]); }
                }
    if (hi3[0] < 0) {
        dims_out[0] = dims_out[1] = dims_out[2] = 0;
        return PSB_OK;
    }
    const int td[3] = {hi3[0] - lo3[0] + 1, hi3[1] - lo3[1] + 1, hi3[2] - lo3[2] + 1};
    for (int i = 0; i < td[0]; ++i)
        for (int j = 0; j < td[1]; ++j)
            for (int k = 0; k < td[2]; ++k)
                out[((size_t)i * td[1] + j) * td[2] + k] =
                    hv[((size_t)(i + lo3[0]) * dims[1] + (j + lo3[1])) * dims[2] + (k + lo3[2])] ? 1 : 0;
    for (int a = 0; a < 3; ++a) dims_out[a] = td[a];
    return PSB_OK;
}

int psb_set_fast_fft(int on) {
    g_fast_fft = on != 0;
    return PSB_OK;
}

int psb_set_share_flips(int on) {
    g_share_flips = on != 0;
    return PSB_OK;
}

int psb_set_cand_filter(int on) {
    g_cand_filter = on != 0;
    return PSB_OK;
}

int psb_set_direct_max(int n) {
    if (n < 0 || n > kCandCap) return fail(PSB_ERR_ARG, "direct limit must be in [0, %d]", kCandCap);
    g_direct_max = n;
    return PSB_OK;
}

int psb_set_filter_cut(int pct) {
    if (pct < 0 || pct > 100) return fail(PSB_ERR_ARG, "filter cut-off must be a percentage in [0, 100]");
    g_filter_cut = pct;
    return PSB_OK;
}

int psb_set_late_direct_max(int n) {
    if (n < 0) return fail(PSB_ERR_ARG, "late direct limit must be >= 0");
    g_late_max = std::min(n, kCandCap);   // every ok cell of such an orientation is a candidate
    return PSB_OK;
}

int psb_set_uf_limit(int n) {
    g_uf_limit = n > 0 ? n : PSB_UF_LIMIT;
    return PSB_OK;
}

int psb_debug_fail_alloc(int n) {
    g_fail_alloc.store(n > 0 ? n : 0);
    return PSB_OK;
}

int psb_debug_live_allocs(long long* n) {
    if (!n) return fail(PSB_ERR_ARG, "null output");
    *n = g_live_allocs.load();
    return PSB_OK;
}

int psb_set_plane_variant(int v) {
    if (v != 2 && v != 3) return fail(PSB_ERR_ARG, "plane variant must be 2 or 3");
    g_plane_variant = v;
    return PSB_OK;
}

int psb_profile_enable(int on) {
    std::lock_guard<std::mutex> lk(g_prof.mu);
    for (auto& r : g_prof.recs) { g_prof.pool.push_back(r.a); g_prof.pool.push_back(r.b); }
    g_prof.recs.clear();
    g_prof.on = on != 0;
    return PSB_OK;
}

int psb_profile_filter(const char* names) {
    std::lock_guard<std::mutex> lk(g_prof.mu);
    g_prof.only.clear();
    if (!names) return PSB_OK;
    std::string cur;
    for (const char* c = names;; ++c) {
        if (*c == ',' || *c == 0) {
            if (!cur.empty()) g_prof.only.push_back(cur);
            cur.clear();
            if (*c == 0) break;
        } else {
            cur += *c;
        }
    }
    return PSB_OK;
}

int psb_profile_report(char* buf, size_t len) {
    if (!buf || len == 0) return fail(PSB_ERR_ARG, "null buffer");
    std::lock_guard<std::mutex> lk(g_prof.mu);
    std::map<std::string, std::pair<int, double>> agg;
    for (auto& r : g_prof.recs) {
        cudaEventSynchronize(r.b);
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) { cudaGetLastError(); continue; }
        auto& e = agg[r.name];
        e.first += 1;
        e.second += ms;
    }
    std::string out;
    for (auto& kv : agg) {
        char line[256];
        snprintf(line, sizeof(line), "%s %d %.6f\n", kv.first.c_str(), kv.second.first, kv.second.second);
        out += line;
    }
    snprintf(buf, len, "%s", out.c_str());
    return out.size() + 1 > len ? fail(PSB_ERR_ARG, "report truncated") : PSB_OK;
}

int psb_tray_fft_dims(const psb_tray* t, int* F) {
    if (!t || !F) return fail(PSB_ERR_ARG, "null pointer");
    F[0] = t->g.F[0]; F[1] = t->g.F[1]; F[2] = t->g.F[2];
    return PSB_OK;
}

int psb_tray_stream(psb_tray* t, void** stream) {
    if (!t || !stream) return fail(PSB_ERR_ARG, "null pointer");
    *stream = (void*)t->st;
    return PSB_OK;
}

int psb_tray_work(psb_tray* t, unsigned long long* out, int reset) {
    if (!t) return fail(PSB_ERR_ARG, "null pointer");
    CK(cudaSetDevice(t->dev));
    if (out) {
        CK(cudaMemcpyAsync(out, t->d_work, sizeof(unsigned long long) * 8, cudaMemcpyDeviceToHost, t->st));
        CK(cudaStreamSynchronize(t->st));
    }
    if (reset) CK(cudaMemsetAsync(t->d_work, 0, sizeof(unsigned long long) * 8, t->st));
    return PSB_OK;
}

}  // extern "C"
