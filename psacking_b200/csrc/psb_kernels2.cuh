// psb_kernels2.cuh — selection, exact tie guard, flood fill, distance field
// and placement kernels.
#pragma once
#include "psb_kernels.cuh"

#define PSB_UF_LIMIT (1 << 22)     // default bound on union-find retries / path steps

// ---------------------------------------------------------------------------
// candidate selection and the exact tie guard
// ---------------------------------------------------------------------------
struct SelectBufs {
    const uint32_t* okbits;        // free bits or reach bits, per orientation stride sBits
    long long sBits;
    const float* Dq;               // per orientation stride sD
    long long sD;
    unsigned long long* smin;      // approx min key per orientation
    int* cand;                     // per orientation stride cap
    int* ncand;                    // per orientation
    double* cscore;                // per orientation stride cap
    unsigned long long* best;      // exact best score key per orientation
    unsigned long long* bestkey;   // tie key per orientation
    unsigned int* diag;
    unsigned int* errmax;          // max |D~ - D| / delta seen by the exact re-check (float bits)
    int cap;
    unsigned long long* pmin;      // per (orientation, x plane) approx min key, stride pstride
    long long pstride;
    const int* gate;               // when set, the kernels run only if *gate != 0
    const unsigned char* okplane;  // when set, per (orientation, x plane): holds an ok cell (stride pstride)
    const int* srch;               // when set: the searched orientations (k_active_list), *nsrch of them;
    const int* nsrch;              // CTA row y takes srch[y], srch[y + gridDim.y], ...
};

__device__ __forceinline__ bool okbit(const uint32_t* bits, const ScoreParams& sp, int x, int y, int z) {
    return (bits[((size_t)x * sp.ny + y) * sp.nzw + (z >> 5)] >> (z & 31)) & 1u;
}

// ordered encoding of floats for atomicMin on unsigned int
__device__ __forceinline__ unsigned int ford_key(float v) {
    unsigned int b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ford_val(unsigned int k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

#define PSB_ZWORDS (PSB_MAX_FFT / 32)   // 32-bit words of z per row, at most

// The reference scores every cell and reduces them (compute_scores_kernel +
// argmin_reduction_kernel, fft3.cu:147-215, 527-563).  Here the minimum is
// found in two steps.  (1) Per (x plane, orientation) the minimum approximate
// score over the plane's ok cells (free or reachable) goes to pmin[o][x] and,
// by atomicMin, to the orientation minimum smin[o]: the score rises with the
// proximity at fixed z, so the plane minimum is the minimum over z of the
// score of the per-z minimum proximity.  k_plane2 / k_plane produce these for
// the free cells while they write the field; k_plane_min produces them for
// another mask (the reachable cells).  (2) k_collect_plane keeps every ok cell
// whose approximate score lies within the window smin + 2 delta of the
// orientation minimum (planes whose minimum is above the window are skipped
// without reading them); k_rescore scores those candidates exactly.

// (1) for an arbitrary ok mask.  One CTA per (x plane, orientation): thread
// (g, l) owns z = l (+128, ...) and walks rows y = g, g + 4, ... (4 row
// groups), so loads are coalesced along z, independent across rows and no
// atomics are needed; the row groups meet in shared memory.
// grid: (nx, n_orient), block PSB_PMIN_THREADS
#define PSB_PMIN_ZL 128
#define PSB_PMIN_RG 4
#define PSB_PMIN_THREADS (PSB_PMIN_ZL * PSB_PMIN_RG)
__global__ void __launch_bounds__(PSB_PMIN_THREADS)
k_plane_min(const OrientDesc* __restrict__ orients, SelectBufs sb, ScoreParams sp) {
    pdl_enter();
    if (sb.gate && !*sb.gate) return;
    const int o = blockIdx.y, x = blockIdx.x;
    const OrientDesc& od = orients[o];
    if (od.skip || x >= od.valid[0]) return;
    const int Yv = od.valid[1], Zv = od.valid[2];
    if (Yv <= 0 || Zv <= 0) return;
    const int l = threadIdx.x % PSB_PMIN_ZL, g = threadIdx.x / PSB_PMIN_ZL;
    const uint32_t* bits = sb.okbits + (size_t)o * sb.sBits + (size_t)x * sp.ny * sp.nzw;
    const float* Dq = sb.Dq + (size_t)o * sb.sD + (size_t)x * sp.ny * sp.nz;
    __shared__ unsigned int part[PSB_PMIN_RG][PSB_PMIN_ZL];
    __shared__ double red[PSB_PMIN_THREADS / 32];
    double pm = 1e300;
    for (int z0 = 0; z0 < Zv; z0 += PSB_PMIN_ZL) {
        const int z = z0 + l;
        unsigned int mk = 0xffffffffu;
        if (z < Zv) {
            const int wz = z >> 5, bz = z & 31;
            int y = g;
#pragma unroll 1
            for (; y + 3 * PSB_PMIN_RG < Yv; y += 4 * PSB_PMIN_RG) {
                uint32_t b[4];
                float d[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int yy = y + u * PSB_PMIN_RG;
                    b[u] = __ldg(&bits[(size_t)yy * sp.nzw + wz]);
                    d[u] = __ldg(&Dq[(size_t)yy * sp.nz + z]);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if ((b[u] >> bz) & 1u) mk = min(mk, ford_key(d[u]));
            }
            for (; y < Yv; y += PSB_PMIN_RG)
                if ((__ldg(&bits[(size_t)y * sp.nzw + wz]) >> bz) & 1u)
                    mk = min(mk, ford_key(__ldg(&Dq[(size_t)y * sp.nz + z])));
        }
        part[g][l] = mk;
        __syncthreads();
        if (g == 0 && z < Zv) {
#pragma unroll
            for (int r = 1; r < PSB_PMIN_RG; ++r) mk = min(mk, part[r][l]);
            if (mk != 0xffffffffu) pm = fmin(pm, ref_score(sp, od.base + (double)ford_val(mk), z));
        }
        __syncthreads();
    }
    for (int off = 16; off > 0; off >>= 1) pm = fmin(pm, __shfl_xor_sync(0xffffffffu, pm, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = pm;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 0; w < PSB_PMIN_THREADS / 32; ++w) pm = fmin(pm, red[w]);
        sb.pmin[(size_t)o * sb.pstride + x] = pm < 1e299 ? ord_key(pm) : 0xffffffffffffffffULL;
        if (pm < 1e299) atomicMin(&sb.smin[o], ord_key(pm));
    }
}

// (2) candidate collection, one CTA per (x plane, orientation), one warp per
// row y.  An FP32 per-z proximity threshold (rounded up, with slack) screens
// the cells before the double-precision score.  grid: (nx, n_orient)
__device__ __forceinline__ void k_collect_plane_body(const int o, const OrientDesc* __restrict__ orients, SelectBufs sb, ScoreParams sp) {
    if (sb.gate && !*sb.gate) return;
    const int x = blockIdx.x;
    const OrientDesc& od = orients[o];
    if (od.skip || x >= od.valid[0]) return;
    const int Yv = od.valid[1], Zv = od.valid[2];
    if (Yv <= 0 || Zv <= 0) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int nw = (Zv + 31) >> 5;
    const uint32_t* bits = sb.okbits + (size_t)o * sb.sBits + (size_t)x * sp.ny * sp.nzw;
    if (od.direct) {
        // a direct orientation (psb_filter.cuh): every ok cell is a candidate,
        // scored exactly by k_direct_score (at most the direct limit of them)
        if (sb.okplane && !sb.okplane[(size_t)o * sb.pstride + x]) return;   // no ok cell in this plane
        int* cand = sb.cand + (size_t)o * sb.cap;
        for (int y = warp; y < Yv; y += nwarp)
            for (int w = 0; w < nw; ++w) {
                const int z = w * 32 + lane;
                const bool take = z < Zv && ((bits[(size_t)y * sp.nzw + w] >> lane) & 1u);
                const unsigned int tk = __ballot_sync(0xffffffffu, take);
                if (!tk) continue;
                int slot0 = 0;
                if (lane == 0) slot0 = atomicAdd(&sb.ncand[o], __popc(tk));
                slot0 = __shfl_sync(0xffffffffu, slot0, 0);
                const int slot = slot0 + __popc(tk & ((1u << lane) - 1u));
                if (take && slot < sb.cap) cand[slot] = (int)(((size_t)x * sp.ny + y) * sp.nz + z);
            }
        return;
    }
    const unsigned long long gk = sb.smin[o];
    if (gk == 0xffffffffffffffffULL) return;  // no ok cell in any plane
    const double pm = ord_val(gk);
    const double lim = pm + 2.0 * od.delta + 1e-4 + 8.0 * (fabs(pm) + 1.0) * 2.220446049250313e-16;
    const unsigned long long pk = sb.pmin[(size_t)o * sb.pstride + x];
    if (pk == 0xffffffffffffffffULL || ord_val(pk) > lim) return;
    const float* Dq = sb.Dq + (size_t)o * sb.sD + (size_t)x * sp.ny * sp.nz;
    const double base = od.base;
    // score(D) <= lim needs D <= lim - score(0) at that z, up to roundings:
    // 1.0 of slack, then rounded up to FP32; the exact test follows
    float m[PSB_ZWORDS];
#pragma unroll
    for (int w = 0; w < PSB_ZWORDS; ++w) {
        const int z = w * 32 + lane;
        m[w] = (w < nw && z < Zv) ? __double2float_ru(lim - ref_score(sp, base, z) + 1.0) : -INFINITY;
    }
    int* cand = sb.cand + (size_t)o * sb.cap;
    double* cs = sb.cscore + (size_t)o * sb.cap;
    for (int y = warp; y < Yv; y += nwarp) {
        const uint32_t* brow = bits + (size_t)y * sp.nzw;
        const float* drow = Dq + (size_t)y * sp.nz;
#pragma unroll
        for (int w = 0; w < PSB_ZWORDS; ++w) {
            if (w < nw) {
                const int z = w * 32 + lane;
                bool take = false;
                double s = 0.0;
                if (((brow[w] >> lane) & 1u) && z < Zv) {
                    const float d = drow[z];
                    if (d <= m[w]) {
                        s = ref_score(sp, base + (double)d, z);
                        take = s <= lim;
                    }
                }
                const unsigned int tk = __ballot_sync(0xffffffffu, take);
                if (tk) {
                    int slot0 = 0;
                    if (lane == 0) slot0 = atomicAdd(&sb.ncand[o], __popc(tk));
                    slot0 = __shfl_sync(0xffffffffu, slot0, 0);
                    if (take) {
                        const int slot = slot0 + __popc(tk & ((1u << lane) - 1u));
                        if (slot < sb.cap) {
                            cand[slot] = (int)(((size_t)x * sp.ny + y) * sp.nz + z);
                            cs[slot] = s;
                        }
                    }
                }
            }
        }
    }
}

__global__ void __launch_bounds__(256)

k_collect_plane(const OrientDesc* __restrict__ orients, SelectBufs sb, ScoreParams sp) {
    pdl_enter();
    if (!sb.srch) {
        const int o = blockIdx.y;
        k_collect_plane_body(o, orients, sb, sp);
        return;
    }
    const int na = *sb.nsrch;
    for (int j = blockIdx.y; j < na; j += gridDim.y) {
        const int o = sb.srch[j];
        k_collect_plane_body(o, orients, sb, sp);
    }
}

// per-orientation selection state back to "nothing seen" (the gated second
// round of the lazy interlocking search)
__global__ void k_sel_reset(SelectBufs sb, int n) {
    pdl_enter();
    if (sb.gate && !*sb.gate) return;
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < n; o += gridDim.x * blockDim.x) {
        sb.smin[o] = 0xffffffffffffffffULL;
        sb.best[o] = 0xffffffffffffffffULL;
        sb.bestkey[o] = 0xffffffffffffffffULL;
        sb.ncand[o] = 0;
    }
}

// exact score of every candidate.  Regime (a): the FP32 value rounds to the
// exact integer.  Regime (b): direct integer sums over the item's z-runs
// (proximity and collision, from the per-column prefix sums pphi / pocc of
// the distance field and the occupancy), the FP64 guard.
// grid: (blocks, n_orient)
__device__ __forceinline__ void k_rescore_body(const int o, const OrientDesc* __restrict__ orients, SelectBufs sb, ScoreParams sp, const int32_t* __restrict__ pocc,
          const int32_t* __restrict__ pphi) {
    if (sb.gate && !*sb.gate) return;
    const OrientDesc& od = orients[o];
    if (od.skip || od.direct) return;   // direct orientations: k_direct_score
    const int n = min(sb.ncand[o], sb.cap);
    const int* cand = sb.cand + (size_t)o * sb.cap;
    double* cs = sb.cscore + (size_t)o * sb.cap;
    const float* Dq = sb.Dq + (size_t)o * sb.sD;
    const double smin = ord_val(sb.smin[o]);
    const double glim = smin + 2.0 * od.delta + 8.0 * (fabs(smin) + 1.0) * 2.220446049250313e-16;
    if (!od.exact) {
        // regime (a): the FP32 value rounds to the exact integer; one thread per candidate
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
            if (cs[c] > glim) { cs[c] = 1e300; continue; }
            const int t = cand[c];
            const double s = ref_score(sp, od.base + (double)rintf(Dq[t]), t % sp.nz);
            cs[c] = s;
            atomicMin(&sb.best[o], ord_key(s));
        }
        return;
    }
    // regime (b): one CTA per candidate sums the item's runs exactly
    __shared__ long long red_acc[8], red_coll[8];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int nz1 = sp.nz + 1;
    for (int c = blockIdx.x; c < n; c += gridDim.x) {
        if (cs[c] > glim) {  // outside the orientation's window: provably not the minimum
            if (tid == 0) cs[c] = 1e300;
            continue;
        }
        const int t = cand[c];
        const int z = t % sp.nz;
        const int y = (t / sp.nz) % sp.ny;
        const int x = t / (sp.nz * sp.ny);
        long long acc = 0, coll = 0;
        const int nr = od.nruns;
#pragma unroll 4
        for (int r = tid; r < nr; r += 256) {
            const int4 q = __ldg(&od.runs[r]);
            int a, b, c0, c1;
            orient_run(od, q, &a, &b, &c0, &c1);
            const size_t g = ((size_t)(x + a) * sp.ny + (y + b)) * nz1 + z;
            acc += (long long)q.w * (__ldg(&pphi[g + c1 + 1]) - __ldg(&pphi[g + c0]));
            coll += (long long)q.w * (__ldg(&pocc[g + c1 + 1]) - __ldg(&pocc[g + c0]));
        }
        for (int off = 16; off > 0; off >>= 1) {
            acc += __shfl_xor_sync(0xffffffffu, acc, off);
            coll += __shfl_xor_sync(0xffffffffu, coll, off);
        }
        if (lane == 0) { red_acc[wid] = acc; red_coll[wid] = coll; }
        __syncthreads();
        if (tid == 0) {
            long long A = 0, Cc = 0;
            for (int w = 0; w < 8; ++w) { A += red_acc[w]; Cc += red_coll[w]; }
            const double D = (double)A;
            const bool valid = Cc == 0;
            const double err = fabs(D - (od.base + (double)Dq[t]));
            if (!valid) atomicOr(&sb.diag[o], 4u);
            if (err > od.delta) atomicOr(&sb.diag[o], 8u);
            atomicMax(&sb.errmax[o], __float_as_uint((float)(err / od.delta)));
            const double s = valid ? ref_score(sp, D, z) : 1e300;
            cs[c] = s;
            if (valid) atomicMin(&sb.best[o], ord_key(s));
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256)

k_rescore(const OrientDesc* __restrict__ orients, SelectBufs sb, ScoreParams sp, const int32_t* __restrict__ pocc,
          const int32_t* __restrict__ pphi) {
    pdl_enter();
    if (!sb.srch) {
        const int o = blockIdx.y;
        k_rescore_body(o, orients, sb, sp, pocc, pphi);
        return;
    }
    const int na = *sb.nsrch;
    for (int j = blockIdx.y; j < na; j += gridDim.y) {
        const int o = sb.srch[j];
        k_rescore_body(o, orients, sb, sp, pocc, pphi);
        __syncthreads();   // shared memory is reused by the next orientation
    }
}

__device__ __forceinline__ unsigned int tie_key(int mode, int idx) {
    if (mode == 0) return (unsigned int)idx;
    return ((unsigned int)idx & ~255u) | (__brev((unsigned int)idx & 255u) >> 24);
}
__device__ __forceinline__ int untie_key(int mode, unsigned int key) {
    if (mode == 0) return (int)key;
    return (int)((key & ~255u) | (__brev(key & 255u) >> 24));
}

__device__ __forceinline__ void k_tiebreak_body(const int o, const OrientDesc* __restrict__ orients, SelectBufs sb, ScoreParams sp) {
    if (sb.gate && !*sb.gate) return;
    if (orients[o].skip) return;
    const int n = min(sb.ncand[o], sb.cap);
    const unsigned long long b = sb.best[o];
    const int* cand = sb.cand + (size_t)o * sb.cap;
    const double* cs = sb.cscore + (size_t)o * sb.cap;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        if (cs[c] < 1e299 && ord_key(cs[c]) == b) atomicMin(&sb.bestkey[o], (unsigned long long)tie_key(sp.mode, cand[c]));
    }
}

__global__ void 
k_tiebreak(const OrientDesc* __restrict__ orients, SelectBufs sb, ScoreParams sp) {
    pdl_enter();
    if (!sb.srch) {
        const int o = blockIdx.y;
        k_tiebreak_body(o, orients, sb, sp);
        return;
    }
    const int na = *sb.nsrch;
    for (int j = blockIdx.y; j < na; j += gridDim.y) {
        const int o = sb.srch[j];
        k_tiebreak_body(o, orients, sb, sp);
    }
}

// After the collision pass (and, in the interlocking mode, the flood fill):
// an orientation with at most late_max ok cells skips the proximity
// transforms (direct = 2); k_collect_plane takes all its ok cells and
// k_direct_score scores them by exact sums.  grid: ceil(n / 128), block 128
__global__ void k_late_direct(OrientDesc* __restrict__ orients, int n, const int* __restrict__ okcount, int late_max) {
    pdl_enter();
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    OrientDesc& od = orients[o];
    if (od.skip || od.direct) return;
    const int c = okcount[o];
    if (c > 0 && c <= late_max) od.direct = 2;
}

struct ResultDev {
    int x, y, z, found;
    double score;
    int ncand;
    unsigned int diag;
    float err_ratio;
    int pad;
};

// orientation o's result from the selection state
__device__ __forceinline__ void finalize_one(const OrientDesc* __restrict__ orients, const SelectBufs& sb,
                                             const ScoreParams& sp, ResultDev* out, int o) {
    ResultDev r;
    r.x = r.y = r.z = -1;
    r.found = 0;
    r.score = 0.0;
    r.ncand = sb.ncand[o];
    r.err_ratio = __uint_as_float(sb.errmax[o]);
    r.pad = 0;
    r.diag = sb.diag[o] | (orients[o].exact ? 1u : 0u);
    if (sb.ncand[o] > sb.cap) r.diag |= 0x100u;
    if (sb.gate) r.diag |= 0x400u;  // the gated second selection (lazy flood fill) ran
    if (orients[o].direct == 1) r.diag |= 0x800u;  // decided without transforms (psb_filter.cuh)
    if (orients[o].direct == 2) r.diag |= 0x1000u; // few ok cells: proximity by exact sums (k_late_direct)
    if (!orients[o].skip && sb.best[o] != 0xffffffffffffffffULL) {
        double s = ord_val(sb.best[o]);
        double cut = sp.mode == 0 ? 1000000000.0 : 1e29;
        if (s < cut) {
            int idx = untie_key(sp.mode, (unsigned int)sb.bestkey[o]);
            r.z = idx % sp.nz;
            r.y = (idx / sp.nz) % sp.ny;
            r.x = idx / (sp.nz * sp.ny);
            r.found = 1;
            r.score = s;
        }
    }
    out[o] = r;
}

__global__ void k_finalize(const OrientDesc* __restrict__ orients, SelectBufs sb, ScoreParams sp, ResultDev* out,
                           int n) {
    pdl_enter();
    if (sb.gate && !*sb.gate) return;
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    finalize_one(orients, sb, sp, out, o);
}

// Index of the best found result (smallest score; on equal scores the lowest
// index, i.e. strict < in index order: fft3.cu:1625, packer.py:500), or -1.
// Called by one full warp; every lane returns the answer.
__device__ __forceinline__ int best_result(const OrientDesc* __restrict__ orients, const ResultDev* __restrict__ res,
                                           int n) {
    const int lane = threadIdx.x & 31;
    double bs = 1e300;
    int bo = -1;
    for (int o = lane; o < n; o += 32) {
        if (orients[o].skip || !res[o].found) continue;
        const double sc = res[o].score;
        if (sc < bs) {  // o grows along a lane: strict < keeps the first
            bs = sc;
            bo = o;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        const double os = __shfl_xor_sync(0xffffffffu, bs, off);
        const int oo = __shfl_xor_sync(0xffffffffu, bo, off);
        if (oo >= 0 && (bo < 0 || os < bs || (os == bs && oo < bo))) {
            bs = os;
            bo = oo;
        }
    }
    return bo;
}

// Lazy interlocking search.  The best cell over the FREE cells of all
// orientations (strict < over orientations, the first minimum wins) is also
// the best over the REACHABLE cells when it is itself reachable, because the
// reachable cells are a subset of the free ones.  A straight run of free
// cells from it to a seed face (i = 0, j = 0, k = 0 always; the far faces
// i = Xv-1, j = Yv-1, k = Zv-1 when the item is non-empty, as k_ff_emit seeds
// them; fft3.cu:263-293) proves it reachable without the flood fill.
// need_ff = 0: proven (or nothing is free: then nothing is reachable either);
// need_ff = 1: the flood fill and a second selection must run.
// grid: 1, block 192 (one warp per ray)
__global__ void k_line_check(const OrientDesc* __restrict__ orients, const ResultDev* __restrict__ res, int n,
                             const uint32_t* __restrict__ freebits, long long sBits, ScoreParams sp, int* need_ff) {
    pdl_enter();
    __shared__ int s_best, s_clear;
    if (threadIdx.x < 32) {
        const int best = best_result(orients, res, n);
        if (threadIdx.x == 0) {
            s_best = best;
            s_clear = 0;
        }
    }
    __syncthreads();
    const int o = s_best;
    if (o < 0) {
        if (threadIdx.x == 0) *need_ff = 0;
        return;
    }
    const OrientDesc& od = orients[o];
    const int t[3] = {res[o].x, res[o].y, res[o].z};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < 6) {
        const int a = warp >> 1, dir = (warp & 1) ? 1 : -1;
        const bool usable = dir < 0 || od.hi[a] >= 0;
        const int len = dir < 0 ? t[a] : od.valid[a] - 1 - t[a];  // cells between t and the face
        bool blocked = !usable || len < 0;
        if (!blocked) {
            for (int s = 1 + lane; s <= len; s += 32) {
                int c[3] = {t[0], t[1], t[2]};
                c[a] += dir * s;
                const uint32_t w =
                    freebits[(size_t)o * sBits + ((size_t)c[0] * sp.ny + c[1]) * sp.nzw + (c[2] >> 5)];
                if (!((w >> (c[2] & 31)) & 1u)) blocked = true;
            }
        }
        blocked = __any_sync(0xffffffffu, blocked);
        if (!blocked && lane == 0) atomicOr(&s_clear, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) *need_ff = s_clear ? 0 : 1;
}

// ---------------------------------------------------------------------------
// flood fill (Algorithm 3) by union-find over z-runs of free cells
// ---------------------------------------------------------------------------
struct FloodBufs {
    const uint32_t* freebits;      // stride sBits
    uint32_t* reach;               // stride sBits
    long long sBits;
    int* cnt;                      // per line run count, stride sLine
    int* off;                      // exclusive offsets, stride sLine
    long long sLine;
    int* rz;                       // run z0 | z1 << 16, stride sRun
    int* rline;
    int* parent;
    int* rflag;
    long long sRun;
    int* total;                    // runs per orientation
    unsigned int* err;             // device error word (limit hit)
    const int* gate;               // when set, the kernels run only if *gate != 0
    unsigned char* okplane;        // when set, k_ff_reach flags planes holding a reachable cell
    long long okstride;            // okplane stride per orientation
    int limit;                     // union-find retries / path steps before err is set
    int* okcount;                  // when set, k_ff_reach adds each orientation's reachable cells
    const int* srch;               // when set: the searched orientations (k_active_list), *nsrch of them;
    const int* nsrch;              // CTA row y takes srch[y], srch[y + gridDim.y], ...
};

// Past `limit` steps both give up, set bit 0 of *err and return a valid run
// index (not necessarily the root): every access stays in bounds and the
// host reports PSB_ERR_LIMIT.
__device__ __forceinline__ int run_find(int* parent, int x, unsigned int* err, int limit) {
    int it = 0;
    int p = __ldcg(&parent[x]);
    while (p != x) {
        int gp = __ldcg(&parent[p]);
        if (gp != p) __stcg(&parent[x], gp);   // path halving; gp is an ancestor
        x = p;
        p = gp;
        if (++it > limit) { atomicOr(err, 1u); return x; }
    }
    return x;
}

__device__ __forceinline__ void run_unite(int* parent, int a, int b, unsigned int* err, int limit) {
    for (int it = 0; it < limit; ++it) {
        a = run_find(parent, a, err, limit);
        b = run_find(parent, b, err, limit);
        if (a == b) return;
        if (a > b) { int t = a; a = b; b = t; }
        int old = atomicCAS(&parent[b], b, a);   // link the larger root under the smaller
        if (old == b) return;
        b = old;
    }
    atomicOr(err, 1u);
}

__device__ __forceinline__ bool fbit(const uint32_t* line, int z) { return (line[z >> 5] >> (z & 31)) & 1u; }

// run starts of a line's free bits (bit z set where a run begins), word by word
__device__ __forceinline__ uint32_t run_starts(const uint32_t* w, int i, uint32_t prevtop) {
    const uint32_t cur = w[i];
    return cur & ~((cur << 1) | prevtop);
}

// Per line (x, y): its free z-runs.  The line's slots are reserved with one
// atomicAdd per warp on the orientation's run counter (total, zeroed first),
// so the run order differs from launch to launch; reachability does not
// depend on it.  Writes cnt/off per line and, per run, (z0 | z1 << 16), its
// line, itself as parent and the seed flag (runs on the seed faces).
// grid: (ceil(nx*ny/256), n_orient), block 256
__device__ __forceinline__ void k_ff_runs_body(const int o, const OrientDesc* __restrict__ orients, FloodBufs fb, ScoreParams sp) {
    if (fb.gate && !*fb.gate) return;
    const OrientDesc& od = orients[o];
    if (od.skip) return;
    const int line = blockIdx.x * blockDim.x + threadIdx.x;
    const bool inl = line < sp.nx * sp.ny;
    const int x = inl ? line / sp.ny : 0, y = inl ? line - x * sp.ny : 0;
    const int Xv = od.valid[0], Yv = od.valid[1], Zv = od.valid[2];
    const bool act = inl && x < Xv && y < Yv;
    const int nzw = sp.nzw;
    const uint32_t* w = fb.freebits + (size_t)o * fb.sBits + (size_t)line * nzw;
    int c = 0;
    if (act) {
        uint32_t prevtop = 0;
        for (int i = 0; i < nzw; ++i) {
            c += __popc(run_starts(w, i, prevtop));
            prevtop = w[i] >> 31;
        }
    }
    // warp-aggregated reservation
    const int lane = threadIdx.x & 31;
    int incl = c;
    for (int d = 1; d < 32; d <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += u;
    }
    int base = 0;
    if (lane == 31 && incl > 0) base = atomicAdd(&fb.total[o], incl);
    base = __shfl_sync(0xffffffffu, base, 31);
    int r = base + incl - c;
    if (!inl) return;
    fb.cnt[(size_t)o * fb.sLine + line] = c;
    fb.off[(size_t)o * fb.sLine + line] = r;
    if (c == 0) return;
    const bool side = (x == 0) || (y == 0) || (od.hi[0] >= 0 && x == Xv - 1) || (od.hi[1] >= 0 && y == Yv - 1);
    int* rz = fb.rz + (size_t)o * fb.sRun;
    int* rl = fb.rline + (size_t)o * fb.sRun;
    int* par = fb.parent + (size_t)o * fb.sRun;
    int* fl = fb.rflag + (size_t)o * fb.sRun;
    // walk runs: start = first set bit at or after z, end = first clear bit after it
    int z = 0;
    while (z < Zv) {
        int wi = z >> 5;
        uint32_t m = w[wi] & (0xffffffffu << (z & 31));
        while (!m && ++wi < nzw) m = w[wi];
        if (!m) break;
        const int z0 = (wi << 5) + __ffs(m) - 1;
        if (z0 >= Zv) break;
        int wj = z0 >> 5;
        uint32_t inv = ~w[wj] & (0xffffffffu << (z0 & 31));
        while (!inv && ++wj < nzw) inv = ~w[wj];
        int z1 = inv ? (wj << 5) + __ffs(inv) - 2 : (nzw << 5) - 1;
        if (z1 >= Zv) z1 = Zv - 1;
        const bool seed = side || z0 == 0 || (od.hi[2] >= 0 && z1 == Zv - 1);
        rz[r] = z0 | (z1 << 16);
        rl[r] = line;
        par[r] = r;
        fl[r] = seed ? 1 : 0;
        ++r;
        z = z1 + 1;
    }
}

__global__ void __launch_bounds__(256)

k_ff_runs(const OrientDesc* __restrict__ orients, FloodBufs fb, ScoreParams sp) {
    pdl_enter();
    if (!fb.srch) {
        const int o = blockIdx.y;
        k_ff_runs_body(o, orients, fb, sp);
        return;
    }
    const int na = *fb.nsrch;
    for (int j = blockIdx.y; j < na; j += gridDim.y) {
        const int o = fb.srch[j];
        k_ff_runs_body(o, orients, fb, sp);
    }
}

// grid: (ceil(nx*ny/256), n_orient)
__device__ __forceinline__ void k_ff_union_body(const int o, const OrientDesc* __restrict__ orients, FloodBufs fb, ScoreParams sp) {
    if (fb.gate && !*fb.gate) return;
    const OrientDesc& od = orients[o];
    if (od.skip) return;
    const int line = blockIdx.x * blockDim.x + threadIdx.x;
    if (line >= sp.nx * sp.ny) return;
    int x = line / sp.ny, y = line - x * sp.ny;
    if (x >= od.valid[0] || y >= od.valid[1]) return;
    const int* cnt = fb.cnt + (size_t)o * fb.sLine;
    const int* off = fb.off + (size_t)o * fb.sLine;
    const int* rz = fb.rz + (size_t)o * fb.sRun;
    int* par = fb.parent + (size_t)o * fb.sRun;
    const int cL = cnt[line], oL = off[line];
    if (cL == 0) return;
    for (int nb = 0; nb < 2; ++nb) {
        int nl;
        if (nb == 0) { if (x == 0) continue; nl = line - sp.ny; }
        else { if (y == 0) continue; nl = line - 1; }
        const int cN = cnt[nl], oN = off[nl];
        int i = 0, j = 0;
        while (i < cL && j < cN) {
            int a = rz[oL + i], b = rz[oN + j];
            int a0 = a & 0xffff, a1 = a >> 16, b0 = b & 0xffff, b1 = b >> 16;
            if (a0 <= b1 && b0 <= a1) run_unite(par, oL + i, oN + j, fb.err, fb.limit);
            if (a1 < b1) ++i; else ++j;
        }
    }
}

__global__ void 
k_ff_union(const OrientDesc* __restrict__ orients, FloodBufs fb, ScoreParams sp) {
    pdl_enter();
    if (!fb.srch) {
        const int o = blockIdx.y;
        k_ff_union_body(o, orients, fb, sp);
        return;
    }
    const int na = *fb.nsrch;
    for (int j = blockIdx.y; j < na; j += gridDim.y) {
        const int o = fb.srch[j];
        k_ff_union_body(o, orients, fb, sp);
    }
}

// grid: (ceil(maxruns/256), n_orient)
__device__ __forceinline__ void k_ff_seed_body(const int o, const OrientDesc* __restrict__ orients, FloodBufs fb) {
    if (fb.gate && !*fb.gate) return;
    if (orients[o].skip) return;
    const int n = fb.total[o];
    int* par = fb.parent + (size_t)o * fb.sRun;
    int* fl = fb.rflag + (size_t)o * fb.sRun;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        if (fl[r] & 1) {
            int root = run_find(par, r, fb.err, fb.limit);
            atomicOr(&fl[root], 2);
        }
    }
}

__global__ void 
k_ff_seed(const OrientDesc* __restrict__ orients, FloodBufs fb) {
    pdl_enter();
    if (!fb.srch) {
        const int o = blockIdx.y;
        k_ff_seed_body(o, orients, fb);
        return;
    }
    const int na = *fb.nsrch;
    for (int j = blockIdx.y; j < na; j += gridDim.y) {
        const int o = fb.srch[j];
        k_ff_seed_body(o, orients, fb);
    }
}

// grid: (ceil(nx*ny/256), n_orient)
__device__ __forceinline__ void k_ff_reach_body(const int o, const OrientDesc* __restrict__ orients, FloodBufs fb, ScoreParams sp) {
    if (fb.gate && !*fb.gate) return;
    const OrientDesc& od = orients[o];
    if (od.skip) return;
    const int line = blockIdx.x * blockDim.x + threadIdx.x;
    if (line >= sp.nx * sp.ny) return;
    int x = line / sp.ny, y = line - x * sp.ny;
    uint32_t* w = fb.reach + (size_t)o * fb.sBits + (size_t)line * sp.nzw;
    for (int i = 0; i < sp.nzw; ++i) w[i] = 0u;
    if (x >= od.valid[0] || y >= od.valid[1]) return;
    const int cL = fb.cnt[(size_t)o * fb.sLine + line], oL = fb.off[(size_t)o * fb.sLine + line];
    const int* rz = fb.rz + (size_t)o * fb.sRun;
    int* par = fb.parent + (size_t)o * fb.sRun;
    const int* fl = fb.rflag + (size_t)o * fb.sRun;
    bool any = false;
    int nreach = 0;
    for (int i = 0; i < cL; ++i) {
        int root = run_find(par, oL + i, fb.err, fb.limit);
        if (!(__ldcg(&fl[root]) & 2)) continue;
        int a = rz[oL + i];
        for (int z = a & 0xffff; z <= (a >> 16); ++z) w[z >> 5] |= 1u << (z & 31);
        nreach += (a >> 16) - (a & 0xffff) + 1;
        any = true;
    }
    if (any && fb.okplane) fb.okplane[(size_t)o * fb.okstride + x] = 1;
    if (fb.okcount) {
        // one atomic per group of lanes that arrive here together
        const unsigned int m = __activemask();
        const int c = __reduce_add_sync(m, nreach);
        if ((threadIdx.x & 31) == __ffs(m) - 1 && c) atomicAdd(&fb.okcount[o], c);
    }
}

__global__ void 
k_ff_reach(const OrientDesc* __restrict__ orients, FloodBufs fb, ScoreParams sp) {
    pdl_enter();
    if (!fb.srch) {
        const int o = blockIdx.y;
        k_ff_reach_body(o, orients, fb, sp);
        return;
    }
    const int na = *fb.nsrch;
    for (int j = blockIdx.y; j < na; j += gridDim.y) {
        const int o = fb.srch[j];
        k_ff_reach_body(o, orients, fb, sp);
    }
}

// ---------------------------------------------------------------------------
// distance field: exact L1 distance to voxels equal to 1 (fft3.cu:887-1004)
// ---------------------------------------------------------------------------
__global__ void k_dist_init(const int32_t* __restrict__ g, int32_t* __restrict__ d, size_t V, int far,
                            const int* gate) {
    pdl_enter();
    if (gate && !*gate) return;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < V; i += (size_t)gridDim.x * blockDim.x)
        d[i] = g[i] == 1 ? 0 : far;
}

// One axis: forward then backward min(d, d_nbr + 1) along lines of length L.
// Lines are staged in shared memory (W lines per CTA) so both the load and
// the store are coalesced; element p of line l sits at base(l) + p*stride.
//   axis x: lines l = y*nz+z,        base = l,                 stride = ny*nz
//   axis y: lines l = x*nz+z,        base = x*ny*nz + z,       stride = nz
//   axis z: lines l = x*ny+y,        base = l*nz,              stride = 1
__global__ void k_dist_axis(int32_t* __restrict__ d, int axis, int nx, int ny, int nz, int W, const int* gate) {
    pdl_enter();
    extern __shared__ int32_t sd[];
    if (gate && !*gate) return;
    const int L = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const long long nlines = axis == 0 ? (long long)ny * nz : (axis == 1 ? (long long)nx * nz : (long long)nx * ny);
    const long long l0 = (long long)blockIdx.x * W;
    if (l0 >= nlines) return;
    const int w = (int)min((long long)W, nlines - l0);
    const size_t stride = axis == 0 ? (size_t)ny * nz : (axis == 1 ? (size_t)nz : 1);
    auto base = [&](long long l) -> size_t {
        if (axis == 0) return (size_t)l;
        if (axis == 1) return (size_t)(l / nz) * ny * nz + (size_t)(l % nz);
        return (size_t)l * nz;
    };
    const int tid = threadIdx.x, nthr = blockDim.x;
    if (axis == 2) {
        for (int idx = tid; idx < w * L; idx += nthr) {
            int li = idx / L, p = idx - li * L;
            sd[li * L + p] = d[base(l0 + li) + p];
        }
    } else {
        for (int idx = tid; idx < w * L; idx += nthr) {
            int p = idx / w, li = idx - p * w;
            sd[li * L + p] = d[base(l0 + li) + (size_t)p * stride];
        }
    }
    __syncthreads();
    for (int li = tid; li < w; li += nthr) {
        int32_t* s = sd + li * L;
        for (int p = L - 2; p >= 0; --p) s[p] = min(s[p], s[p + 1] + 1);
        for (int p = 1; p < L; ++p) s[p] = min(s[p], s[p - 1] + 1);
    }
    __syncthreads();
    if (axis == 2) {
        for (int idx = tid; idx < w * L; idx += nthr) {
            int li = idx / L, p = idx - li * L;
            d[base(l0 + li) + p] = sd[li * L + p];
        }
    } else {
        for (int idx = tid; idx < w * L; idx += nthr) {
            int p = idx / w, li = idx - p * w;
            d[base(l0 + li) + (size_t)p * stride] = sd[li * L + p];
        }
    }
}

// fallback for very long lines: sequential in global memory, one thread per line
__global__ void k_dist_axis_global(int32_t* __restrict__ d, int axis, int nx, int ny, int nz, const int* gate) {
    pdl_enter();
    if (gate && !*gate) return;
    const int L = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const long long nlines = axis == 0 ? (long long)ny * nz : (axis == 1 ? (long long)nx * nz : (long long)nx * ny);
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    size_t stride = axis == 0 ? (size_t)ny * nz : (axis == 1 ? (size_t)nz : 1);
    size_t b = axis == 0 ? (size_t)l : (axis == 1 ? (size_t)(l / nz) * ny * nz + (size_t)(l % nz) : (size_t)l * nz);
    for (int p = L - 2; p >= 0; --p) d[b + p * stride] = min(d[b + p * stride], d[b + (p + 1) * stride] + 1);
    for (int p = 1; p < L; ++p) d[b + p * stride] = min(d[b + p * stride], d[b + (p - 1) * stride] + 1);
}

// sum and sum of squares (around a shift) for the distance spectrum's mean
// subtraction; also the max absolute deviation.
__global__ void k_stats(const int32_t* __restrict__ v, size_t n, int shift, unsigned long long* out) {
    pdl_enter();
    long long s = 0, s2 = 0;
    int mx = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        long long d = (long long)v[i] - shift;
        s += d;
        s2 += d * d;
        mx = max(mx, (int)(d < 0 ? -d : d));
    }
    for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, off);
        s2 += __shfl_xor_sync(0xffffffffu, s2, off);
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&out[0], (unsigned long long)s);
        atomicAdd(&out[1], (unsigned long long)s2);
        atomicMax((unsigned int*)&out[2], (unsigned int)mx);
    }
}

// any negative value?
__global__ void k_any_negative(const int32_t* __restrict__ v, size_t n, unsigned int* flag) {
    pdl_enter();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (v[i] < 0) { atomicOr(flag, 1u); return; }
}

// ---------------------------------------------------------------------------
// placement (packing.cpp:773-788)
// ---------------------------------------------------------------------------
// first tray cell (row-major) where an item voxel > 0 meets a tray voxel > 0
__global__ void k_place_check(const OrientDesc* __restrict__ od_p, const int32_t* __restrict__ tray, int nx, int ny,
                              int nz, int px, int py, int pz, unsigned long long* first) {
    pdl_enter();
    const OrientDesc od = *od_p;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < od.nvox; v += gridDim.x * blockDim.x) {
        int4 q = od.vox[v];
        if (q.w <= 0) continue;
        int oc[3];
        orient_voxel(od, q.x, q.y, q.z, oc);
        int i = px + oc[0], j = py + oc[1], k = pz + oc[2];
        if (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz) continue;
        size_t t = ((size_t)i * ny + j) * nz + k;
        if (tray[t] > 0) atomicMin(first, (unsigned long long)t);
    }
}

__global__ void k_place_write(const OrientDesc* __restrict__ od_p, int32_t* __restrict__ tray, int nx, int ny, int nz,
                              int px, int py, int pz, int32_t id) {
    pdl_enter();
    const OrientDesc od = *od_p;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < od.nvox; v += gridDim.x * blockDim.x) {
        int4 q = od.vox[v];
        if (q.w <= 0) continue;
        int oc[3];
        orient_voxel(od, q.x, q.y, q.z, oc);
        int i = px + oc[0], j = py + oc[1], k = pz + oc[2];
        if (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz) continue;
        size_t t = ((size_t)i * ny + j) * nz + k;
        if (tray[t] == 0) tray[t] = id;
    }
}

// collision_grid post-pass: out-of-tray positions raised to max(c, 1)
__global__ void k_oob_raise(int32_t* __restrict__ c, int nx, int ny, int nz, int hx, int hy, int hz) {
    pdl_enter();
    size_t V = (size_t)nx * ny * nz;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < V; t += (size_t)gridDim.x * blockDim.x) {
        int k = (int)(t % nz), j = (int)((t / nz) % ny), i = (int)(t / ((size_t)ny * nz));
        bool in = ((long long)i + hx <= nx - 1) && ((long long)j + hy <= ny - 1) && ((long long)k + hz <= nz - 1);
        if (!in) c[t] = max(c[t], 1);
    }
}

// labels for interlocking_free_positions: free = collision 0 and in bounds
__global__ void k_bits_from_coll(const int32_t* __restrict__ c, uint32_t* __restrict__ bits, int nx, int ny, int nz,
                                 int nzw, int Xv, int Yv, int Zv) {
    pdl_enter();
    size_t nl = (size_t)nx * ny;
    for (size_t line = blockIdx.x * (size_t)blockDim.x + threadIdx.x; line < nl;
         line += (size_t)gridDim.x * blockDim.x) {
        int x = (int)(line / ny), y = (int)(line % ny);
        uint32_t* w = bits + line * nzw;
        for (int i = 0; i < nzw; ++i) w[i] = 0u;
        if (x >= Xv || y >= Yv) continue;
        for (int z = 0; z < Zv; ++z)
            if (c[line * nz + z] == 0) w[z >> 5] |= 1u << (z & 31);
    }
}

__global__ void k_bits_to_mask(const uint32_t* __restrict__ bits, int32_t* __restrict__ out, int nx, int ny, int nz,
                               int nzw) {
    pdl_enter();
    size_t V = (size_t)nx * ny * nz;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < V; t += (size_t)gridDim.x * blockDim.x) {
        size_t line = t / nz;
        int z = (int)(t % nz);
        out[t] = (bits[line * nzw + (z >> 5)] >> (z & 31)) & 1u;
    }
}

// The per-search reset of the selection and flood-fill state, one launch in
// place of a memset per array (a memset between two kernels also ends their
// launch overlap): the plane minima, best cells and tie keys to all ones,
// the diagnostics, error maxima, candidate and run counters to zero, the
// union-find error word to zero and, when given, the plane flags of the n
// orientations (okbytes bytes) to zero.  grid: 4, block 256
struct SearchReset {
    unsigned long long* smin;
    unsigned long long* best;
    unsigned long long* bestkey;
    unsigned int* diag;
    unsigned int* errmax;
    int* ncand;
    int* total;
    unsigned int* err;
    unsigned char* okplane;
    long long okbytes;
    int n;
};
__global__ void k_search_reset(SearchReset a) {
    pdl_enter();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    for (int o = tid; o < a.n; o += nth) {
        a.smin[o] = ~0ULL;
        a.best[o] = ~0ULL;
        a.bestkey[o] = ~0ULL;
        a.diag[o] = 0u;
        a.errmax[o] = 0u;
        a.ncand[o] = 0;
        a.total[o] = 0;
    }
    if (tid == 0) *a.err = 0u;
    if (a.okplane)
        for (long long i = tid; i < a.okbytes; i += nth) a.okplane[i] = 0;
}
