// psb_loop.cuh — device-side decisions of the greedy packing loop, so the
// host can queue a whole run without waiting on any item.
//
// Per item the stream runs: k_prep (error bounds from the current distance
// statistics) -> the search -> k_decide (best orientation, strict <, first
// wins: fft3.cu:1625 / packer.py:500) -> k_place_item (check, write and
// commit, packing.cpp:773-788) -> the occupancy spectrum rebuild, gated
// on "placed".  Gated kernels read a device flag and return at once when it
// is 0.
#pragma once
#include <climits>

#include "psb_kernels2.cuh"

struct PhiStats {
    unsigned long long raw[4];  // k_stats accumulators (sum, sum of squares, max |.|)
    int mean;                   // rounded mean of phi
    int maxabs;                 // max |phi - mean|
    double norm;                // || phi - mean ||_2
};

struct LoopState {
    int placed;       // items placed so far in this run
    int id_offset;
    int do_place;     // current item found a position
    int placed_now;   // current item was written into the tray (gate of the rebuild)
    int need_phi;     // current item wrote voxels equal to 1 (gate of the distance rebuild)
    int orient;       // chosen orientation of the current item
    int px, py, pz;
    int id;
    unsigned int err; // 1: union-find limit, 2: candidate overflow, 4: placement overlap
    unsigned long long first;  // first overlapping tray cell of the current item
};

// error bound and base of one orientation from the current distance
// statistics (psb_tray::describe)
__device__ __forceinline__ void prep_orient(OrientDesc& d, const PhiStats* __restrict__ ps) {
    const double maxD = (double)d.sabs * (double)ps->maxabs;
    double ulp = 1.1920928955078125e-07;
    if (maxD >= 1.0) {
        int e;
        frexp(maxD, &e);
        ulp = ldexp(1.0, e - 24);
    }
    const double eps = 1.1920928955078125e-07;
    d.delta = 2.0 * eps * sqrt(d.sumsq) * ps->norm + 0.5 * ulp + 1e-3;
    d.exact = (d.delta >= 0.4 || maxD >= 8388608.0) ? 1 : 0;
    d.base = (double)ps->mean * (double)d.sumI;
}

// prep_orient for every orientation of one item.  grid: ceil(n / 64), block 64
__global__ void k_prep(OrientDesc* __restrict__ od, int n, const PhiStats* __restrict__ ps) {
    pdl_enter();
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    prep_orient(od[o], ps);
}

struct DecisionDev {
    int x, y, z, found;
    double score;
    int orientation;
    unsigned int diag;
    int ncand;
    float err_ratio;
};

// One rank's decision in the orientation-sharded loop
// (psb_pack_staged_sharded): its best over the orientations it searched,
// with the global orientation index.  32 bytes, exchanged between ranks.
struct ShardRecord {
    double score;
    int found, orientation, x, y, z;
    int pad;
};

// best over orientations (strict <: the first minimum wins), one warp.
// rec (may be null): the same decision as a ShardRecord for the exchange.
// (the body, run by one full warp)
__device__ __forceinline__ void decide_warp(const OrientDesc* __restrict__ od, const ResultDev* __restrict__ res,
                                            int n, LoopState* ls, DecisionDev* out, const unsigned int* uf_err,
                                            ShardRecord* rec) {
    const int best = best_result(od, res, n);
    unsigned int diag = 0;
    int ncand = 0;
    float er = 0.f;
    for (int o = threadIdx.x; o < n; o += 32) {
        const ResultDev& r = res[o];
        diag |= r.diag;
        ncand += r.ncand;
        er = fmaxf(er, r.err_ratio);
    }
    diag = __reduce_or_sync(0xffffffffu, diag);
    ncand = __reduce_add_sync(0xffffffffu, ncand);
    for (int off = 16; off > 0; off >>= 1) er = fmaxf(er, __shfl_xor_sync(0xffffffffu, er, off));
    if (threadIdx.x != 0) return;
    if (diag & 0x100u) ls->err |= 2u;
    if (*uf_err) ls->err |= 1u;
    DecisionDev d;
    d.diag = diag;
    d.ncand = ncand;
    d.err_ratio = er;
    if (best >= 0) {
        const ResultDev r = res[best];
        d.x = r.x; d.y = r.y; d.z = r.z;
        d.found = 1;
        d.score = r.score;
        d.orientation = best;
        ls->do_place = 1;
        ls->orient = best;
        ls->px = r.x; ls->py = r.y; ls->pz = r.z;
        ls->id = ls->id_offset + ls->placed + 1;
    } else {
        d.x = d.y = d.z = -1;
        d.found = 0;
        d.score = 0.0;
        d.orientation = -1;
        ls->do_place = 0;
    }
    ls->placed_now = 0;
    ls->need_phi = 0;
    ls->first = 0xffffffffffffffffULL;
    *out = d;
    if (rec) {
        ShardRecord r;
        r.score = d.score;
        r.found = d.found;
        r.orientation = d.orientation;
        r.x = d.x; r.y = d.y; r.z = d.z;
        r.pad = 0;
        *rec = r;
    }
}

__global__ void k_decide(const OrientDesc* __restrict__ od, const ResultDev* __restrict__ res, int n,
                         LoopState* ls, DecisionDev* out, const unsigned int* uf_err, ShardRecord* rec) {
    pdl_enter();
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    decide_warp(od, res, n, ls, out, uf_err, rec);
}

// The loop's decision fused into the selection's last step: every
// orientation's result (k_finalize), then the best over them (k_decide), in
// one block.  Arguments of the decision part:
struct DecideArgs {
    LoopState* ls;
    DecisionDev* out;
    const unsigned int* uf_err;
    ShardRecord* rec;
};
// grid: 1, block 128
__global__ void k_finalize_decide(const OrientDesc* __restrict__ orients, SelectBufs sb, ScoreParams sp, ResultDev* res,
                                  int n, DecideArgs da) {
    pdl_enter();
    for (int o = threadIdx.x; o < n; o += blockDim.x) finalize_one(orients, sb, sp, res, o);
    __syncthreads();
    if (threadIdx.x < 32) decide_warp(orients, res, n, da.ls, da.out, da.uf_err, da.rec);
}

// The winner over every rank's record (rank order): the smallest score, on
// equal scores the lowest orientation index -- the reference's strict < over
// the orientations in order (fft3.cu:1625, packer.py:500); every rank then
// places the same item the same way.  Overrides k_decide's local choice.
// grid: 1, block 1
__global__ void k_decide_merge(const ShardRecord* __restrict__ all, int world, LoopState* ls, DecisionDev* out) {
    pdl_enter();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int best = -1;
    for (int r = 0; r < world; ++r) {
        const ShardRecord& c = all[r];
        if (!c.found) continue;
        if (best < 0 || c.score < all[best].score ||
            (c.score == all[best].score && c.orientation < all[best].orientation))
            best = r;
    }
    if (best >= 0) {
        const ShardRecord c = all[best];
        out->x = c.x; out->y = c.y; out->z = c.z;
        out->found = 1;
        out->score = c.score;
        out->orientation = c.orientation;
        ls->do_place = 1;
        ls->orient = c.orientation;
        ls->px = c.x; ls->py = c.y; ls->pz = c.z;
        ls->id = ls->id_offset + ls->placed + 1;
    } else {
        out->x = out->y = out->z = -1;
        out->found = 0;
        out->score = 0.0;
        out->orientation = -1;
        ls->do_place = 0;
    }
}

// The decided placement in one block: the item's z-runs (each a contiguous
// stretch of one tray column) are checked against the tray (the smallest
// overlapped index), then, without an overlap, written with the id and the
// placement is committed (packing.cpp:773-788); an overlap (an FP32 "free"
// cell that the exact check rejects) marks the item unplaced and raises the
// run's error word.  grid: 1, block 1024
// (An 8-CTA thread-block cluster version, the overlap minimum combined in
// CTA 0's distributed shared memory, measured the same: 1488.2 items/s.)
// The check reads the occupancy prefix sums of the tray columns (pocc,
// k_col_prefix<1>, current up to the previous placement): a run meets an
// occupied cell iff its column's count over the run's z range is nonzero,
// two loads per run; only then are the run's cells scanned for the index.
__global__ void __launch_bounds__(1024)
k_place_item(const OrientDesc* __restrict__ od_item, LoopState* ls, int32_t* __restrict__ tray, int nx, int ny,
             int nz, DecisionDev* out, const int32_t* __restrict__ pocc) {
    pdl_enter();
    if (!ls->do_place) return;
    __shared__ unsigned long long s_first;
    if (threadIdx.x == 0) s_first = 0xffffffffffffffffULL;
    __syncthreads();
    const OrientDesc& od = od_item[ls->orient];
    const int px = ls->px, py = ls->py, pz = ls->pz, id = ls->id;
    for (int r = threadIdx.x; r < od.nruns; r += blockDim.x) {
        const int4 q = od.runs[r];
        if (q.w <= 0) continue;
        int a, b, c0, c1;
        orient_run(od, q, &a, &b, &c0, &c1);
        const int i = px + a, j = py + b;
        if (i < 0 || j < 0 || i >= nx || j >= ny) continue;
        const size_t col = ((size_t)i * ny + j) * nz;
        const int k0 = max(0, pz + c0), k1 = min(nz - 1, pz + c1);
        if (k0 > k1) continue;
        const int32_t* P = pocc + ((size_t)i * ny + j) * (nz + 1);
        if (P[k1 + 1] - P[k0] == 0) continue;
        for (int k = k0; k <= k1; ++k)
            if (tray[col + k] > 0) {
                atomicMin(&s_first, (unsigned long long)(col + k));
                break;   // the run's first overlap is its smallest index
            }
    }
    __syncthreads();
    const unsigned long long first = s_first;
    if (first == 0xffffffffffffffffULL) {
        for (int r = threadIdx.x; r < od.nruns; r += blockDim.x) {
            const int4 q = od.runs[r];
            if (q.w <= 0) continue;
            int a, b, c0, c1;
            orient_run(od, q, &a, &b, &c0, &c1);
            const int i = px + a, j = py + b;
            if (i < 0 || j < 0 || i >= nx || j >= ny) continue;
            const size_t col = ((size_t)i * ny + j) * nz;
            for (int k = max(0, pz + c0); k <= min(nz - 1, pz + c1); ++k)
                if (tray[col + k] == 0) tray[col + k] = id;
        }
    }
    if (threadIdx.x != 0) return;
    ls->first = first;
    if (first != 0xffffffffffffffffULL) {
        ls->err |= 4u;
        out->found = 0;
        out->x = out->y = out->z = -1;
        out->orientation = -1;
        out->score = 0.0;
        ls->do_place = 0;
        return;
    }
    ls->placed += 1;
    ls->placed_now = od.nvox > 0 ? 1 : 0;
    ls->need_phi = (id == 1 && od.nvox > 0) ? 1 : 0;
}

// distance statistics on the device: mean after the first k_stats pass,
// norm and max after the second
__global__ void k_phi_mean(PhiStats* ps, unsigned long long V, const int* gate) {
    pdl_enter();
    if (gate && !*gate) return;
    const long long sum = (long long)ps->raw[0];
    ps->mean = (int)llround((double)sum / (double)V);
    ps->raw[0] = ps->raw[1] = ps->raw[2] = ps->raw[3] = 0ULL;
}

__global__ void k_phi_norm(PhiStats* ps, const int* gate) {
    pdl_enter();
    if (gate && !*gate) return;
    ps->norm = sqrt((double)(long long)ps->raw[1]);
    ps->maxabs = (int)(unsigned int)(ps->raw[2] & 0xffffffffULL);
}

// k_stats with a device-side shift and a gate
__global__ void k_stats_g(const int32_t* __restrict__ v, size_t n, const int* shiftp, unsigned long long* out,
                          const int* gate) {
    pdl_enter();
    if (gate && !*gate) return;
    const int shift = shiftp ? *shiftp : 0;
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

// After a placement only the columns under the placed item's box change:
// refresh their occupancy prefix sums (k_col_prefix, MODE 1) and, when the
// candidate filter keeps them (tbits != null, nq uint4 per column), their
// free bits (k_tray_bits), gated on ls->placed_now.  One warp per column.
// grid: ceil(max box columns / 8), block 256
__global__ void k_box_refresh(const int32_t* __restrict__ tray, int32_t* __restrict__ P, uint4* __restrict__ tbits,
                              int nq, int nx, int ny, int nz, const LoopState* __restrict__ ls,
                              const OrientDesc* __restrict__ od_item) {
    pdl_enter();
    if (!ls->placed_now) return;
    const OrientDesc& od = od_item[ls->orient];
    const int by = od.e[1];
    const int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= od.e[0] * by) return;
    const int i = ls->px + k / by, j = ls->py + k % by;
    if (i < 0 || j < 0 || i >= nx || j >= ny) return;
    const size_t col = (size_t)i * ny + j;
    const int32_t* t = tray + col * nz;
    col_prefix<1>(t, P + col * (nz + 1), nz, lane);
    if (tbits) {
        uint32_t* out = (uint32_t*)(tbits + col * nq);
        for (int w = 0; w < 4 * nq; ++w) {
            const int z = 32 * w + lane;
            const unsigned int b = __ballot_sync(0xffffffffu, z < nz && t[z] == 0);
            if (lane == 0) out[w] = b;
        }
    }
}

// Occupied cells (> 0) of the tray and their bounding box, for the packing
// result's statistics (packer.py:582-601): count += cells, box[0..2] = min
// i, j, k, box[3..5] = max (preset to 0, INT_MAX and -1).
// grid: 148 * 4, block 256
__global__ void k_occ_stats(const int32_t* __restrict__ tray, int nx, int ny, int nz, unsigned long long* count,
                            int* box) {
    pdl_enter();
    const size_t V = (size_t)nx * ny * nz;
    unsigned int c = 0;
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {-1, -1, -1};
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < V; t += (size_t)gridDim.x * blockDim.x) {
        if (tray[t] <= 0) continue;
        ++c;
        const int k = (int)(t % nz);
        const size_t r = t / nz;
        const int j = (int)(r % ny), i = (int)(r / ny);
        lo[0] = min(lo[0], i); lo[1] = min(lo[1], j); lo[2] = min(lo[2], k);
        hi[0] = max(hi[0], i); hi[1] = max(hi[1], j); hi[2] = max(hi[2], k);
    }
    c = __reduce_add_sync(0xffffffffu, c);
    for (int a = 0; a < 3; ++a) {
        lo[a] = __reduce_min_sync(0xffffffffu, lo[a]);
        hi[a] = __reduce_max_sync(0xffffffffu, hi[a]);
    }
    if ((threadIdx.x & 31) != 0 || c == 0) return;
    atomicAdd(count, (unsigned long long)c);
    for (int a = 0; a < 3; ++a) {
        atomicMin(&box[a], lo[a]);
        atomicMax(&box[3 + a], hi[a]);
    }
}
