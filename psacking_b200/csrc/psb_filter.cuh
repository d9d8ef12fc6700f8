// psb_filter.cuh — exact pre-filter of the collision search.
//
// A translation t is collision-free only if every voxel of the item lands on
// an empty tray cell (packing.cpp:254-270 counts overlaps; with non-negative
// item values and the binary occupancy a zero count means no overlap).  So
// the translations where a SUBSET S of the item's voxels lands on empty cells
// are a superset of the free ones.  With S a spread sample of up to
// PSB_FSAMP voxels this superset ("candidates") is computed with bit
// operations on a bit-packed copy of the tray: for each (x, y) column of
// translations and all z at once, AND over s in S of the tray's free bits of
// column (x + s.x, y + s.y) shifted down by s.z.  Nothing here guesses: an
// orientation without any candidate has no free translation (its search is
// skipped: not found, as the full search would say), and a plane without
// candidates holds no free cell (the collision plane pass leaves its zero
// words and skips it).  Every other cell is decided exactly: by the FFT
// collision count, or, for an orientation left with few candidates (at most
// the direct limit), by a direct check of each candidate against the item's
// voxel columns (k_cand_verify_list); such a "direct" orientation also gets its
// proximity as exact integer sums over the item's voxels (k_direct_score)
// and needs no transform at all.
#pragma once
#include "psb_kernels2.cuh"
#include "psb_loop.cuh"

#define PSB_FSAMP 128          // sample voxels per item
#define PSB_FILT_THREADS 128   // translations (y) per CTA row
#define PSB_FBATCH 8           // filter samples whose loads are issued together
#define PSB_FBOUND 9           // bucket bounds per orientation (up to 8 word shifts + 1)
#define PSB_FCUT_AFTER 32      // samples before the cut-off test of k_cand_filter

// Free bits of the tray: tbits[(i*ny + j)*nq + q] holds z in [128q, 128q+128),
// bit set when the cell is empty; bits at z >= nz are clear (not free).
// One warp per column, one ballot per 32 cells.  grid: ceil(nx*ny / 8), block 256
__global__ void k_tray_bits(const int32_t* __restrict__ tray, int nx, int ny, int nz, int nq,
                            uint4* __restrict__ tbits) {
    pdl_enter();
    const int col = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (col >= nx * ny) return;
    const int32_t* t = tray + (size_t)col * nz;
    uint32_t* out = (uint32_t*)(tbits + (size_t)col * nq);
    for (int w = 0; w < 4 * nq; ++w) {
        const int z = 32 * w + lane;
        const unsigned int b = __ballot_sync(0xffffffffu, z < nz && t[z] == 0);
        if (lane == 0) out[w] = b;
    }
}

// The samples of each orientation, oriented and sorted by their word shift
// s.z / 32 (bucket k holds fs[o][bound[o][k] .. bound[o][k+1])), once per
// item, so the filter's CTAs only load them.  One warp per orientation.
// grid: n, block 32
// It also zeroes the orientation's filter counters (candidates, verified
// cells, item columns: counts[o], counts[cap + o], counts[2 cap + o]) and,
// when ps is given, fills its error bound (k_prep's work, one launch less).
template <int NQ>
__global__ void k_cand_prep(OrientDesc* __restrict__ orients, int4* __restrict__ fs, int* __restrict__ fbound,
                            int* __restrict__ counts, int cap, const PhiStats* __restrict__ ps) {
    pdl_enter();
    constexpr int NW = 4 * NQ;
    const int o = blockIdx.x, lane = threadIdx.x;
    if (lane < 3) counts[(size_t)lane * cap + o] = 0;
    if (ps && lane == 0) prep_orient(orients[o], ps);
    __syncwarp();
    const OrientDesc& od = orients[o];
    if (od.skip || od.nsamp <= 0) return;
    const int ns = min(od.nsamp, PSB_FSAMP);
    int4* S = fs + (size_t)o * PSB_FSAMP;
    int* bound = fbound + (size_t)o * (PSB_FBOUND);
    int base = 0;
    for (int k = 0; k < NW; ++k) {
        if (lane == 0) bound[k] = base;
        for (int s0 = 0; s0 < ns; s0 += 32) {
            const int s = s0 + lane;
            int c[3] = {0, 0, 0};
            if (s < ns) {
                const int4 v = od.samp[s];
                orient_voxel(od, v.x, v.y, v.z, c);
            }
            const bool hit = s < ns && (c[2] >> 5) == k;
            const unsigned int b = __ballot_sync(0xffffffffu, hit);
            if (hit) S[base + __popc(b & ((1u << lane) - 1u))] = make_int4(c[0], c[1], c[2], 0);
            base += __popc(b);
        }
    }
    if (lane == 0) bound[NW] = base;
}

__device__ __forceinline__ uint32_t low_bits(int n) { return n >= 32 ? 0xffffffffu : (n <= 0 ? 0u : (1u << n) - 1u); }

// Candidate words of one x plane of one orientation: for rows y < Yv, the
// words cand[(x*ny + y)*nzw + w] (the free-bit layout of the search, so the
// collision pass can refine them in place), candplane[o][x] = "the plane
// holds a candidate", and the orientation's candidate count.  Samples come
// sorted by their word shift s.z / 32 (k_cand_prep) so every shift is a
// compile-time register index; lanes of a warp share the sample; loads go in
// batches; a warp stops once none of its lanes holds a candidate.
// grid: (max Xv, n_orient), block PSB_FILT_THREADS
// The candidate words of one warp's rows (lane = row y0 + lane < Yv) for one
// orientation and x plane: AND over the samples of the tray's free bits of
// column (x + s.x, y + s.y) shifted down by s.z.  col(dx, yy) gives the NQ
// uint4 free-bit words of tray column (x + dx, yy) (from global memory or a
// shared-memory window), samp(i) the i-th shift-sorted sample; bound[k] ..
// bound[k+1] are the samples with whole-word shift k (k_cand_prep).
template <int NQ, int BATCH, class COLF, class SAMPF>
__device__ __forceinline__ void filter_rows(int y0, int Yv, int Zv, COLF col, SAMPF samp, const int* bound, int cut_pct,
                                            uint32_t (&c)[4 * NQ]) {
    constexpr int NW = 4 * NQ;
    const int lane = threadIdx.x & 31;
    const int y = y0 + lane;
    const bool act = y < Yv;
    int n0 = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        c[w] = act ? low_bits(Zv - 32 * w) : 0u;
        n0 += __popc(c[w]);
    }
    // Cut-off: any subset of the samples gives a valid (wider) candidate
    // set, so a warp whose translations still mostly survive after
    // PSB_FCUT_AFTER samples (open space, nothing to skip) stops there.
    bool stop = false, checked = cut_pct <= 0;
    int done = 0;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
        // shift of k whole words: word w of the shifted column is
        // funnel(T[w + k], T[w + k + 1]) >> (s.z & 31)
        const int s1 = bound[k + 1];
        for (int s0 = bound[k]; s0 < s1 && !stop; s0 += BATCH) {
            uint32_t a = 0u;
            int nb = 0;
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                a |= c[w];
                nb += __popc(c[w]);
            }
            if (!__any_sync(0xffffffffu, a != 0u)) {
                stop = true;
                break;
            }
            if (!checked && done >= PSB_FCUT_AFTER) {
                checked = true;
                int t0 = n0, t1 = nb;
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) {
                    t0 += __shfl_xor_sync(0xffffffffu, t0, d);
                    t1 += __shfl_xor_sync(0xffffffffu, t1, d);
                }
                if ((long long)t1 * 100 > (long long)t0 * cut_pct) {
                    stop = true;
                    break;
                }
            }
            done += BATCH;
            uint4 v[BATCH][NQ];
            int off[BATCH];
#pragma unroll
            for (int i = 0; i < BATCH; ++i) {
                off[i] = 0;
#pragma unroll
                for (int q = 0; q < NQ; ++q) v[i][q] = make_uint4(0u, 0u, 0u, 0u);
                if (s0 + i < s1) {
                    const int3 p = samp(s0 + i);
                    off[i] = p.z & 31;
                    if (act) {
                        const uint4* cp = col(p.x, y + p.y);
#pragma unroll
                        for (int q = 0; q < NQ; ++q) v[i][q] = cp[q];
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < BATCH; ++i) {
                if (s0 + i >= s1) break;
                uint32_t T[NW];
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    T[4 * q] = v[i][q].x;
                    T[4 * q + 1] = v[i][q].y;
                    T[4 * q + 2] = v[i][q].z;
                    T[4 * q + 3] = v[i][q].w;
                }
#pragma unroll
                for (int w = 0; w < NW; ++w) {
                    const uint32_t lo = (w + k < NW) ? T[w + k] : 0u;
                    const uint32_t hi = (w + k + 1 < NW) ? T[w + k + 1] : 0u;
                    c[w] &= __funnelshift_r(lo, hi, off[i]);
                }
            }
        }
    }
}

// One warp's rows: store the candidate words, count them and list them while
// the orientation has at most ccap (a list for the direct checks of
// k_cand_verify_list); returns whether the rows hold a candidate.
template <int NQ>
__device__ __forceinline__ bool filter_store(const uint32_t (&c)[4 * NQ], int o, int x, int y0, int Yv, int ny,
                                             int nzw, int nz, uint32_t* __restrict__ cw, int* __restrict__ ccount,
                                             int* __restrict__ clist, int ccap) {
    constexpr int NW = 4 * NQ;
    const int lane = threadIdx.x & 31;
    const int y = y0 + lane;
    int mine = 0;
    bool any = false;
    if (y < Yv) {
#pragma unroll
        for (int w = 0; w < NW; ++w)
            if (w < nzw) {
                cw[(size_t)y * nzw + w] = c[w];
                any |= c[w] != 0u;
                mine += __popc(c[w]);
            }
    }
    int incl = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += u;
    }
    int base = 0;
    if (lane == 31 && incl) base = atomicAdd(&ccount[o], incl);
    base = __shfl_sync(0xffffffffu, base, 31);
    int slot = base + incl - mine;
    if (mine && slot < ccap) {
        int* L = clist + (size_t)o * ccap;
        const int t0 = (x * ny + y) * nz;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            uint32_t m = w < nzw ? c[w] : 0u;
            while (m && slot < ccap) {
                const int bit = __ffs(m) - 1;
                m &= m - 1u;
                L[slot++] = t0 + 32 * w + bit;
            }
        }
    }
    return __any_sync(0xffffffffu, any);
}

// Candidate words of one x plane of one orientation: for rows y < Yv, the
// words cand[(x*ny + y)*nzw + w] (the free-bit layout of the search, so the
// collision pass can refine them in place), candplane[o][x] = "the plane
// holds a candidate", the orientation's candidate count and, while there are
// few, its candidate list.  Samples come sorted by their word shift s.z / 32
// (k_cand_prep) so every shift is a compile-time register index; lanes of a
// warp share the sample; loads go in batches; a warp stops once none of its
// lanes holds a candidate.  The tray's free bits are read from global memory
// (L1/L2); k_cand_filter_plane reads them from a shared-memory window.
// grid: (max Xv, n_orient), block PSB_FILT_THREADS
template <int NQ, int BATCH = PSB_FBATCH, int MINB = 8>
__global__ void __launch_bounds__(PSB_FILT_THREADS, MINB)
k_cand_filter(const OrientDesc* __restrict__ orients, const uint4* __restrict__ tbits, int ny, int nzw,
              uint32_t* __restrict__ cand, long long sBits, unsigned char* __restrict__ candplane, long long pstride,
              int* __restrict__ ccount, const int4* __restrict__ fs, const int* __restrict__ fbound, int cut_pct,
              int* __restrict__ clist, int ccap, int nz) {
    pdl_enter();
    constexpr int NW = 4 * NQ;
    const int o = blockIdx.y, x = blockIdx.x;
    const OrientDesc& od = orients[o];
    if (od.skip || od.nsamp <= 0) return;
    const int Xv = od.valid[0], Yv = od.valid[1], Zv = od.valid[2];
    if (x >= Xv || Yv <= 0 || Zv <= 0) return;
    const int tid = threadIdx.x, warp = tid >> 5;
    __shared__ int3 S[PSB_FSAMP];
    __shared__ int bound[NW + 1];   // samples with shift k are S[bound[k] .. bound[k+1])
    const int ns = min(od.nsamp, PSB_FSAMP);
    for (int s = tid; s < ns; s += PSB_FILT_THREADS) {
        const int4 v = __ldg(&fs[(size_t)o * PSB_FSAMP + s]);
        S[s] = make_int3(v.x, v.y, v.z);
    }
    if (tid <= NW) bound[tid] = __ldg(&fbound[(size_t)o * PSB_FBOUND + tid]);
    __syncthreads();
    uint32_t* cw = cand + (size_t)o * sBits + (size_t)x * ny * nzw;
    int any = 0;
    for (int y0 = warp * 32; y0 < Yv; y0 += PSB_FILT_THREADS) {
        uint32_t c[NW];
        filter_rows<NQ, BATCH>(
            y0, Yv, Zv, [&](int dx, int yy) { return tbits + ((size_t)(x + dx) * ny + yy) * NQ; },
            [&](int i) { return S[i]; }, bound, cut_pct, c);
        any |= filter_store<NQ>(c, o, x, y0, Yv, ny, nzw, nz, cw, ccount, clist, ccap) ? 1 : 0;
    }
    any = __syncthreads_or(any);
    if (tid == 0) candplane[(size_t)o * pstride + x] = any ? 1 : 0;
}

// The same candidate words, one CTA per x plane for every orientation: the
// tray's free bits of planes x .. x + E - 1 (E = the items' largest x extent)
// are staged once in shared memory, and the CTA's warps take the
// (orientation, 32-row block) tasks of the plane, reading samples from the
// k_cand_prep buffers (L1-resident).  Staging the window replaces the L2
// round trip of every sample load.  grid: (max Xv, orientation groups),
// block PSB_FILT_PLANE_THREADS,
// dynamic shared memory E * ny * NQ uint4 + n bytes of plane flags
#define PSB_FILT_PLANE_THREADS 512
template <int NQ>
__global__ void __launch_bounds__(PSB_FILT_PLANE_THREADS, 2)
k_cand_filter_plane(const OrientDesc* __restrict__ orients, int n, const uint4* __restrict__ tbits, int nx, int ny,
                    int nzw, int E, uint32_t* __restrict__ cand, long long sBits,
                    unsigned char* __restrict__ candplane, long long pstride, int* __restrict__ ccount,
                    const int4* __restrict__ fs, const int* __restrict__ fbound, int cut_pct,
                    int* __restrict__ clist, int ccap, int nz) {
    pdl_enter();
    constexpr int NW = 4 * NQ;
    extern __shared__ uint4 win[];   // [E][ny][NQ]
    const int x = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarp = PSB_FILT_PLANE_THREADS / 32;
    unsigned char* flag = (unsigned char*)(win + (size_t)E * ny * NQ);
    const int planes = min(E, nx - x);
    const size_t nwords = (size_t)planes * ny * NQ;
    const uint4* src = tbits + (size_t)x * ny * NQ;   // planes x .. x + planes - 1 are contiguous
    for (size_t i = tid; i < nwords; i += PSB_FILT_PLANE_THREADS) win[i] = __ldg(&src[i]);
    for (int o = tid; o < n; o += PSB_FILT_PLANE_THREADS) flag[o] = 0;
    __syncthreads();
    // CTA row blockIdx.y takes the orientations o = blockIdx.y (mod gridDim.y)
    const int yblocks = (ny + 31) / 32;
    const int nog = (n - (int)blockIdx.y + (int)gridDim.y - 1) / (int)gridDim.y;
    for (int task = warp; task < nog * yblocks; task += nwarp) {
        const int o = (task / yblocks) * gridDim.y + blockIdx.y, y0 = (task % yblocks) * 32;
        const OrientDesc& od = orients[o];
        if (od.skip || od.nsamp <= 0) continue;
        const int Xv = od.valid[0], Yv = od.valid[1], Zv = od.valid[2];
        if (x >= Xv || y0 >= Yv || Zv <= 0) continue;
        const int4* S = fs + (size_t)o * PSB_FSAMP;
        int bound[NW + 1];
#pragma unroll
        for (int k = 0; k <= NW; ++k) bound[k] = __ldg(&fbound[(size_t)o * PSB_FBOUND + k]);
        uint32_t c[NW];
        filter_rows<NQ, PSB_FBATCH>(
            y0, Yv, Zv, [&](int dx, int yy) { return win + ((size_t)dx * ny + yy) * NQ; },
            [&](int i) {
                const int4 v = __ldg(&S[i]);
                return make_int3(v.x, v.y, v.z);
            },
            bound, cut_pct, c);
        uint32_t* cw = cand + (size_t)o * sBits + (size_t)x * ny * nzw;
        if (filter_store<NQ>(c, o, x, y0, Yv, ny, nzw, nz, cw, ccount, clist, ccap) && lane == 0) flag[o] = 1;
    }
    __syncthreads();
    for (int o = blockIdx.y + tid * gridDim.y; o < n; o += PSB_FILT_PLANE_THREADS * gridDim.y) {
        const OrientDesc& od = orients[o];
        if (od.skip || od.nsamp <= 0 || x >= od.valid[0] || od.valid[1] <= 0 || od.valid[2] <= 0) continue;
        candplane[(size_t)o * pstride + x] = flag[o];
    }
}

// Stage 0 (after k_cand_filter, count = candidates): an orientation without
// a candidate is skipped; one with at most direct_max candidates and an item
// at most 64 cells high (two mask words per column) becomes direct.
// Stage 1 (after k_cand_verify_list, count = verified free cells): a direct
// orientation without a free cell is skipped.  okclear, when given, has the
// orientation's nclear plane flags (stride okstride) cleared first, for the
// verification to set.  grid: ceil(n / 128), block 128
__global__ void k_cand_apply(OrientDesc* __restrict__ orients, int n, const int* __restrict__ count, int stage,
                             int direct_max, unsigned char* __restrict__ okclear, long long okstride, int nclear) {
    pdl_enter();
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    if (okclear)
        for (int x = 0; x < nclear; ++x) okclear[(size_t)o * okstride + x] = 0;
    OrientDesc& od = orients[o];
    if (od.skip || od.nsamp <= 0) return;
    if (stage == 0) {
        if (count[o] == 0) od.skip = 1;
        else if (count[o] <= direct_max && od.e[2] <= 64) od.direct = 1;
    } else if (od.direct && count[o] == 0) {
        od.skip = 1;
    }
}

// Column masks of a direct orientation's item: for each (a, b) holding a
// positive voxel, {a | b << 16, bits of c < 32, bits of 32 <= c < 64} in
// cols[o][k], k < ncol[o] (any order).  grid: (max e[0], n), block 64
__global__ void k_item_cols(const OrientDesc* __restrict__ orients, uint4* __restrict__ cols, long long cstride,
                            int* __restrict__ ncol) {
    pdl_enter();
    const int o = blockIdx.y, a = blockIdx.x;
    const OrientDesc& od = orients[o];
    if (od.skip || !od.direct || a >= od.e[0]) return;
    const int lane = threadIdx.x & 31;
    for (int b0 = 0; b0 < od.e[1]; b0 += blockDim.x) {
        const int b = b0 + threadIdx.x;
        uint32_t m0 = 0u, m1 = 0u;
        if (b < od.e[1])
            for (int c = 0; c < od.e[2]; ++c)
                if (__ldg(&od.item[orient_src_index(od, a, b, c)]) > 0) {
                    if (c < 32) m0 |= 1u << c;
                    else m1 |= 1u << (c - 32);
                }
        const bool has = (m0 | m1) != 0u;
        const unsigned int bal = __ballot_sync(0xffffffffu, has);
        int slot = 0;
        if (lane == 0 && bal) slot = atomicAdd(&ncol[o], __popc(bal));
        slot = __shfl_sync(0xffffffffu, slot, 0);
        if (has)
            cols[(size_t)o * cstride + slot + __popc(bal & ((1u << lane) - 1u))] =
                make_uint4((uint32_t)a | ((uint32_t)b << 16), m0, m1, 0u);
    }
}

// k_item_cols for every orientation of a range of staged items at once
// (they depend on the item only, not on the tray), ahead of the packing
// loop: item i's columns go to cols + off[i] with stride[i] entries per
// orientation, counts to ncol[i * n + o] (zeroed first).  Orientations that
// do not fit the tray (skip) are left out; which ones become direct is known
// only per item, and the verification reads the direct ones only.
// grid: (max e[0], n, items), block 64
__global__ void k_item_cols_all(const OrientDesc* __restrict__ od_all, int n, int i0, uint4* __restrict__ cols,
                                const long long* __restrict__ off, const int* __restrict__ stride,
                                int* __restrict__ ncol) {
    pdl_enter();
    const int it = i0 + blockIdx.z, o = blockIdx.y, a = blockIdx.x;
    const OrientDesc& od = od_all[(size_t)it * n + o];
    if (od.skip || a >= od.e[0]) return;
    const int lane = threadIdx.x & 31;
    uint4* out = cols + off[it] + (size_t)o * stride[it];
    int* cnt = ncol + (size_t)it * n + o;
    for (int b0 = 0; b0 < od.e[1]; b0 += blockDim.x) {
        const int b = b0 + threadIdx.x;
        uint32_t m0 = 0u, m1 = 0u;
        if (b < od.e[1])
            for (int c = 0; c < od.e[2] && c < 64; ++c)
                if (__ldg(&od.item[orient_src_index(od, a, b, c)]) > 0) {
                    if (c < 32) m0 |= 1u << c;
                    else m1 |= 1u << (c - 32);
                }
        const bool has = (m0 | m1) != 0u;
        const unsigned int bal = __ballot_sync(0xffffffffu, has);
        int slot = 0;
        if (lane == 0 && bal) slot = atomicAdd(cnt, __popc(bal));
        slot = __shfl_sync(0xffffffffu, slot, 0);
        if (has) out[slot + __popc(bal & ((1u << lane) - 1u))] = make_uint4((uint32_t)a | ((uint32_t)b << 16), m0, m1, 0u);
    }
}

// Exact collision check of every candidate of the direct orientations, from
// the candidate lists k_cand_filter wrote: the translation (x, y, z) is free
// when no item column (a, b) meets an occupied cell of tray column
// (x + a, y + b) over z .. z + 63.  The candidates of all orientations are
// spread over the whole grid, one warp each, its lanes one item column each,
// stopping at the first overlap.  A blocked candidate's bit is cleared in the
// candidate words (which become the free words); free cells are counted
// (stage 1 of k_cand_apply) and, outside the interlocking mode, flag their
// plane (okplane).  grid: any, block 256; dynamic shared memory (n+1) ints
__global__ void __launch_bounds__(256)
k_cand_verify_list(const OrientDesc* __restrict__ orients, int n, const uint4* __restrict__ tbits, int ny, int nz,
                   int nzw, int tq, uint32_t* __restrict__ cand, long long sBits, const int* __restrict__ clist,
                   int ccap, const int* __restrict__ ccount, const uint4* __restrict__ cols, long long cstride,
                   const int* __restrict__ ncol, int* __restrict__ vcount, unsigned char* __restrict__ okplane,
                   long long pstride, int set_okplane) {
    pdl_enter();
    extern __shared__ int pre[];   // pre[o]: direct candidates of orientations before o
    if (threadIdx.x < 32) {
        // warp 0: the orientations' counts loaded in parallel, an exclusive scan
        int acc = 0;
        for (int o0 = 0; o0 < n; o0 += 32) {
            const int o = o0 + threadIdx.x;
            int c = 0;
            if (o < n) {
                const OrientDesc& od = orients[o];
                if (!od.skip && od.direct == 1) c = min(ccount[o], ccap);
            }
            int incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, incl, d);
                if ((int)threadIdx.x >= d) incl += u;
            }
            if (o < n) pre[o] = acc + incl - c;
            acc += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (threadIdx.x == 0) pre[n] = acc;
    }
    __syncthreads();
    const int total = pre[n];
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const uint32_t* T = (const uint32_t*)tbits;
    const int tw = 4 * tq;   // words per tray column
    for (int g = blockIdx.x * wpb + (threadIdx.x >> 5); g < total; g += gridDim.x * wpb) {
        int o = 0;
        while (pre[o + 1] <= g) ++o;
        const int t = clist[(size_t)o * ccap + (g - pre[o])];
        const int z = t % nz, y = (t / nz) % ny, x = t / (nz * ny);
        const int nc = ncol[o];
        const uint4* cl = cols + (size_t)o * cstride;
        const int sh = z >> 5, off = z & 31;
        bool hit = false;
        for (int k0 = 0; k0 < nc && !hit; k0 += 32) {
            const int k = k0 + lane;
            bool c = false;
            if (k < nc) {
                const uint4 r = __ldg(&cl[k]);
                const int a = (int)(r.x & 0xffffu), b = (int)(r.x >> 16);
                const uint32_t* tc = T + ((size_t)(x + a) * ny + (y + b)) * tw;
                const uint32_t t0 = __ldg(&tc[sh]);
                const uint32_t t1 = sh + 1 < nzw ? __ldg(&tc[sh + 1]) : 0u;
                const uint32_t f0 = __funnelshift_r(t0, t1, off);
                uint32_t f1 = 0u;
                if (r.z) {
                    const uint32_t t2 = sh + 2 < nzw ? __ldg(&tc[sh + 2]) : 0u;
                    f1 = __funnelshift_r(t1, t2, off);
                }
                c = ((r.y & ~f0) | (r.z & ~f1)) != 0u;
            }
            hit = __any_sync(0xffffffffu, c);
        }
        if (lane == 0) {
            if (hit) {
                atomicAnd(&cand[(size_t)o * sBits + ((size_t)x * ny + y) * nzw + sh], ~(1u << off));
            } else {
                atomicAdd(&vcount[o], 1);
                if (set_okplane) okplane[(size_t)o * pstride + x] = 1;
            }
        }
    }
}

// Exact score of every ok cell of a direct orientation (k_collect_plane
// collected all of them): the proximity sum over the item's z-runs in
// integers (the exact value the reference's FFT rounds to; pphi holds the
// distance field's prefix sums along z, psb_kernels.cuh), then the
// reference's score.  One warp per cell.  grid: (blocks, n_orient), block 256
__device__ __forceinline__ void k_direct_score_body(const int o, const OrientDesc* __restrict__ orients, SelectBufs sb, ScoreParams sp, const int32_t* __restrict__ pphi) {
    if (sb.gate && !*sb.gate) return;
    const OrientDesc& od = orients[o];
    if (od.skip || !od.direct) return;
    const int n = min(sb.ncand[o], sb.cap);
    const int* cand = sb.cand + (size_t)o * sb.cap;
    double* cs = sb.cscore + (size_t)o * sb.cap;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int c = blockIdx.x * wpb + (threadIdx.x >> 5); c < n; c += gridDim.x * wpb) {
        const int t = cand[c];
        const int z = t % sp.nz;
        const int y = (t / sp.nz) % sp.ny;
        const int x = t / (sp.nz * sp.ny);
        long long acc = 0;
        for (int r = lane; r < od.nruns; r += 32) {
            const int4 q = __ldg(&od.runs[r]);
            int a, b, c0, c1;
            orient_run(od, q, &a, &b, &c0, &c1);
            const int32_t* P = pphi + ((size_t)(x + a) * sp.ny + (y + b)) * (sp.nz + 1) + z;
            acc += (long long)q.w * (__ldg(&P[c1 + 1]) - __ldg(&P[c0]));
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, d);
        if (lane == 0) {
            const double s = ref_score(sp, (double)acc, z);
            cs[c] = s;
            atomicMin(&sb.best[o], ord_key(s));
        }
    }
}

__global__ void __launch_bounds__(256)

k_direct_score(const OrientDesc* __restrict__ orients, SelectBufs sb, ScoreParams sp, const int32_t* __restrict__ pphi) {
    pdl_enter();
    if (!sb.srch) {
        const int o = blockIdx.y;
        k_direct_score_body(o, orients, sb, sp, pphi);
        return;
    }
    const int na = *sb.nsrch;
    for (int j = blockIdx.y; j < na; j += gridDim.y) {
        const int o = sb.srch[j];
        k_direct_score_body(o, orients, sb, sp, pphi);
    }
}
