// psb_kernels4.cuh — the plane pass with warp-owned transforms.
//
// Same inputs, outputs and semantics as k_plane2 (psb_kernels3.cuh): per x
// plane and orientation, the inverse along y and the C2R along z of the
// collision and proximity products, free bits and the FP32 proximity field.
// The difference is the work split.  In k_plane2 every radix pass of every
// line is spread over the whole CTA, so each pass ends in a block barrier
// (four per field).  Here a line belongs to a group of lanes of one warp for
// both of its passes: pass 1 loads, transforms and parks its outputs in a
// warp-private, padded shared-memory slab, a __syncwarp hands them to pass 2.
// Block barriers remain only where the data changes owner (after the y pass,
// when all columns of the plane are needed by the z lines, and before the
// next field overwrites the plane buffer): two per field.  The collision
// field's free bits are assembled with warp ballots straight into 32-bit
// words, without the byte mask and packing loop of k_plane2.
#pragma once
#include "psb_kernels3.cuh"

#define PSB_PLANE3_THREADS 512

// A two-pass line transform of length N = R0 * R1 owned by L = R1 lanes.
// Pass 1: lane j1 < R1 runs the radix-R0 butterfly over elements j1 + r*R1.
// Pass 2: the R0 radix-R1 butterflies j2 (k = j2, twiddles W^(r*j2)) read
// elements j2 + r*R0 and produce outputs j2 + r*R0 (Stockham, auto-sorted).
// Pass-1 output m = j1*R0 + r1 is parked at j1*(R0+1) + r1: the padding keeps
// both the stores of pass 1 and the loads of pass 2 free of bank conflicts.
template <int N>
struct WarpLine {
    static constexpr int R0 = Plan2<N>::R0, R1 = Plan2<N>::R1;
    static constexpr int L = R1;                 // lanes per line
    static constexpr int PER = 32 / L;           // lines per warp
    static constexpr int B2 = R0 / R1;           // pass-2 butterflies per lane
    static constexpr int SLAB = R1 * (R0 + 1);   // padded floats2 per line
    static_assert(R0 % R1 == 0, "pass-2 butterflies must divide evenly over the lanes");
    __device__ __forceinline__ static int park(int j1, int r) { return j1 * (R0 + 1) + r; }
    __device__ __forceinline__ static int fetch(int j2, int r) { return r * (R0 + 1) + j2; }
};

// Row stride of the y-inverted plane: HZ rounded up to 2 (mod 4) floats2, so
// the y pass's stores (8 lanes per column, rows 16 apart, 4 columns per warp)
// fall on distinct banks
__host__ __device__ constexpr int plane3_row(int NZ) { return ((NZ / 2 + 1) + 1) / 4 * 4 + 2; }

inline size_t plane3_smem(int NY, int NZ, int ny) {
    auto known = [](int N) { return N == 64 || N == 100 || N == 128; };
    if (!known(NY) || !known(NZ)) return 0;   // no specialised plan for these lengths
    auto slab = [](int N) {
        const int r0 = N == 128 ? 16 : (N == 100 ? 10 : 8);
        const int r1 = N / r0;
        return (size_t)r1 * (r0 + 1);
    };
    auto per = [](int N) {
        const int r1 = N / (N == 128 ? 16 : (N == 100 ? 10 : 8));
        return (size_t)(32 / r1);
    };
    const size_t HZ = NZ / 2 + 1;
    const size_t wy = ((HZ + per(NY) - 1) / per(NY)) * per(NY) * slab(NY);      // y pass: one slab per column
    const size_t wz = (size_t)(PSB_PLANE3_THREADS / 32) * per(NZ) * slab(NZ);   // z pass: per warp
    // the plane buffer also holds the per-warp per-z minima at the end
    const size_t q = std::max((size_t)ny * plane3_row(NZ), (size_t)(PSB_PLANE3_THREADS / 32) * NZ / 2 + 1);
    return sizeof(float2) * (NY + NZ + std::max(wy, wz) + q);
}

// One field of the plane pass.  FIELD 0 (collision): free bits, and when
// pb.set_okplane the plane's "has a free cell" flag.  FIELD 1 (proximity):
// runs only for planes whose okplane flag is set (a free cell, or after the
// flood fill a reachable one); writes the FP32 proximity field and the
// plane's minimum approximate score over its ok cells (pmin, smin).
// grid: (nx, n_orient), block PSB_PLANE3_THREADS
template <int NY, int NZ, int FIELD>
__device__ __forceinline__ void plane3_body(const int o, const OrientDesc* __restrict__ orients, const SearchBufs& sb,
                                            const PlaneBufs& pb, const ScoreParams& sp,
                                            const float2* __restrict__ g_twy, const float2* __restrict__ g_twz) {
    using LY = WarpLine<NY>;
    using LZ = WarpLine<NZ>;
    constexpr int HZ = NZ / 2 + 1;
    constexpr int HZP = plane3_row(NZ);   // row stride of Q (see plane3_row)
    constexpr int NZW = (NZ + 31) / 32;
    constexpr int NWARP = PSB_PLANE3_THREADS / 32;
    constexpr int WY = ((HZ + LY::PER - 1) / LY::PER) * LY::PER * LY::SLAB;
    constexpr int WZ = NWARP * LZ::PER * LZ::SLAB;
    extern __shared__ float2 sm[];
    const OrientDesc& od = orients[o];
    if (od.skip || od.direct) return;   // direct orientations: psb_filter.cuh
    const int x = blockIdx.x;
    const int Xv = od.valid[0], Yv = od.valid[1], Zv = od.valid[2];
    if (x >= Xv || Yv <= 0 || Zv <= 0) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (FIELD == 1 && !pb.okplane[(size_t)o * pb.pstride + x]) {
        if (tid == 0) pb.pmin[(size_t)o * pb.pstride + x] = 0xffffffffffffffffULL;
        return;
    }
    // FIELD 0 after the candidate filter (psb_filter.cuh): a plane without a
    // candidate holds no free cell, and the filter already wrote its words
    const bool filtered = FIELD == 0 && pb.candplane != nullptr && od.nsamp > 0;
    if (filtered && !pb.candplane[(size_t)o * pb.pstride + x]) return;
    const int ny = sp.ny, nzw = sp.nzw;
    const int npairs = (Yv + 1) / 2;
    float2* twy = sm;
    float2* twz = twy + NY;
    float2* W = twz + NZ;                                   // warp slabs
    float2* Q = W + (WY > WZ ? WY : WZ);                    // y-inverted plane [y][HZ]
    load_twiddles(twy, g_twy, NY, tid, PSB_PLANE3_THREADS);
    load_twiddles(twz, g_twz, NZ, tid, PSB_PLANE3_THREADS);
    const float scale = sp.scale;
    unsigned int diag = 0;
    float* Dq = pb.Dq + (size_t)o * pb.sD + (size_t)x * ny * sp.nz;
    uint32_t* fbits = pb.freebits + (size_t)o * pb.sBits + (size_t)x * ny * nzw;
    const uint32_t* obits = pb.okbits + (size_t)o * pb.sBits + (size_t)x * ny * nzw;
    // the row pairs the z pass computes: all of them, or (FIELD 0 filtered)
    // those holding a candidate, or (FIELD 1) those holding an ok cell; the
    // others' words stay zero and their proximity is never read
    __shared__ int plist[(NY + 1) / 2];
    __shared__ int nact;
    if (warp == 0) {
        const uint32_t* rows = FIELD == 0 ? fbits : obits;
        const bool all = FIELD == 0 && !filtered;
        int base = 0;
        for (int p0 = 0; p0 < npairs; p0 += 32) {
            const int p = p0 + lane;
            bool on = p < npairs;
            if (on && !all) {
                uint32_t a = 0u;
                for (int i = 0; i < nzw; ++i) {
                    a |= rows[(size_t)(2 * p) * nzw + i];
                    if (2 * p + 1 < Yv) a |= rows[(size_t)(2 * p + 1) * nzw + i];
                }
                on = a != 0u;
            }
            const unsigned int b = __ballot_sync(0xffffffffu, on);
            if (on) plist[base + __popc(b & ((1u << lane) - 1u))] = p;
            base += __popc(b);
        }
        if (lane == 0) nact = base;
    }
    __syncthreads();
    if (nact == 0) {
        if (FIELD == 1 && tid == 0) pb.pmin[(size_t)o * pb.pstride + x] = 0xffffffffffffffffULL;
        return;
    }
    if (sb.work && tid == 0) {
        if (FIELD == 0) {
            atomicAdd(&sb.work[3], 1ull);
            atomicAdd(&sb.work[4], (unsigned long long)nact);
        } else {
            atomicAdd(&sb.work[7], (unsigned long long)nact);
        }
    }

    // y pass: line (column) c = t*PER + lane / L, lane j = lane % L
    const int yl = lane / LY::L, yj = lane - yl * LY::L;
    // z pass: line (row pair) p = t*PER + lane / L
    const int zl = lane / LZ::L, zj = lane - zl * LZ::L;

    // FIELD 1: per-z minimum proximity of the ok cells, per lane: lane zj of
    // line zl sees z = z0(s, r) + zj in every task, so slot (s, r) always means
    // the same z; the lines of a warp are folded together by shuffles
    float zmin[FIELD == 1 ? LZ::B2 * LZ::R1 : 1];
#pragma unroll
    for (int i = 0; i < (FIELD == 1 ? LZ::B2 * LZ::R1 : 1); ++i) zmin[i] = INFINITY;
    unsigned int anyfree = 0u;
    int nfree = 0;   // FIELD 0: free cells written by this lane

    const float2* P = (FIELD == 0 ? sb.Pc : sb.Pd) + (size_t)o * sb.sP + (size_t)x * NY * HZ;
    for (int t = warp; t * LY::PER < HZ; t += NWARP) {
        const int c = t * LY::PER + yl;
        const bool act = yl < LY::PER && c < HZ;
        float2* slab = W + (size_t)(t * LY::PER + (act ? yl : 0)) * LY::SLAB;
        if (act) {
            float2 v[LY::R0];
#pragma unroll
            for (int r = 0; r < LY::R0; ++r) v[r] = P[(size_t)(yj + r * LY::L) * HZ + c];
            RDFT<LY::R0, 1>::run(v);
#pragma unroll
            for (int r = 0; r < LY::R0; ++r) slab[LY::park(yj, r)] = v[r];
        }
        __syncwarp();
        if (act) {
#pragma unroll
            for (int s = 0; s < LY::B2; ++s) {
                const int j2 = yj + s * LY::L;
                float2 u[LY::R1];
#pragma unroll
                for (int r = 0; r < LY::R1; ++r) u[r] = slab[LY::fetch(j2, r)];
                if (j2 != 0) {
#pragma unroll
                    for (int r = 1; r < LY::R1; ++r) {
                        float2 w = twy[r * j2];
                        w.y = -w.y;
                        u[r] = c_mul(u[r], w);
                    }
                }
                RDFT<LY::R1, 1>::run(u);
#pragma unroll
                for (int r = 0; r < LY::R1; ++r) {
                    const int y = j2 + r * LY::R0;
                    if (y < Yv) Q[y * HZP + c] = u[r];
                }
            }
        }
        __syncwarp();
    }
    __syncthreads();
    // z pass: C2R of two rows per complex line (rows 2p, 2p+1)
    const int na = nact;
    for (int t = warp; t * LZ::PER < na; t += NWARP) {
        const int pi = t * LZ::PER + zl;
        const bool act = zl < LZ::PER && pi < na;
        const int p = act ? plist[pi] : 0;
        const int ya = 2 * p, yb = ya + 1;
        const bool hb = yb < Yv;
        float2* slab = W + (size_t)(warp * LZ::PER + (act ? zl : 0)) * LZ::SLAB;
        if (act) {
            float2 v[LZ::R0];
#pragma unroll
            for (int r = 0; r < LZ::R0; ++r) {
                const int k = zj + r * LZ::L;
                if (k < HZ) {
                    const float2 xa = Q[ya * HZP + k];
                    const float2 xb = hb ? Q[yb * HZP + k] : make_float2(0.f, 0.f);
                    v[r] = make_float2(xa.x - xb.y, xa.y + xb.x);
                } else {
                    const float2 xa = Q[ya * HZP + (NZ - k)];
                    const float2 xb = hb ? Q[yb * HZP + (NZ - k)] : make_float2(0.f, 0.f);
                    v[r] = make_float2(xa.x + xb.y, xb.x - xa.y);
                }
            }
            RDFT<LZ::R0, 1>::run(v);
#pragma unroll
            for (int r = 0; r < LZ::R0; ++r) slab[LZ::park(zj, r)] = v[r];
        }
        __syncwarp();
        // FIELD 0: free words being assembled; FIELD 1: the ok words of rows ya, yb
        uint32_t wa[NZW], wb[NZW];
#pragma unroll
        for (int i = 0; i < NZW; ++i) {
            wa[i] = wb[i] = 0u;
            if (FIELD == 1 && i < nzw) {
                if (act) wa[i] = obits[(size_t)ya * nzw + i];
                if (act && hb) wb[i] = obits[(size_t)yb * nzw + i];
            }
        }
#pragma unroll
        for (int s = 0; s < LZ::B2; ++s) {
            const int j2 = zj + s * LZ::L;
            float2 u[LZ::R1];
#pragma unroll
            for (int r = 0; r < LZ::R1; ++r) u[r] = make_float2(0.f, 0.f);
            if (act) {
#pragma unroll
                for (int r = 0; r < LZ::R1; ++r) u[r] = slab[LZ::fetch(j2, r)];
                if (j2 != 0) {
#pragma unroll
                    for (int r = 1; r < LZ::R1; ++r) {
                        float2 w = twz[r * j2];
                        w.y = -w.y;
                        u[r] = c_mul(u[r], w);
                    }
                }
                RDFT<LZ::R1, 1>::run(u);
            }
#pragma unroll
            for (int r = 0; r < LZ::R1; ++r) {
                // lanes zj = 0..L-1 of this line hold z = z0 + zj, L consecutive cells
                const int z0 = s * LZ::L + r * LZ::R0;
                const int z = z0 + zj;
                const bool zin = act && z < Zv;
                const float va = u[r].x * scale, vb = u[r].y * scale;
                const int w0 = z0 >> 5, sh = z0 & 31;  // compile-time: static word index
                if (FIELD == 0) {
                    const float ra = rintf(va), rb = rintf(vb);
                    if (zin && fabsf(va - ra) > 0.25f) diag |= 2u;
                    if (zin && hb && fabsf(vb - rb) > 0.25f) diag |= 2u;
                    const unsigned int ba = __ballot_sync(0xffffffffu, zin && ra == 0.f);
                    const unsigned int bb = __ballot_sync(0xffffffffu, zin && hb && rb == 0.f);
                    const unsigned int msk = (1u << LZ::L) - 1u;
                    const unsigned int ca = (ba >> (zl * LZ::L)) & msk;
                    const unsigned int cb = (bb >> (zl * LZ::L)) & msk;
                    wa[w0] |= ca << sh;
                    wb[w0] |= cb << sh;
                    if (sh + LZ::L > 32 && w0 + 1 < NZW) {
                        wa[w0 + 1] |= ca >> (32 - sh);
                        wb[w0 + 1] |= cb >> (32 - sh);
                    }
                } else {
                    if (zin) {
                        Dq[(size_t)ya * sp.nz + z] = va;
                        if (hb) Dq[(size_t)yb * sp.nz + z] = vb;
                    }
                    uint32_t ca = wa[w0] >> sh, cb = wb[w0] >> sh;
                    if (sh + LZ::L > 32 && w0 + 1 < NZW) {
                        ca |= wa[w0 + 1] << (32 - sh);
                        cb |= wb[w0 + 1] << (32 - sh);
                    }
                    float m = INFINITY;
                    if (zin && ((ca >> zj) & 1u)) m = va;
                    if (zin && hb && ((cb >> zj) & 1u)) m = fminf(m, vb);
#pragma unroll
                    for (int d = LZ::L; d < 32; d <<= 1) m = fminf(m, __shfl_down_sync(0xffffffffu, m, d));
                    zmin[s * LZ::R1 + r] = fminf(zmin[s * LZ::R1 + r], m);
                }
            }
        }
        if (FIELD == 0 && act && zj == 0) {
#pragma unroll
            for (int i = 0; i < NZW; ++i) {
                if (i < nzw) {
                    fbits[(size_t)ya * nzw + i] = wa[i];
                    if (hb) fbits[(size_t)yb * nzw + i] = wb[i];
                    anyfree |= wa[i] | wb[i];
                    nfree += __popc(wa[i]) + (hb ? __popc(wb[i]) : 0);
                }
            }
        }
        __syncwarp();
    }
    if (FIELD == 0) {
        const unsigned int dg = __reduce_or_sync(0xffffffffu, diag);
        if (lane == 0 && dg) atomicOr(&pb.diag[o], dg);
        if (pb.set_okplane && __any_sync(0xffffffffu, anyfree != 0u) && lane == 0)
            pb.okplane[(size_t)o * pb.pstride + x] = 1;
        if (pb.set_okplane && pb.okcount) {
            const int c = __reduce_add_sync(0xffffffffu, nfree);
            if (lane == 0 && c) atomicAdd(&pb.okcount[o], c);
        }
        return;
    }
    // FIELD 1: the plane's minimum approximate score over its ok cells (the
    // score rises with the proximity at fixed z): per-warp per-z minima meet
    // in the plane buffer Q (idle once every warp has passed the barrier)
    __syncthreads();
    float* zw = (float*)Q;   // [NWARP][NZ]
    for (int i = tid; i < NWARP * NZ; i += PSB_PLANE3_THREADS) zw[i] = INFINITY;
    __syncthreads();
    if (zl == 0) {
#pragma unroll
        for (int s = 0; s < LZ::B2; ++s)
#pragma unroll
            for (int r = 0; r < LZ::R1; ++r) {
                const int z = s * LZ::L + r * LZ::R0 + zj;
                zw[warp * NZ + z] = zmin[(FIELD == 1) ? s * LZ::R1 + r : 0];
            }
    }
    __syncthreads();
    double pm = 1e300;
    for (int z = tid; z < Zv; z += PSB_PLANE3_THREADS) {
        float m = INFINITY;
#pragma unroll
        for (int w = 0; w < NWARP; ++w) m = fminf(m, zw[w * NZ + z]);
        if (m != INFINITY) pm = fmin(pm, ref_score(sp, od.base + (double)m, z));
    }
    for (int off = 16; off > 0; off >>= 1) pm = fmin(pm, __shfl_xor_sync(0xffffffffu, pm, off));
    __shared__ double red[NWARP];
    if (lane == 0) red[warp] = pm;
    __syncthreads();
    if (tid == 0) {
#pragma unroll
        for (int w = 0; w < NWARP; ++w) pm = fmin(pm, red[w]);
        pb.pmin[(size_t)o * pb.pstride + x] = pm < 1e299 ? ord_key(pm) : 0xffffffffffffffffULL;
        if (pm < 1e299) atomicMin(&pb.smin[o], ord_key(pm));
    }
}

template <int NY, int NZ, int FIELD>
__global__ void __launch_bounds__(PSB_PLANE3_THREADS, 2)
k_plane3(const OrientDesc* __restrict__ orients, SearchBufs sb, PlaneBufs pb, ScoreParams sp,
         const float2* __restrict__ g_twy, const float2* __restrict__ g_twz) {
    pdl_enter();
    if (!sb.act) {
        plane3_body<NY, NZ, FIELD>(blockIdx.y, orients, sb, pb, sp, g_twy, g_twz);
        return;
    }
    const int na = *sb.nact;
    for (int j = blockIdx.y; j < na; j += gridDim.y) {
        plane3_body<NY, NZ, FIELD>(sb.act[j], orients, sb, pb, sp, g_twy, g_twz);
        __syncthreads();   // shared memory is reused by the next orientation
    }
}
