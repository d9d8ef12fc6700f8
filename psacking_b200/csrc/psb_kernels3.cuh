// psb_kernels3.cuh — the search's two hot kernels specialised for FFT
// lengths with two-pass radix plans (Plan2 in psb_fft2.cuh).  Same inputs,
// outputs and semantics as k_xpass / k_plane in psb_kernels.cuh, which remain
// the path for other lengths.
#pragma once
#include "psb_fft2.cuh"
#include "psb_kernels2.cuh"

#define PSB_XCOLS 16   // spectrum columns (ky*Hz + kz) per CTA in k_xpass2
// (Measured and not taken: the one-product modes with the item's x transform
// kept in the work buffer, its second pass and the product pass in place, to
// halve the tile's shared memory for a fourth CTA per SM.  Holding a radix-16
// butterfly across the in-place barrier takes 126 registers, and capped at 64
// it spills 224 bytes: 1393.8 against 1451.8 items placed/s.)

// ---------------------------------------------------------------------------
// z,y transforms shared by the flips of one axis permutation
// ---------------------------------------------------------------------------
// The 24 orientations are 6 axis permutations x 4 sign patterns.  After the z
// and y transforms, x is still in real space: with I_p the permuted
// (unflipped) item and flips x_a -> e_a - 1 - x_a,
//   G_o(x, ky, kz) = phase(ky, kz) * G_p(x', ky', kz')     (conjugated if z is flipped)
// where x' = e_x - 1 - x on an x flip (a row reversal, no phase), and for the
// half spectrum in z (real slices are Hermitian in (ky, kz)):
//   z not flipped: ky' = -ky on a y flip, kz' = kz;
//   z flipped:     ky' = -ky unless y is flipped too, kz' = kz, conjugate;
//   phase = W_y^(ky (e_y - 1)) on a y flip * W_z^(kz (e_z - 1)) on a z flip,
// W = exp(-2 pi i / F).  So k_fwd_plane runs once per permutation and the x
// pass reads each orientation's slabs from its permutation's ("base" slots
// 0..5 of the slab buffer).
struct BaseMap {
    int Fy, Hz, Fz;
    const float2* twy;        // exp(-2 pi i n / Fy), n < Fy
    const float2* twz;        // exp(-2 pi i n / Fz), n < Fz
};


// Fused x pass over a tile of PSB_XCOLS consecutive columns c = ky*Hz + kz
// (contiguous in memory, so every row access of the tile is one 128-byte
// segment): item forward along x (pass 1 reads global), products with the
// tray's spectra fused into the first inverse pass, inverse along x (last
// pass writes global rows x < Xv).
//   MODE 0: both products (collision -> Pc, proximity -> Pd)
//   MODE 1: the collision product only (Pc)
//   MODE 2: the proximity product only (Pd), for orientations with an ok
//           plane (okplane, see k_plane3), and stored only on those planes
// In MODE 1 a non-null okplane holds the candidate-filter plane flags: only
// those planes' rows are stored.
// grid: (ceil(Fy*Hz / PSB_XCOLS), n_orient), block 256
template <int N, int MODE, bool SHARED>
__device__ __forceinline__ void
xpass2_body(const int o, const OrientDesc* __restrict__ orients, const SearchBufs& sb, const float2* __restrict__ Socc,
            const float2* __restrict__ Sphi, int ncols, const float2* __restrict__ g_tw,
            const unsigned char* __restrict__ okplane, long long okstride, const BaseMap& bm) {
    constexpr int C = PSB_XCOLS;
    constexpr int R0 = Plan2<N>::R0, R1 = Plan2<N>::R1;
    extern __shared__ float2 sm[];
    const OrientDesc& od = orients[o];
    if (od.skip || od.direct || od.valid[0] <= 0) return;
    const int c0 = blockIdx.x * C;
    const int nl = min(C, ncols - c0);
    float2* tw = sm;
    float2* A = tw + N;
    float2* X = A + N * C;
    unsigned char* okp = (unsigned char*)(X + N * C);   // MODE 2: the orientation's plane flags
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int ex = od.e[0], Xv = od.valid[0];
    // plane flags: MODE 2 the ok planes; MODE 1 (when given) the planes that
    // hold a filter candidate (psb_filter.cuh): rows of other planes are not stored
    const bool flags = MODE == 2 || (MODE == 1 && okplane != nullptr && od.nsamp > 0);
    if (flags) {
        int cnt = 0;
        for (int x = tid; x < Xv; x += nthr) {
            const unsigned char f = okplane[(size_t)o * okstride + x];
            okp[x] = f;
            cnt += f;
        }
        if (!__syncthreads_or(cnt)) return;
        if (MODE != 0 && sb.work && blockIdx.x == 0) {
            for (int d = 16; d > 0; d >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, d);
            if ((tid & 31) == 0 && cnt) atomicAdd(&sb.work[MODE == 1 ? 2 : 6], (unsigned long long)cnt);
            if (MODE == 2 && tid == 0) atomicAdd(&sb.work[5], 1ull);
        }
    } else if (MODE == 1 && sb.work && blockIdx.x == 0 && tid == 0) {
        atomicAdd(&sb.work[2], (unsigned long long)Xv);
    }
    if (MODE == 1 && sb.work && blockIdx.x == 0 && tid == 0) {
        atomicAdd(&sb.work[0], 1ull);
        atomicAdd(&sb.work[1], (unsigned long long)od.e[0]);
    }
    load_twiddles(tw, g_tw, N, tid, nthr);
    __shared__ int srccol[C];
    __shared__ float2 colph[C];
    const int sx = SHARED ? od.flip[0] : 0, sy = SHARED ? od.flip[1] : 0, sz = SHARED ? od.flip[2] : 0;
    if (SHARED && tid < C) {
        const int c = c0 + tid;
        int sc = c;
        float2 ph = make_float2(1.f, 0.f);
        if (tid < nl) {
            const int ky = c / bm.Hz, kz = c - (c / bm.Hz) * bm.Hz;
            const int kys = (sy != sz) ? (ky == 0 ? 0 : bm.Fy - ky) : ky;
            sc = kys * bm.Hz + kz;
            if (sy) ph = c_mul(ph, bm.twy[(int)(((long long)ky * (od.e[1] - 1)) % bm.Fy)]);
            if (sz) ph = c_mul(ph, bm.twz[(int)(((long long)kz * (od.e[2] - 1)) % bm.Fz)]);
        }
        srccol[tid] = sc - c0;
        colph[tid] = ph;
    }
    __syncthreads();
    // the orientation's own slabs, or its permutation's (SHARED)
    const float2* Bi = sb.Bi + (size_t)(SHARED ? od.perm : o) * sb.sB + c0;
    float2* Pc = sb.Pc + (size_t)o * sb.sP + c0;
    float2* Pd = sb.Pd + (size_t)o * sb.sP + c0;
    const float2* So = Socc + c0;
    const float2* Sp = Sphi + c0;
    tpass<N, R0, 1, -1, C, false>(
        [&](int c, int n) {
            if (n >= ex) return make_float2(0.f, 0.f);
            if (!SHARED) return Bi[(size_t)n * ncols + c];
            float2 v = Bi[(size_t)(sx ? ex - 1 - n : n) * ncols + srccol[c]];
            if (sz) v.y = -v.y;
            return c_mul(v, colph[c]);
        },
        [&](int c, int n, float2 v) { A[n * C + c] = v; }, nl, tw, tid, nthr);
    __syncthreads();
    tpass<N, R1, R0, -1, C, false>([&](int c, int n) { return A[n * C + c]; },
                                   [&](int c, int k, float2 v) { X[k * C + c] = v; }, nl, tw, tid, nthr);
    __syncthreads();
    if (MODE != 2) {
        // products conj(I^) * S formed as the inverse's first pass loads them
        tpass<N, R0, 1, 1, C, false>([&](int c, int n) { return c_cmul(X[n * C + c], So[(size_t)n * ncols + c]); },
                                     [&](int c, int n, float2 v) { A[n * C + c] = v; }, nl, tw, tid, nthr);
        __syncthreads();
        tpass<N, R1, R0, 1, C, false>([&](int c, int n) { return A[n * C + c]; },
                                      [&](int c, int x, float2 v) {
                                          if (x < Xv && (!flags || okp[x])) Pc[(size_t)x * ncols + c] = v;
                                      },
                                      nl, tw, tid, nthr);
        if (MODE == 1) return;
        __syncthreads();
    }
    tpass<N, R0, 1, 1, C, false>([&](int c, int n) { return c_cmul(X[n * C + c], Sp[(size_t)n * ncols + c]); },
                                 [&](int c, int n, float2 v) { A[n * C + c] = v; }, nl, tw, tid, nthr);
    __syncthreads();
    tpass<N, R1, R0, 1, C, false>([&](int c, int n) { return A[n * C + c]; },
                                  [&](int c, int x, float2 v) {
                                      if (x < Xv && (!flags || okp[x])) Pd[(size_t)x * ncols + c] = v;
                                  },
                                  nl, tw, tid, nthr);
}

template <int N, int MODE, bool SHARED>
__global__ void __launch_bounds__(256)
k_xpass2(const OrientDesc* __restrict__ orients, SearchBufs sb, const float2* __restrict__ Socc,
         const float2* __restrict__ Sphi, int ncols, const float2* __restrict__ g_tw,
         const unsigned char* __restrict__ okplane, long long okstride, BaseMap bm) {
    pdl_enter();
    if (!sb.act) {
        xpass2_body<N, MODE, SHARED>(blockIdx.y, orients, sb, Socc, Sphi, ncols, g_tw, okplane, okstride, bm);
        return;
    }
    const int na = *sb.nact;
    for (int j = blockIdx.y; j < na; j += gridDim.y) {
        xpass2_body<N, MODE, SHARED>(sb.act[j], orients, sb, Socc, Sphi, ncols, g_tw, okplane, okstride, bm);
        __syncthreads();   // shared memory is reused by the next orientation
    }
}

constexpr size_t xpass2_smem(int N) {
    return sizeof(float2) * ((size_t)N + 2 * (size_t)N * PSB_XCOLS) + (size_t)N;  // + plane flags
}

// shared memory of k_plane2: twiddles, work buffer A and the y-inverted plane
// Q (ny rows; it also holds the plane's free mask as one byte per (y, z)
// while Q is idle)
inline size_t plane2_smem(int NY, int NZ, int ny, int nzw) {
    (void)nzw;
    const size_t HZ = NZ / 2 + 1;
    const size_t a = std::max((size_t)NY * HZ, (size_t)((ny + 1) / 2) * NZ);
    return sizeof(float2) * (NY + NZ + a + (size_t)ny * HZ);
}

// Per (x-plane, orientation): inverse along y then C2R along z (two rows per
// complex transform) for the collision field, then the proximity field.
// grid: (nx, n_orient), block PSB_PLANE_THREADS
#define PSB_PLANE_THREADS 512
template <int NY, int NZ>
__global__ void __launch_bounds__(PSB_PLANE_THREADS, 2)
k_plane2(const OrientDesc* __restrict__ orients, SearchBufs sb, PlaneBufs pb, ScoreParams sp,
         const float2* __restrict__ g_twy, const float2* __restrict__ g_twz) {
    pdl_enter();
    constexpr int HZ = NZ / 2 + 1;
    constexpr int RY0 = Plan2<NY>::R0, RY1 = Plan2<NY>::R1;
    constexpr int RZ0 = Plan2<NZ>::R0, RZ1 = Plan2<NZ>::R1;
    extern __shared__ float2 sm[];
    const int o = blockIdx.y;
    const OrientDesc& od = orients[o];
    if (od.skip) return;
    const int x = blockIdx.x;
    const int Xv = od.valid[0], Yv = od.valid[1], Zv = od.valid[2];
    if (x >= Xv || Yv <= 0 || Zv <= 0) return;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int ny = sp.ny, nzw = sp.nzw;
    const int npairs = (Yv + 1) / 2;
    float2* twy = sm;
    float2* twz = twy + NY;
    float2* A = twz + NZ;
    const size_t asz = max((size_t)NY * HZ, (size_t)((ny + 1) / 2) * NZ);
    float2* Q = A + asz;
    // free mask of field 0 as bytes [y][z] (NZ per row), over Q: Q is idle from
    // the first z pass of field 0 until the second y pass of field 1
    uint8_t* freeb = (uint8_t*)Q;
    load_twiddles(twy, g_twy, NY, tid, nthr);
    load_twiddles(twz, g_twz, NZ, tid, nthr);
    __syncthreads();
    const float scale = sp.scale;
    unsigned int diag = 0;
    float* Dq = pb.Dq + (size_t)o * pb.sD;
    for (int field = 0; field < 2; ++field) {
        const float2* P = (field == 0 ? sb.Pc : sb.Pd) + (size_t)o * sb.sP + (size_t)x * NY * HZ;
        tpass<NY, RY0, 1, 1, HZ, false>([&](int c, int n) { return P[(size_t)n * HZ + c]; },
                                        [&](int c, int n, float2 v) { A[n * HZ + c] = v; }, HZ, twy, tid, nthr);
        __syncthreads();
        tpass<NY, RY1, RY0, 1, HZ, false>([&](int c, int n) { return A[n * HZ + c]; },
                                          [&](int c, int y, float2 v) {
                                              if (y < Yv) Q[y * HZ + c] = v;
                                          },
                                          HZ, twy, tid, nthr);
        __syncthreads();
        tpass<NZ, RZ0, 1, 1, 1, true>(
            [&](int p, int k) {
                const int ya = 2 * p, yb = ya + 1;
                const bool hb = yb < Yv;
                if (k < HZ) {
                    float2 xa = Q[ya * HZ + k];
                    float2 xb = hb ? Q[yb * HZ + k] : make_float2(0.f, 0.f);
                    return make_float2(xa.x - xb.y, xa.y + xb.x);
                }
                float2 xa = Q[ya * HZ + (NZ - k)];
                float2 xb = hb ? Q[yb * HZ + (NZ - k)] : make_float2(0.f, 0.f);
                return make_float2(xa.x + xb.y, xb.x - xa.y);
            },
            [&](int p, int n, float2 v) { A[p * NZ + n] = v; }, npairs, twz, tid, nthr);
        __syncthreads();
        tpass<NZ, RZ1, RZ0, 1, 1, true>(
            [&](int p, int n) { return A[p * NZ + n]; },
            [&](int p, int z, float2 v) {
                if (z >= Zv) return;
#pragma unroll
                for (int half = 0; half < 2; ++half) {
                    const int y = 2 * p + half;
                    if (y >= Yv) break;
                    const float val = (half ? v.y : v.x) * scale;
                    if (field == 0) {
                        const float rv = rintf(val);
                        freeb[y * NZ + z] = rv == 0.f;  // one writer per (y, z): no atomics
                        if (fabsf(val - rv) > 0.25f) diag |= 2u;
                    } else {
                        Dq[((size_t)x * ny + y) * sp.nz + z] = val;
                    }
                }
            },
            npairs, twz, tid, nthr);
        __syncthreads();
        if (field == 0) {
            // pack the byte mask into the plane's free bits (z < Zv; the rest
            // zero) before field 1 reuses Q; its first y pass writes only A,
            // and the barrier after that pass orders these reads first
            uint32_t* fb = pb.freebits + (size_t)o * pb.sBits + (size_t)x * ny * nzw;
            for (int i = tid; i < Yv * nzw; i += nthr) {
                const int y = i / nzw, w = i - y * nzw;
                uint32_t word = 0u;
                const int z0 = w * 32, z1 = min(Zv, z0 + 32);
                for (int z = z0; z < z1; ++z) word |= (uint32_t)freeb[y * NZ + z] << (z - z0);
                fb[i] = word;
            }
        }
    }
    unsigned int dg = __reduce_or_sync(0xffffffffu, diag);
    if ((tid & 31) == 0 && dg) atomicOr(&pb.diag[o], dg);
}

// ---------------------------------------------------------------------------
// forward transforms of the item (per orientation) and of the tray's grids
// ---------------------------------------------------------------------------
struct FwdSrc {
    int kind;            // SRC_ITEM (orientation gather) or SRC_GRID_OCC / SRC_GRID_SUB
    const int32_t* grid; // tray grid (n0, n1, n2)
    int n0, n1, n2;
    const int* subp;     // SRC_GRID_SUB: device-side shift
    const int* gate;     // when set, run only if *gate != 0
    float2* out;         // [n0][NY][HZ] per batch element
    long long out_stride;
    const int* x0p;      // grid sources: when set, CTA i transforms slab *x0p + i (a placed item's planes)
    const int* act;      // SRC_ITEM: when set, CTA row y takes orientations act[y], act[y + gridDim.y], ...
    const int* nact;     //   (*nact of them, k_active_list)
};

// One x slab per CTA: each z line (real, zero-padded to NZ) is transformed as
// a complex line (half the outputs kept), then every kz column is transformed
// along y.  Writes out[i][ky][kz] for all ky < NY.  Replaces k_rfft_z + the y
// k_fft_mid of the generic path.  grid: (max slabs, batch), block 256
template <int NY, int NZ>
__device__ __forceinline__ void fwd_plane_body(const int b, const FwdSrc& src, const OrientDesc* __restrict__ orients,
                                               const float2* __restrict__ g_twy, const float2* __restrict__ g_twz) {
    constexpr int HZ = NZ / 2 + 1;
    constexpr int RY0 = Plan2<NY>::R0, RY1 = Plan2<NY>::R1;
    constexpr int RZ0 = Plan2<NZ>::R0, RZ1 = Plan2<NZ>::R1;
    extern __shared__ float2 sm[];
    int n0 = src.n0, n1 = src.n1, n2 = src.n2;
    OrientDesc od;
    if (src.kind == SRC_ITEM) {
        od = orients[b];
        if (od.skip || od.direct) return;   // direct orientations need no transform
        n0 = od.e[0]; n1 = od.e[1]; n2 = od.e[2];
    }
    const int i = blockIdx.x + (src.x0p ? *src.x0p : 0);
    if (i < 0 || i >= n0) return;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int shift = (src.kind == SRC_GRID_SUB && src.subp) ? *src.subp : 0;
    float2* twy = sm;
    float2* twz = twy + NY;
    float2* A = twz + NZ;
    const int asz = max(n1 * NZ, NY * HZ);
    float2* Q = A + asz;
    load_twiddles(twy, g_twy, NY, tid, nthr);
    load_twiddles(twz, g_twz, NZ, tid, nthr);
    __syncthreads();
    // z: complex transform of each real line j < n1
    tpass<NZ, RZ0, 1, -1, 1, true>(
        [&](int j, int k) {
            float v = 0.f;
            if (k < n2) {
                if (src.kind == SRC_ITEM) {
                    v = (float)od.item[orient_src_index(od, i, j, k)];
                } else {
                    const int r = src.grid[((size_t)i * n1 + j) * n2 + k];
                    v = (float)(src.kind == SRC_GRID_OCC ? (r != 0) : (r - shift));
                }
            }
            return make_float2(v, 0.f);
        },
        [&](int j, int n, float2 v) { A[j * NZ + n] = v; }, n1, twz, tid, nthr);
    __syncthreads();
    tpass<NZ, RZ1, RZ0, -1, 1, true>([&](int j, int n) { return A[j * NZ + n]; },
                                     [&](int j, int kz, float2 v) {
                                         if (kz < HZ) Q[j * HZ + kz] = v;
                                     },
                                     n1, twz, tid, nthr);
    __syncthreads();
    // y: columns kz (rows j >= n1 are zero)
    tpass<NY, RY0, 1, -1, HZ, false>([&](int c, int n) { return n < n1 ? Q[n * HZ + c] : make_float2(0.f, 0.f); },
                                     [&](int c, int n, float2 v) { A[n * HZ + c] = v; }, HZ, twy, tid, nthr);
    __syncthreads();
    float2* out = src.out + (size_t)b * src.out_stride + (size_t)i * NY * HZ;
    tpass<NY, RY1, RY0, -1, HZ, false>([&](int c, int n) { return A[n * HZ + c]; },
                                       [&](int c, int ky, float2 v) { out[(size_t)ky * HZ + c] = v; }, HZ, twy, tid,
                                       nthr);
}

template <int NY, int NZ>
__global__ void __launch_bounds__(256)
k_fwd_plane(FwdSrc src, const OrientDesc* __restrict__ orients, const float2* __restrict__ g_twy,
            const float2* __restrict__ g_twz) {
    pdl_enter();
    if (src.gate && !*src.gate) return;
    if (!src.act) {
        fwd_plane_body<NY, NZ>(blockIdx.y, src, orients, g_twy, g_twz);
        return;
    }
    const int na = *src.nact;
    for (int j = blockIdx.y; j < na; j += gridDim.y) {
        fwd_plane_body<NY, NZ>(src.act[j], src, orients, g_twy, g_twz);
        __syncthreads();   // shared memory is reused by the next orientation
    }
}

inline size_t fwd_plane_smem(int NY, int NZ, int n1) {
    const size_t HZ = NZ / 2 + 1;
    const size_t a = std::max((size_t)n1 * NZ, (size_t)NY * HZ);
    return sizeof(float2) * (NY + NZ + a + (size_t)n1 * HZ);
}

// x forward of a [n0][ncols] slab stack into the spectrum [N][ncols]
// (rows >= n0 are zero).  grid: ceil(ncols / PSB_XCOLS), block 256
template <int N>
__global__ void __launch_bounds__(256)
k_xfwd(const float2* __restrict__ in, float2* __restrict__ out, int n0, int ncols, const int* gate,
       const float2* __restrict__ g_tw) {
    pdl_enter();
    constexpr int C = PSB_XCOLS;
    constexpr int R0 = Plan2<N>::R0, R1 = Plan2<N>::R1;
    extern __shared__ float2 sm[];
    if (gate && !*gate) return;
    const int c0 = blockIdx.x * C;
    const int nl = min(C, ncols - c0);
    float2* tw = sm;
    float2* A = tw + N;
    const int tid = threadIdx.x, nthr = blockDim.x;
    load_twiddles(tw, g_tw, N, tid, nthr);
    __syncthreads();
    const float2* src = in + c0;
    float2* dst = out + c0;
    tpass<N, R0, 1, -1, C, false>(
        [&](int c, int n) { return n < n0 ? src[(size_t)n * ncols + c] : make_float2(0.f, 0.f); },
        [&](int c, int n, float2 v) { A[n * C + c] = v; }, nl, tw, tid, nthr);
    __syncthreads();
    tpass<N, R1, R0, -1, C, false>([&](int c, int n) { return A[n * C + c]; },
                                   [&](int c, int k, float2 v) { dst[(size_t)k * ncols + c] = v; }, nl, tw, tid,
                                   nthr);
}

constexpr size_t xfwd_smem(int N) { return sizeof(float2) * ((size_t)N + (size_t)N * PSB_XCOLS); }
