// psb_kernels.cuh — device kernels of the placement search (sm_100a).
//
// Grid layout: the tray is (nx, ny, nz) int32, element (i,j,k) at
// (i*ny + j)*nz + k.  Spectra are half spectra along z: [Fx][Fy][Hz] float2
// with Hz = Fz/2 + 1, Fx >= nx, Fy >= ny, Fz >= nz.  Search correlations use
// the circular grid F >= n, which is exact for every translation that keeps
// the item inside the tray (t + x <= n - 1 < F never wraps); the reference
// pads to 2n+1 (fft3.cu:1111) and masks the rest anyway (fft3.cu:166).
#pragma once
#include "psb_fft.cuh"

#define PSB_TILE 8          // columns per CTA in strided-axis transforms
#define PSB_PAIRS 8         // line pairs per CTA in z transforms
#define PSB_THREADS 256

// ---------------------------------------------------------------------------
// value sources for real -> half-spectrum z transforms
// ---------------------------------------------------------------------------
enum SrcKind { SRC_GRID_RAW = 0, SRC_GRID_OCC = 1, SRC_GRID_SUB = 2, SRC_ITEM = 3 };

struct OrientDesc {
    // oriented item dims and the signed axis permutation into the base item
    int e[3];
    int src_axis[3];
    int flip[3];
    int b[3];                 // base item dims
    int hi[3];                // max index of positive voxels (oriented), -1 if none
    int valid[3];             // Xv, Yv, Zv : translations t with t + hi <= n - 1
    int skip;                 // orientation larger than the tray
    int exact;                // 1: FP32 bound >= 0.4, candidates re-scored exactly
    long long sumI;           // sum of item values
    double delta;             // bound on |D~ - D|
    double base;              // m * sumI (integer, exact in double)
    const int32_t* item;      // device base item
    const int4* vox;          // device voxel list of the base item (x,y,z,value); the
                              // synchronous calls only (null in the packing loop, which
                              // places items by their runs)
    int nvox;
    int perm;                 // index of its axis permutation among the item's 6 bases
    double sumsq;             // sum of squared item values
    long long sabs;           // sum of |item values|
    const int4* samp;         // sample voxels of the base item for the candidate filter (psb_filter.cuh)
    int nsamp;                // their count; 0: no filter
    int direct;               // set on the device: few candidates, decided without transforms (psb_filter.cuh)
    const int4* runs;         // device z-runs of the base item along source axis src_axis[2] (item_run)
    int nruns;
};

// A run of equal nonzero values along one source axis s of the base item:
// {u, v, r0 | r1 << 16, value}, u and v the coordinates along the other two
// source axes (u along the lower axis index), r0..r1 the range along s.
// oriented position (a, b) of the run's column and its z range c0..c1 for
// an orientation whose z axis comes from s (= d.src_axis[2]).
__device__ __forceinline__ void orient_run(const OrientDesc& d, int4 q, int* a, int* b, int* c0, int* c1) {
    const int s = d.src_axis[2];
    const int lo = s == 0 ? 1 : 0;          // the lower of the two other source axes
    const int va = d.src_axis[0] == lo ? q.x : q.y;
    const int vb = d.src_axis[1] == lo ? q.x : q.y;
    *a = d.flip[0] ? d.e[0] - 1 - va : va;
    *b = d.flip[1] ? d.e[1] - 1 - vb : vb;
    const int r0 = q.z & 0xffff, r1 = q.z >> 16;
    *c0 = d.flip[2] ? d.e[2] - 1 - r1 : r0;
    *c1 = d.flip[2] ? d.e[2] - 1 - r0 : r1;
}

// Prefix sums along z of every tray column: P[col * (nz + 1) + k] is the sum
// over z < k of the column's distance values (MODE 0) or of its occupied
// cells (MODE 1), so a run [c0, c1] of an item placed at height z collects
// P[z + c1 + 1] - P[z + c0].  One warp per column (a shuffle scan per 32
// cells).
template <int MODE>
__device__ __forceinline__ void col_prefix(const int32_t* __restrict__ src, int32_t* __restrict__ P, int nz,
                                           int lane) {
    int carry = 0;
    if (lane == 0) P[0] = 0;
    for (int z0 = 0; z0 < nz; z0 += 32) {
        const int z = z0 + lane;
        int v = 0;
        if (z < nz) v = MODE == 0 ? src[z] : (src[z] != 0 ? 1 : 0);
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, d);
            if (lane >= d) v += u;
        }
        if (z < nz) P[z + 1] = carry + v;
        carry += __shfl_sync(0xffffffffu, v, 31);
    }
}

// every column; gated on *gate when given.  grid: ceil(ncols / 8), block 256
template <int MODE>
__global__ void k_col_prefix(const int32_t* __restrict__ src, int32_t* __restrict__ P, int ncols, int nz,
                             const int* gate) {
    pdl_enter();
    if (gate && !*gate) return;
    const int col = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (col >= ncols) return;
    col_prefix<MODE>(src + (size_t)col * nz, P + (size_t)col * (nz + 1), nz, threadIdx.x & 31);
}

__device__ __forceinline__ int orient_src_index(const OrientDesc& d, int i0, int i1, int i2) {
    int o[3] = {i0, i1, i2};
    int s[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int v = d.flip[a] ? (d.e[a] - 1 - o[a]) : o[a];
        s[d.src_axis[a]] = v;
    }
    return (s[0] * d.b[1] + s[1]) * d.b[2] + s[2];
}

// oriented coordinates of a base voxel (inverse of the map above)
__device__ __forceinline__ void orient_voxel(const OrientDesc& d, int bx, int by, int bz, int* o) {
    int s[3] = {bx, by, bz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int v = s[d.src_axis[a]];
        o[a] = d.flip[a] ? (d.e[a] - 1 - v) : v;
    }
}

struct RzDesc {
    int kind;                 // SrcKind
    const int32_t* grid;      // SRC_GRID_*: (n0, n1, n2) grid
    int n0, n1, n2;           // lines = n0*n1 of length n2 (<= Fz)
    int sub;                  // SRC_GRID_SUB: value - sub
    int orient;               // SRC_ITEM: index into OrientDesc array
    float2* out;              // [n0*n1][Hz]
    const int* gate;          // when set, the transform runs only if *gate != 0
    const int* subp;          // SRC_GRID_SUB: device-side shift (overrides sub)
};

// real lines -> half spectra along z.  Two real lines are packed into one
// complex transform and separated afterwards (works for odd Fz too).
// grid: (ceil(pairs / PSB_PAIRS), nbatch)
__global__ void __launch_bounds__(PSB_THREADS)
k_rfft_z(const RzDesc* __restrict__ descs, const OrientDesc* __restrict__ orients,
         AxisPlan plan, const float2* __restrict__ g_tw) {
    pdl_enter();
    extern __shared__ float2 sm[];
    const RzDesc d = descs[blockIdx.y];
    if (d.gate && !*d.gate) return;
    const int N = plan.n, Hz = N / 2 + 1;
    int n0 = d.n0, n1 = d.n1, n2 = d.n2;
    const int sub = d.subp ? *d.subp : d.sub;
    OrientDesc od;
    if (d.kind == SRC_ITEM) {
        od = orients[d.orient];
        if (od.skip) return;
        n0 = od.e[0]; n1 = od.e[1]; n2 = od.e[2];
    }
    const int nlines = n0 * n1;
    const int npairs = (nlines + 1) / 2;
    const int p0 = blockIdx.x * PSB_PAIRS;
    if (p0 >= npairs) return;
    const int np = min(PSB_PAIRS, npairs - p0);
    float2* tw = sm;
    float2* A = sm + N;
    float2* B = A + PSB_PAIRS * N;
    const int tid = threadIdx.x, nthr = blockDim.x;
    load_twiddles(tw, g_tw, N, tid, nthr);
    for (int idx = tid; idx < np * N; idx += nthr) {
        int p = idx / N, z = idx - p * N;
        int la = 2 * (p0 + p), lb = la + 1;
        float va = 0.f, vb = 0.f;
        if (z < n2) {
            if (d.kind == SRC_ITEM) {
                int i = la / n1, j = la - (la / n1) * n1;
                va = (float)od.item[orient_src_index(od, i, j, z)];
                if (lb < nlines) {
                    i = lb / n1; j = lb - i * n1;
                    vb = (float)od.item[orient_src_index(od, i, j, z)];
                }
            } else {
                int ra = d.grid[(size_t)la * n2 + z];
                int rb = lb < nlines ? d.grid[(size_t)lb * n2 + z] : 0;
                if (d.kind == SRC_GRID_OCC) { ra = ra != 0; rb = rb != 0; }
                else if (d.kind == SRC_GRID_SUB) { ra -= sub; rb = lb < nlines ? rb - sub : 0; }
                va = (float)ra;
                vb = (float)rb;
            }
        }
        A[p * N + z] = make_float2(va, vb);
    }
    __syncthreads();
    float2* R = smem_fft<-1>(A, B, np, N, plan, tw, tid, nthr);
    for (int idx = tid; idx < np * Hz; idx += nthr) {
        int p = idx / Hz, k = idx - p * Hz;
        float2 Zk = R[p * N + k];
        float2 Zn = R[p * N + (k == 0 ? 0 : N - k)];
        // X = (Zk + conj(Zn))/2 ; Y = (Zk - conj(Zn))/(2i)
        float2 X = make_float2(0.5f * (Zk.x + Zn.x), 0.5f * (Zk.y - Zn.y));
        float2 Y = make_float2(0.5f * (Zk.y + Zn.y), -0.5f * (Zk.x - Zn.x));
        int la = 2 * (p0 + p), lb = la + 1;
        d.out[(size_t)la * Hz + k] = X;
        if (lb < nlines) d.out[(size_t)lb * Hz + k] = Y;
    }
}

// half spectra along z -> real lines (two lines per complex transform),
// scaled, rounded to int32.  in: [lines][Hz]; out: [lines][n2] int32.
__global__ void __launch_bounds__(PSB_THREADS)
k_irfft_z_int(const float2* __restrict__ in, int32_t* __restrict__ out, int nlines, int n2,
              float scale, AxisPlan plan, const float2* __restrict__ g_tw) {
    pdl_enter();
    extern __shared__ float2 sm[];
    const int N = plan.n, Hz = N / 2 + 1;
    const int npairs = (nlines + 1) / 2;
    const int p0 = blockIdx.x * PSB_PAIRS;
    if (p0 >= npairs) return;
    const int np = min(PSB_PAIRS, npairs - p0);
    float2* tw = sm;
    float2* A = sm + N;
    float2* B = A + PSB_PAIRS * N;
    const int tid = threadIdx.x, nthr = blockDim.x;
    load_twiddles(tw, g_tw, N, tid, nthr);
    for (int idx = tid; idx < np * N; idx += nthr) {
        int p = idx / N, k = idx - p * N;
        int la = 2 * (p0 + p), lb = la + 1;
        bool hb = lb < nlines;
        float2 z;
        if (k < Hz) {
            float2 xa = in[(size_t)la * Hz + k];
            float2 xb = hb ? in[(size_t)lb * Hz + k] : make_float2(0.f, 0.f);
            z = make_float2(xa.x - xb.y, xa.y + xb.x);
        } else {
            float2 xa = in[(size_t)la * Hz + (N - k)];
            float2 xb = hb ? in[(size_t)lb * Hz + (N - k)] : make_float2(0.f, 0.f);
            z = make_float2(xa.x + xb.y, xb.x - xa.y);
        }
        A[p * N + k] = z;
    }
    __syncthreads();
    float2* R = smem_fft<1>(A, B, np, N, plan, tw, tid, nthr);
    for (int idx = tid; idx < np * n2; idx += nthr) {
        int p = idx / n2, z = idx - p * n2;
        int la = 2 * (p0 + p), lb = la + 1;
        float2 v = R[p * N + z];
        out[(size_t)la * n2 + z] = (int32_t)rintf(v.x * scale);
        if (lb < nlines) out[(size_t)lb * n2 + z] = (int32_t)rintf(v.y * scale);
    }
}

// ---------------------------------------------------------------------------
// strided-axis transform: element (a, l, c) of a [A][L][C] layout
// ---------------------------------------------------------------------------
struct MidDesc {
    const float2* in;
    float2* out;
    int A, C, Lin, Lout;
    long long in_sa, out_sa;
    int in_sl, out_sl;
    int orient;               // >= 0: take A/Lin from the orientation (item y pass)
    int pad;
    const int* gate;          // when set, the transform runs only if *gate != 0
};

// grid: (ceil(Cmax / PSB_TILE), Amax, nbatch)
template <int DIR>
__global__ void __launch_bounds__(PSB_THREADS)
k_fft_mid(const MidDesc* __restrict__ descs, const OrientDesc* __restrict__ orients, AxisPlan plan,
          const float2* __restrict__ g_tw) {
    pdl_enter();
    extern __shared__ float2 sm[];
    MidDesc d = descs[blockIdx.z];
    if (d.gate && !*d.gate) return;
    if (d.orient >= 0) {
        const OrientDesc& od = orients[d.orient];
        if (od.skip) return;
        d.A = od.e[0];
        d.Lin = od.e[1];
        d.in_sa = (long long)od.e[1] * d.C;  // item partials are [ex][ey][C]
    }
    const int a = blockIdx.y;
    const int c0 = blockIdx.x * PSB_TILE;
    if (a >= d.A || c0 >= d.C) return;
    const int N = plan.n, T = PSB_TILE, ls = N;
    float2* tw = sm;
    float2* A = sm + N;
    float2* B = A + T * ls;
    const int tid = threadIdx.x, nthr = blockDim.x;
    load_twiddles(tw, g_tw, N, tid, nthr);
    const float2* in = d.in + (size_t)a * d.in_sa;
    for (int idx = tid; idx < T * N; idx += nthr) {
        int l = idx / T, cl = idx - l * T;
        int c = c0 + cl;
        float2 v = make_float2(0.f, 0.f);
        if (l < d.Lin && c < d.C) v = in[(size_t)l * d.in_sl + c];
        A[cl * ls + l] = v;
    }
    __syncthreads();
    float2* R = smem_fft<DIR>(A, B, T, ls, plan, tw, tid, nthr);
    float2* out = d.out + (size_t)a * d.out_sa;
    for (int idx = tid; idx < T * d.Lout; idx += nthr) {
        int l = idx / T, cl = idx - l * T;
        int c = c0 + cl;
        if (c < d.C) out[(size_t)l * d.out_sl + c] = R[cl * ls + l];
    }
}

// elementwise spectrum product for the stateless correlation / convolution:
// out = conj(b) * a (corr) or a * b (conv)
__global__ void k_spec_mul(const float2* __restrict__ a, const float2* __restrict__ b, float2* __restrict__ out,
                           size_t n, int conj_b) {
    pdl_enter();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float2 x = a[i], y = b[i];
        out[i] = conj_b ? c_cmul(y, x) : c_mul(x, y);
    }
}

// ---------------------------------------------------------------------------
// fused x pass of the search: item forward along x, products with the tray's
// occupancy and distance spectra, inverse along x for both.
// Replaces per orientation: padded item FFT (fft3.cu:1269), two
// element_wise_cmplx_mul (fft3.cu:1274) and the first inverse stage.
// in : Bi[o] = item spectrum after z,y passes, [ex][Fy][Hz]
// out: Pc[o], Pd[o] = [Xv][Fy][Hz]
// grid: (ceil(Hz / PSB_TILE), Fy, n_orient)
// ---------------------------------------------------------------------------
struct SearchBufs {
    float2* Bi;          // per orientation stride sB
    float2* Pc;          // per orientation stride sP
    float2* Pd;
    long long sB, sP;
    // work counters of the transform kernels (algorithmic bytes of the
    // measurement), or null: collision [0] x-pass orientations, [1] their item
    // rows ex, [2] their stored product planes, [3] plane-pass planes, [4]
    // their row pairs; proximity [5] x-pass orientations, [6] their stored
    // planes (= plane-pass planes), [7] plane-pass row pairs
    unsigned long long* work;
    // when set: the orientations to work on (k_active_list), *nact of them;
    // CTA row y takes act[y], act[y + gridDim.y], ... instead of orientation y
    const int* act;
    const int* nact;
};

// The orientations a search's transforms work on (act: neither skipped nor
// decided directly) and the ones it searches at all (srch: not skipped; the
// flood fill and the selection), compacted, so those kernels launch a few
// CTA rows that loop over them instead of one row per orientation, most of
// which would only read their descriptor and exit.  vcount, when given,
// first applies the candidate filter's verification (stage 1 of
// k_cand_apply, one launch less): a direct orientation without a verified
// free cell is skipped.  grid 1, block 32
__global__ void k_active_list(OrientDesc* __restrict__ od, int n, int* __restrict__ act, int* __restrict__ nact,
                              int* __restrict__ srch, int* __restrict__ nsrch, const int* __restrict__ vcount) {
    pdl_enter();
    int base = 0, sbase = 0;
    const unsigned int below = (1u << threadIdx.x) - 1u;
    for (int o0 = 0; o0 < n; o0 += 32) {
        const int o = o0 + threadIdx.x;
        if (vcount && o < n && !od[o].skip && od[o].direct && vcount[o] == 0) od[o].skip = 1;
        const bool s = o < n && !od[o].skip;
        const bool on = s && !od[o].direct;
        const unsigned int b = __ballot_sync(0xffffffffu, on);
        const unsigned int bs = __ballot_sync(0xffffffffu, s);
        if (on) act[base + __popc(b & below)] = o;
        if (s) srch[sbase + __popc(bs & below)] = o;
        base += __popc(b);
        sbase += __popc(bs);
    }
    if (threadIdx.x == 0) {
        *nact = base;
        *nsrch = sbase;
    }
}

__global__ void __launch_bounds__(PSB_THREADS)
k_xpass(const OrientDesc* __restrict__ orients, SearchBufs sb, const float2* __restrict__ Socc,
        const float2* __restrict__ Sphi, int Fy, int Hz, AxisPlan plan, const float2* __restrict__ g_tw) {
    pdl_enter();
    extern __shared__ float2 sm[];
    const int o = blockIdx.z;
    const OrientDesc& od = orients[o];
    if (od.skip || od.valid[0] <= 0) return;
    const int ky = blockIdx.y;
    const int c0 = blockIdx.x * PSB_TILE;
    const int N = plan.n, T = PSB_TILE, ls = N;
    float2* tw = sm;
    float2* A = sm + N;            // 2T lines
    float2* B = A + 2 * T * ls;    // 2T lines
    const int tid = threadIdx.x, nthr = blockDim.x;
    load_twiddles(tw, g_tw, N, tid, nthr);
    const int ex = od.e[0];
    const float2* Bi = sb.Bi + (size_t)o * sb.sB;
    const size_t rowstride = (size_t)Fy * Hz;
    for (int idx = tid; idx < T * N; idx += nthr) {
        int x = idx / T, cl = idx - x * T;
        int kz = c0 + cl;
        float2 v = make_float2(0.f, 0.f);
        if (x < ex && kz < Hz) v = Bi[(size_t)x * rowstride + (size_t)ky * Hz + kz];
        A[cl * ls + x] = v;
    }
    __syncthreads();
    float2* R = smem_fft<-1>(A, B, T, ls, plan, tw, tid, nthr);
    float2* Q = (R == A) ? B : A;
    for (int idx = tid; idx < T * N; idx += nthr) {
        int kx = idx / T, cl = idx - kx * T;
        int kz = c0 + cl;
        float2 pc = make_float2(0.f, 0.f), pd = pc;
        if (kz < Hz) {
            size_t g = (size_t)kx * rowstride + (size_t)ky * Hz + kz;
            float2 it = R[cl * ls + kx];
            pc = c_cmul(it, Socc[g]);
            pd = c_cmul(it, Sphi[g]);
        }
        Q[cl * ls + kx] = pc;
        Q[(T + cl) * ls + kx] = pd;
    }
    __syncthreads();
    float2* R2 = smem_fft<1>(Q, R, 2 * T, ls, plan, tw, tid, nthr);
    const int Xv = od.valid[0];
    float2* Pc = sb.Pc + (size_t)o * sb.sP;
    float2* Pd = sb.Pd + (size_t)o * sb.sP;
    for (int idx = tid; idx < T * Xv; idx += nthr) {
        int x = idx / T, cl = idx - x * T;
        int kz = c0 + cl;
        if (kz < Hz) {
            size_t g = (size_t)x * rowstride + (size_t)ky * Hz + kz;
            Pc[g] = R2[cl * ls + x];
            Pd[g] = R2[(T + cl) * ls + x];
        }
    }
}

// ordered encoding of doubles for atomicMin on unsigned long long
__device__ __forceinline__ unsigned long long ord_key(double v) {
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ __forceinline__ double ord_val(unsigned long long k) {
    unsigned long long b = (k & 0x8000000000000000ULL) ? (k & 0x7fffffffffffffffULL) : ~k;
    return __longlong_as_double((long long)b);
}

struct ScoreParams {
    int nx, ny, nz;
    int mode;                 // PSB_MODE_SCAN / PSB_MODE_BLOCK
    const double* pen;        // SCAN: P*pow(k/nz,3) per k (host libm)
    const double* qa;         // BLOCK: (P*qz)*qz per k, qz = k/nz (IEEE, host)
    const double* qz;         // BLOCK: qz per k
    float scale;              // 1/(Fx*Fy*Fz)
    int nzw;                  // 32-bit words per (x,y) line of bit masks
};

// score of the reference for proximity value D at height k:
//   SCAN  packing.cpp:630-631  prox + P*pow(k/nz,3)          (plain add)
//   BLOCK fft3.cu:172-173      prox + P*qz*qz*qz, the last multiply-add fused
__device__ __forceinline__ double ref_score(const ScoreParams& sp, double D, int k) {
    if (sp.mode == 0) return __dadd_rn(D, __ldg(&sp.pen[k]));
    return __fma_rn(__ldg(&sp.qa[k]), __ldg(&sp.qz[k]), D);
}

struct PlaneBufs {
    uint32_t* freebits;       // per orientation [nx*ny][nzw]
    float* Dq;                // per orientation [nx*ny*nz]: D~ - base
    unsigned long long* smin; // per orientation approx min score key
    unsigned int* diag;       // per orientation diag bits
    long long sBits, sD;
    unsigned long long* pmin; // per (orientation, x plane) approx min score key over ok cells
    long long pstride;        // pmin / okplane stride per orientation
    const uint32_t* okbits;   // k_plane3 field 1: cells that count (free, or reachable)
    unsigned char* okplane;   // k_plane3: per (orientation, x plane) "has an ok cell"
    int set_okplane;          // k_plane3 field 0 sets okplane from the free cells
    const unsigned char* candplane;  // k_plane3 field 0: per (orientation, x plane) "holds a candidate"
                                     // (k_cand_filter wrote the candidate words); null: no filter ran
    int* okcount;             // k_plane3 field 0 with set_okplane: free cells per orientation (or null)
};

// Per (x-plane, orientation): inverse along y, C2R along z for the collision
// field then the proximity field; writes free bits (collision rounds to 0 and
// translation valid) and the approximate proximity.  Replaces the inverse FFT
// (fft3.cu:1277), scale/round/extract (1280-1283), truncate_flip (1290) and
// compute_scores_kernel (147-175).
// grid: (nx, n_orient)
__global__ void __launch_bounds__(PSB_THREADS)
k_plane(const OrientDesc* __restrict__ orients, SearchBufs sb, PlaneBufs pb, ScoreParams sp, int Fy, int Fz,
        AxisPlan py, AxisPlan pz, const float2* __restrict__ g_twy, const float2* __restrict__ g_twz) {
    pdl_enter();
    extern __shared__ float2 sm[];
    const int o = blockIdx.y;
    const OrientDesc& od = orients[o];
    if (od.skip) return;
    const int x = blockIdx.x;
    const int Xv = od.valid[0], Yv = od.valid[1], Zv = od.valid[2];
    if (x >= Xv || Yv <= 0 || Zv <= 0) return;
    const int Hz = Fz / 2 + 1;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int T = PSB_TILE;
    // smem: twy[Fy] twz[Fz] Q[Yv][Hz] work A/B [max(T*Fy, 2*PSB_PAIRS... )] bits[Yv*nzw]
    float2* twy = sm;
    float2* twz = twy + Fy;
    float2* Q = twz + Fz;
    const int wsz = max(T * Fy, PSB_PAIRS * Fz);
    float2* A = Q + (size_t)Yv * Hz;
    float2* B = A + wsz;
    uint32_t* bits = (uint32_t*)(B + wsz);
    const int nzw = sp.nzw;
    load_twiddles(twy, g_twy, Fy, tid, nthr);
    load_twiddles(twz, g_twz, Fz, tid, nthr);
    for (int i = tid; i < Yv * nzw; i += nthr) bits[i] = 0u;
    const size_t rowstride = (size_t)Fy * Hz;
    const float scale = sp.scale;
    double local_min = 1e300;
    unsigned int diag = 0;
    float* Dq = pb.Dq + (size_t)o * pb.sD;
    for (int field = 0; field < 2; ++field) {
        const float2* P = (field == 0 ? sb.Pc : sb.Pd) + (size_t)o * sb.sP + (size_t)x * rowstride;
        // inverse along y, column chunks of T
        for (int c0 = 0; c0 < Hz; c0 += T) {
            __syncthreads();
            for (int idx = tid; idx < T * Fy; idx += nthr) {
                int l = idx / T, cl = idx - l * T;
                int kz = c0 + cl;
                A[cl * Fy + l] = kz < Hz ? P[(size_t)l * Hz + kz] : make_float2(0.f, 0.f);
            }
            __syncthreads();
            float2* R = smem_fft<1>(A, B, T, Fy, py, twy, tid, nthr);
            for (int idx = tid; idx < T * Yv; idx += nthr) {
                int y = idx / T, cl = idx - y * T;
                int kz = c0 + cl;
                if (kz < Hz) Q[(size_t)y * Hz + kz] = R[cl * Fy + y];
            }
        }
        // C2R along z, two rows per complex transform
        const int npairs = (Yv + 1) / 2;
        for (int q0 = 0; q0 < npairs; q0 += PSB_PAIRS) {
            const int np = min(PSB_PAIRS, npairs - q0);
            __syncthreads();
            for (int idx = tid; idx < np * Fz; idx += nthr) {
                int p = idx / Fz, k = idx - p * Fz;
                int ya = 2 * (q0 + p), yb = ya + 1;
                bool hb = yb < Yv;
                float2 z;
                if (k < Hz) {
                    float2 xa = Q[(size_t)ya * Hz + k];
                    float2 xb = hb ? Q[(size_t)yb * Hz + k] : make_float2(0.f, 0.f);
                    z = make_float2(xa.x - xb.y, xa.y + xb.x);
                } else {
                    float2 xa = Q[(size_t)ya * Hz + (Fz - k)];
                    float2 xb = hb ? Q[(size_t)yb * Hz + (Fz - k)] : make_float2(0.f, 0.f);
                    z = make_float2(xa.x + xb.y, xb.x - xa.y);
                }
                A[p * Fz + k] = z;
            }
            __syncthreads();
            float2* R = smem_fft<1>(A, B, np, Fz, pz, twz, tid, nthr);
            for (int idx = tid; idx < np * 2 * Zv; idx += nthr) {
                int p = idx / (2 * Zv), r = idx - p * 2 * Zv;
                int half = r / Zv, z = r - half * Zv;
                int y = 2 * (q0 + p) + half;
                if (y >= Yv) continue;
                float2 v = R[p * Fz + z];
                float val = (half ? v.y : v.x) * scale;
                if (field == 0) {
                    float rv = rintf(val);
                    if (rv == 0.f) atomicOr(&bits[y * nzw + (z >> 5)], 1u << (z & 31));
                    if (fabsf(val - rv) > 0.25f) diag |= 2u;
                } else {
                    bool fr = (bits[y * nzw + (z >> 5)] >> (z & 31)) & 1u;
                    size_t t = ((size_t)x * sp.ny + y) * sp.nz + z;
                    Dq[t] = val;
                    if (fr) {
                        double s = ref_score(sp, od.base + (double)val, z);
                        local_min = fmin(local_min, s);
                    }
                }
            }
        }
        __syncthreads();
    }
    // write free bits of this plane
    uint32_t* fb = pb.freebits + (size_t)o * pb.sBits + (size_t)x * sp.ny * nzw;
    for (int i = tid; i < Yv * nzw; i += nthr) fb[i] = bits[i];
    // block min
    __shared__ double red[PSB_THREADS / 32];
    for (int off = 16; off > 0; off >>= 1) local_min = fmin(local_min, __shfl_xor_sync(0xffffffffu, local_min, off));
    if ((tid & 31) == 0) red[tid >> 5] = local_min;
    unsigned int dg = __reduce_or_sync(0xffffffffu, diag);
    if ((tid & 31) == 0 && dg) atomicOr(&pb.diag[o], dg);
    __syncthreads();
    if (tid == 0) {
        double m = red[0];
        for (int w = 1; w < nthr / 32; ++w) m = fmin(m, red[w]);
        pb.pmin[(size_t)o * pb.pstride + x] = m < 1e299 ? ord_key(m) : 0xffffffffffffffffULL;
        if (m < 1e299) atomicMin(&pb.smin[o], ord_key(m));
    }
}
