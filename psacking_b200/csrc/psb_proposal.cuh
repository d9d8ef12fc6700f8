// psb_proposal.cuh — the learned orientation proposal: a small 3-D CNN that
// ranks an item's orientations before the exact search.
//
// Network (parameters in one flat FP32 master vector, BF16 copies of the
// weights for the forward and backward passes, FP32 accumulation):
//   item branch, per orientation, 32^3 occupancy grid:
//     conv3d 1->16, 16->32, 32->64, 64->64 (kernel 3, stride 2, padding 1,
//     ReLU) -> 64 x 2^3 = 512 -> linear 512->64, ReLU
//   tray branch, per item, 32x32 pooled height map: linear 1024->64, ReLU
//   head, per orientation: [item 64 | tray 64] -> linear 128->64, ReLU ->
//     linear 64->1 = logit
// Loss: masked softmax cross-entropy over an item's orientations against a
// soft target from the plain search (weight 2^-rank by exact score among the
// orientations that fit somewhere), mean over the items that have one.
// Training and inference use the same kernels; the packing loop runs the
// forward pass on the device and keeps only the top-k orientations (all of
// them when the top-k probability mass is below a margin).
// No counterpart in the reference: the learned-proposal form is an addition.
#pragma once
#include <stdint.h>

#include "psb_pdl.cuh"

#define PSB_PG 32          // item grid side
#define PSB_PG3 (PSB_PG * PSB_PG * PSB_PG)
#define PSB_PH 32          // pooled height-map side
#define PSB_PNO 24         // orientations per item in the network's output

// BF16 storage as uint16 (round to nearest even; inputs are finite)
__host__ __device__ __forceinline__ uint16_t bf16_bits(float f) {
#ifdef __CUDA_ARCH__
    uint32_t u = __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
#endif
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
__device__ __forceinline__ float bf16_val(uint16_t h) { return __uint_as_float((uint32_t)h << 16); }

// ---------------------------------------------------------------------------
// inputs
// ---------------------------------------------------------------------------
// base grid of one item from its voxel list (the synchronous item-grid call;
// the packing loop uses k_base_grid_runs): cell floor(v / s) gains 1/s^3,
// s = ceil(max extent / 32).  grid: (ceil(nvox/256)), block 256; out zeroed
__global__ void k_base_grid(const int4* __restrict__ vox, int nvox, int s, float* __restrict__ out) {
    pdl_enter();
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    const int4 q = vox[v];
    if (q.w <= 0) return;
    const int i = q.x / s, j = q.y / s, k = q.z / s;
    atomicAdd(&out[(i * PSB_PG + j) * PSB_PG + k], 1.0f / (float)(s * s * s));
}

// the same base grid from the item's z-runs ({x, y, z0 | z1 << 16, value},
// one per run of equal nonzero values along z): the cells and weights of the
// voxel form.  grid: (ceil(nruns/256)), block 256; out zeroed
__global__ void k_base_grid_runs(const int4* __restrict__ runs, int nruns, int s, float* __restrict__ out) {
    pdl_enter();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nruns) return;
    const int4 q = runs[r];
    if (q.w <= 0) return;
    const float w = 1.0f / (float)(s * s * s);
    const int i = q.x / s, j = q.y / s, z1 = q.z >> 16;
    for (int z = q.z & 0xffff; z <= z1; ++z) atomicAdd(&out[(i * PSB_PG + j) * PSB_PG + z / s], w);
}

// oriented grids: out[b*no + o] = the base grid of item b turned by map o
// (src_axis[3], flip[3]) within its scaled extent G (cells per axis).
// grid: (PSB_PG3 / 256, no, B), block 256
__global__ void k_orient_grids(const float* __restrict__ base, const int* __restrict__ G, const int* __restrict__ maps,
                               int no, float* __restrict__ out) {
    pdl_enter();
    const int b = blockIdx.z, o = blockIdx.y;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= PSB_PG3) return;
    const int* m = maps + 6 * o;
    const int ijk[3] = {c / (PSB_PG * PSB_PG), (c / PSB_PG) % PSB_PG, c % PSB_PG};
    int src[3];
    float v = 0.f;
    bool in = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int sa = m[a];
        const int ga = G[3 * b + sa];
        if (ijk[a] >= ga) in = false;
        src[sa] = m[3 + a] ? ga - 1 - ijk[a] : ijk[a];
    }
    if (in) v = base[(size_t)b * PSB_PG3 + (src[0] * PSB_PG + src[1]) * PSB_PG + src[2]];
    out[((size_t)b * no + o) * PSB_PG3 + c] = v;
}

// pooled height map: per column 1 + highest occupied z (0 when empty), over
// nz, averaged over ceil(nx/32) x ceil(ny/32) blocks.  One CTA per pooled
// cell, one warp per column at a time: lanes read 32 consecutive z from the
// top down and a ballot finds the highest occupied one.
// grid: 1024, block 256
__global__ void k_height_map(const int32_t* __restrict__ tray, int nx, int ny, int nz, float* __restrict__ out) {
    pdl_enter();
    const int cell = blockIdx.x;  // 0..1023
    const int ci = cell / PSB_PH, cj = cell % PSB_PH;
    const int bx = (nx + PSB_PH - 1) / PSB_PH, by = (ny + PSB_PH - 1) / PSB_PH;
    const int x0 = ci * bx, y0 = cj * by;
    const int x1 = min(nx, x0 + bx), y1 = min(ny, y0 + by);
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nwp = blockDim.x >> 5;
    __shared__ float red[8];
    __shared__ int cnt[8];
    float acc = 0.f;
    int n = 0;
    const int w = max(0, y1 - y0);
    const int ncol = max(0, x1 - x0) * w;
    for (int c = wp; c < ncol; c += nwp) {
        const int x = x0 + c / w, y = y0 + c % w;
        const int32_t* col = tray + ((size_t)x * ny + y) * nz;
        int top = 0;
        for (int zb = ((nz - 1) / 32) * 32; zb >= 0; zb -= 32) {
            const int z = zb + lane;
            const unsigned int bal = __ballot_sync(0xffffffffu, z < nz && col[z] > 0);
            if (bal) {
                top = zb + 32 - __clz(bal);
                break;
            }
        }
        acc += (float)top / (float)nz;
        ++n;
    }
    if (lane == 0) {
        red[wp] = acc;
        cnt[wp] = n;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        int k = 0;
        for (int i = 0; i < nwp; ++i) { s += red[i]; k += cnt[i]; }
        out[cell] = k ? s / (float)k : 0.f;
    }
}

// ---------------------------------------------------------------------------
// convolution, kernel 3, stride 2, padding 1 (activations [S][C][D^3])
// ---------------------------------------------------------------------------
// forward with ReLU; each thread computes one output voxel for PSB_CPT
// consecutive output channels, so every input value it loads feeds PSB_CPT
// multiply-adds.  grid: (ceil(S*Do^3/256), Co/PSB_CPT), block 256;
// smem PSB_CPT*Ci*27 floats
#define PSB_CPT 4
__global__ void k_conv_fwd(const float* __restrict__ in, int S, int Ci, int D, const uint16_t* __restrict__ w,
                           const float* __restrict__ bias, float* __restrict__ out, int Co) {
    pdl_enter();
    extern __shared__ float ws[];   // [PSB_CPT][Ci*27]
    const int c0 = blockIdx.y * PSB_CPT;
    for (int i = threadIdx.x; i < PSB_CPT * Ci * 27; i += blockDim.x) {
        const int c = i / (Ci * 27), r = i % (Ci * 27);
        ws[i] = bf16_val(w[(size_t)(c0 + c) * Ci * 27 + r]);
    }
    __syncthreads();
    const int Do = D / 2, Do3 = Do * Do * Do, D3 = D * D * D;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)S * Do3) return;
    const int s = (int)(idx / Do3), r = (int)(idx % Do3);
    const int od = r / (Do * Do), oh = (r / Do) % Do, ow = r % Do;
    float acc[PSB_CPT];
#pragma unroll
    for (int c = 0; c < PSB_CPT; ++c) acc[c] = bias[c0 + c];
    for (int ci = 0; ci < Ci; ++ci) {
        const float* x = in + ((size_t)s * Ci + ci) * D3;
        const float* wc = ws + ci * 27;
#pragma unroll
        for (int kd = 0; kd < 3; ++kd) {
            const int id = 2 * od - 1 + kd;
            if (id < 0 || id >= D) continue;
#pragma unroll
            for (int kh = 0; kh < 3; ++kh) {
                const int ih = 2 * oh - 1 + kh;
                if (ih < 0 || ih >= D) continue;
#pragma unroll
                for (int kw = 0; kw < 3; ++kw) {
                    const int iw = 2 * ow - 1 + kw;
                    if (iw < 0 || iw >= D) continue;
                    const float xv = x[(id * D + ih) * D + iw];
                    const int t = kd * 9 + kh * 3 + kw;
#pragma unroll
                    for (int c = 0; c < PSB_CPT; ++c) acc[c] = fmaf(xv, wc[c * Ci * 27 + t], acc[c]);
                }
            }
        }
    }
#pragma unroll
    for (int c = 0; c < PSB_CPT; ++c) out[((size_t)s * Co + c0 + c) * Do3 + r] = fmaxf(acc[c], 0.f);
}

// gradient w.r.t. the input, times the ReLU mask of that input (the previous
// layer's output; mask_relu = 0 for the network input).
// grid: (ceil(S*D^3/256), Ci), block 256; smem Co*27 floats
__global__ void k_conv_bwd_data(const float* __restrict__ dout, int S, int Ci, int D, const uint16_t* __restrict__ w,
                                int Co, const float* __restrict__ in, int mask_relu, float* __restrict__ din) {
    pdl_enter();
    extern __shared__ float ws[];
    const int ci = blockIdx.y;
    for (int i = threadIdx.x; i < Co * 27; i += blockDim.x) {
        const int co = i / 27, t = i % 27;
        ws[i] = bf16_val(w[((size_t)co * Ci + ci) * 27 + t]);
    }
    __syncthreads();
    const int Do = D / 2, Do3 = Do * Do * Do, D3 = D * D * D;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)S * D3) return;
    const int s = (int)(idx / D3), r = (int)(idx % D3);
    const int id = r / (D * D), ih = (r / D) % D, iw = r % D;
    float acc = 0.f;
    // od = (id + 1 - kd) / 2 for the kd of matching parity
    for (int kd = (id + 1) & 1; kd < 3; kd += 2) {
        const int od = (id + 1 - kd) >> 1;
        if (od < 0 || od >= Do) continue;
        for (int kh = (ih + 1) & 1; kh < 3; kh += 2) {
            const int oh = (ih + 1 - kh) >> 1;
            if (oh < 0 || oh >= Do) continue;
            for (int kw = (iw + 1) & 1; kw < 3; kw += 2) {
                const int ow = (iw + 1 - kw) >> 1;
                if (ow < 0 || ow >= Do) continue;
                const int t = kd * 9 + kh * 3 + kw;
                const float* g = dout + (size_t)s * Co * Do3 + (od * Do + oh) * Do + ow;
                for (int co = 0; co < Co; ++co) acc = fmaf(g[(size_t)co * Do3], ws[co * 27 + t], acc);
            }
        }
    }
    const size_t at = ((size_t)s * Ci + ci) * D3 + r;
    if (mask_relu && in[at] <= 0.f) acc = 0.f;
    din[at] = acc;
}

// gradient w.r.t. the weights and bias: each CTA sums a chunk of samples for
// one (co, ci) pair and adds its 27 partial sums (and the bias sum when ci ==
// 0) with atomics.  grid: (Ci, Co, nchunk), block 256; dw, db zeroed first
__global__ void k_conv_bwd_weight(const float* __restrict__ dout, const float* __restrict__ in, int S, int Ci, int D,
                                  int Co, int chunk, float* __restrict__ dw, float* __restrict__ db) {
    pdl_enter();
    const int ci = blockIdx.x, co = blockIdx.y;
    const int s0 = blockIdx.z * chunk, s1 = min(S, s0 + chunk);
    const int Do = D / 2, Do3 = Do * Do * Do, D3 = D * D * D;
    float acc[27];
#pragma unroll
    for (int t = 0; t < 27; ++t) acc[t] = 0.f;
    float bacc = 0.f;
    const long long n = (long long)(s1 - s0) * Do3;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        const int s = s0 + (int)(i / Do3), r = (int)(i % Do3);
        const int od = r / (Do * Do), oh = (r / Do) % Do, ow = r % Do;
        const float g = dout[((size_t)s * Co + co) * Do3 + r];
        if (g == 0.f) continue;
        bacc += g;
        const float* x = in + ((size_t)s * Ci + ci) * D3;
#pragma unroll
        for (int kd = 0; kd < 3; ++kd) {
            const int id = 2 * od - 1 + kd;
            if (id < 0 || id >= D) continue;
#pragma unroll
            for (int kh = 0; kh < 3; ++kh) {
                const int ih = 2 * oh - 1 + kh;
                if (ih < 0 || ih >= D) continue;
#pragma unroll
                for (int kw = 0; kw < 3; ++kw) {
                    const int iw = 2 * ow - 1 + kw;
                    if (iw < 0 || iw >= D) continue;
                    acc[kd * 9 + kh * 3 + kw] = fmaf(g, x[(id * D + ih) * D + iw], acc[kd * 9 + kh * 3 + kw]);
                }
            }
        }
    }
    __shared__ float red[8][28];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < 27; ++t) {
        float v = acc[t];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[wp][t] = v;
    }
    for (int off = 16; off > 0; off >>= 1) bacc += __shfl_xor_sync(0xffffffffu, bacc, off);
    if (lane == 0) red[wp][27] = bacc;
    __syncthreads();
    if (threadIdx.x < 28) {
        float v = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += red[k][threadIdx.x];
        if (threadIdx.x < 27) atomicAdd(&dw[((size_t)co * Ci + ci) * 27 + threadIdx.x], v);
        else if (ci == 0) atomicAdd(&db[co], v);
    }
}

// ---------------------------------------------------------------------------
// linear layers y[S][N] = x[S][K] W^T + b (W [N][K] BF16)
// ---------------------------------------------------------------------------
// forward; relu applied when relu != 0.  grid: ceil(S*N/256)
__global__ void k_lin_fwd(const float* __restrict__ x, int S, int K, const uint16_t* __restrict__ w,
                          const float* __restrict__ b, int N, int relu, float* __restrict__ y) {
    pdl_enter();
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)S * N) return;
    const int s = (int)(idx / N), n = (int)(idx % N);
    const float* xr = x + (size_t)s * K;
    const uint16_t* wr = w + (size_t)n * K;
    float acc = b[n];
    for (int k = 0; k < K; ++k) acc = fmaf(xr[k], bf16_val(wr[k]), acc);
    y[idx] = relu ? fmaxf(acc, 0.f) : acc;
}

// dx[S][K] = dy[S][N] W, times the ReLU mask of x when xmask != NULL.
// grid: ceil(S*K/256)
__global__ void k_lin_bwd_data(const float* __restrict__ dy, int S, int N, const uint16_t* __restrict__ w, int K,
                               const float* __restrict__ xmask, float* __restrict__ dx) {
    pdl_enter();
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)S * K) return;
    const int s = (int)(idx / K), k = (int)(idx % K);
    float acc = 0.f;
    for (int n = 0; n < N; ++n) acc = fmaf(dy[(size_t)s * N + n], bf16_val(w[(size_t)n * K + k]), acc);
    if (xmask && xmask[idx] <= 0.f) acc = 0.f;
    dx[idx] = acc;
}

// dW[N][K] = dy^T x, db[N] = sum_s dy.  grid: (ceil(K/256), N); the K == 0
// column of threads also sums the bias
__global__ void k_lin_bwd_weight(const float* __restrict__ dy, const float* __restrict__ x, int S, int N, int K,
                                 float* __restrict__ dw, float* __restrict__ db) {
    pdl_enter();
    const int n = blockIdx.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    float acc = 0.f, bacc = 0.f;
    for (int s = 0; s < S; ++s) {
        const float g = dy[(size_t)s * N + n];
        acc = fmaf(g, x[(size_t)s * K + k], acc);
        bacc += g;
    }
    dw[(size_t)n * K + k] = acc;
    if (k == 0) db[n] = bacc;
}

// head input: [f1[s] | t[s / no]] (64 + 64).  grid: ceil(S*128/256)
__global__ void k_concat(const float* __restrict__ f1, const float* __restrict__ t, int S, int no, float* __restrict__ hin) {
    pdl_enter();
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)S * 128) return;
    const int s = (int)(idx / 128), c = (int)(idx % 128);
    hin[idx] = c < 64 ? f1[(size_t)s * 64 + c] : t[(size_t)(s / no) * 64 + (c - 64)];
}

// split the head-input gradient: df1 = dhin[:, :64] * (f1 > 0);
// dt[b] = sum over its orientations of dhin[:, 64:] * (t > 0).  grid: ceil(S*64/256) and ceil(B*64/256)
__global__ void k_split_item(const float* __restrict__ dhin, const float* __restrict__ f1, int S,
                             float* __restrict__ df1) {
    pdl_enter();
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)S * 64) return;
    const int s = (int)(idx / 64), c = (int)(idx % 64);
    df1[idx] = f1[idx] > 0.f ? dhin[(size_t)s * 128 + c] : 0.f;
}
__global__ void k_split_tray(const float* __restrict__ dhin, const float* __restrict__ t, int B, int no,
                             float* __restrict__ dt) {
    pdl_enter();
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * 64) return;
    const int b = idx / 64, c = idx % 64;
    float acc = 0.f;
    for (int o = 0; o < no; ++o) acc += dhin[((size_t)b * no + o) * 128 + 64 + c];
    dt[idx] = t[idx] > 0.f ? acc : 0.f;
}

// masked softmax cross-entropy over each item's no logits, mean over the
// items that have a target and an unmasked orientation; loss accumulated in
// *loss (zeroed first), gradient written to dlogit.  One warp per item.
__global__ void k_softmax_ce(const float* __restrict__ logit, const float* __restrict__ target,
                             const float* __restrict__ mask, int B, int no, float* __restrict__ dlogit,
                             float* __restrict__ loss) {
    pdl_enter();
    const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    // items counted in the mean (the same for every warp)
    int nb = 0;
    for (int i = lane; i < B; i += 32) {
        float ts = 0.f, ms = 0.f;
        for (int o = 0; o < no; ++o) { ts += target[(size_t)i * no + o]; ms += mask[(size_t)i * no + o]; }
        nb += (ts > 0.f && ms > 0.f) ? 1 : 0;
    }
    nb = __reduce_add_sync(0xffffffffu, nb);
    if (b >= B) return;
    const float inv = 1.f / (float)max(1, nb);
    const bool m = lane < no && mask[(size_t)b * no + lane] > 0.f;
    const float z = m ? logit[(size_t)b * no + lane] : -INFINITY;
    float zmax = z;
    for (int off = 16; off > 0; off >>= 1) zmax = fmaxf(zmax, __shfl_xor_sync(0xffffffffu, zmax, off));
    const float e = m ? expf(z - zmax) : 0.f;
    float s = e;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    const float q = (lane < no) ? target[(size_t)b * no + lane] : 0.f;
    float qs = q;
    for (int off = 16; off > 0; off >>= 1) qs += __shfl_xor_sync(0xffffffffu, qs, off);
    int anym = __any_sync(0xffffffffu, m);
    const bool has = qs > 0.f && anym;
    float lterm = 0.f, g = 0.f;
    if (has && m) {
        const float p = e / s;
        lterm = -q * (z - zmax - logf(s));
        g = (p * qs - q) * inv;
    }
    if (lane < no) dlogit[(size_t)b * no + lane] = g;
    for (int off = 16; off > 0; off >>= 1) lterm += __shfl_xor_sync(0xffffffffu, lterm, off);
    if (lane == 0 && has) atomicAdd(loss, lterm * inv);
}

// Adam on the FP32 master vector; weights (flag 1) get their BF16 copy
// refreshed.  grid: ceil(n/256)
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       uint16_t* __restrict__ p16, const unsigned char* __restrict__ is_weight, long long n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
    pdl_enter();
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (is_weight[i]) p16[i] = bf16_bits(pi);
}

// ---------------------------------------------------------------------------
// per-item head in the packing loop (the item branch is precomputed for the
// whole run: it does not depend on the tray state)
// ---------------------------------------------------------------------------
// Tray features of one item: t[n] = relu(hmap . W2[n] + b2[n]), one CTA per
// output.  grid: 64, block 256
__global__ void k_prop_tray_feat(const float* __restrict__ hmap, const uint16_t* __restrict__ w2,
                                 const float* __restrict__ b2, float* __restrict__ t) {
    pdl_enter();
    const int n = blockIdx.x;
    float acc = 0.f;
    for (int k = threadIdx.x; k < PSB_PH * PSB_PH; k += blockDim.x)
        acc = fmaf(hmap[k], bf16_val(w2[(size_t)n * PSB_PH * PSB_PH + k]), acc);
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    __shared__ float red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float v = b2[n];
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v += red[i];
        t[n] = fmaxf(v, 0.f);
    }
}

// Head of one item: per orientation o (one CTA), h1 = relu([f1_o | t] H1^T +
// bh1) (64 threads) and logit_o = h1 . H2 + bh2.  grid: no, block 64
__global__ void k_prop_item_head(const float* __restrict__ f1, const float* __restrict__ t,
                                 const uint16_t* __restrict__ wh1, const float* __restrict__ bh1,
                                 const uint16_t* __restrict__ wh2, const float* __restrict__ bh2,
                                 float* __restrict__ logit) {
    pdl_enter();
    const int o = blockIdx.x, n = threadIdx.x;
    __shared__ float in[128];
    __shared__ float red[2];
    in[n] = f1[(size_t)o * 64 + n];
    in[64 + n] = t[n];
    __syncthreads();
    const uint16_t* wr = wh1 + (size_t)n * 128;
    float acc = bh1[n];
    for (int k = 0; k < 128; ++k) acc = fmaf(in[k], bf16_val(wr[k]), acc);
    float v = fmaxf(acc, 0.f) * bf16_val(wh2[n]);
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((n & 31) == 0) red[n >> 5] = v;
    __syncthreads();
    if (n == 0) logit[o] = red[0] + red[1] + bh2[0];
}

// ---------------------------------------------------------------------------
// gating in the packing loop
// ---------------------------------------------------------------------------
// Keep the top-k orientations of one item by logit (ties: lower index), all
// of them when their softmax mass over the fitting orientations is below
// `margin`; the others are marked skipped for the search.  Orientations the
// tray cannot hold are skipped already.  One warp.
template <class OD>
__global__ void k_gate(const float* __restrict__ logit, OD* __restrict__ od, int n, int topk, float margin,
                       int* __restrict__ stats) {
    pdl_enter();
    const int lane = threadIdx.x;
    if (lane >= 32) return;
    const bool fit = lane < n && !od[lane].skip;
    const float z = fit ? logit[lane] : -INFINITY;
    float zmax = z;
    for (int off = 16; off > 0; off >>= 1) zmax = fmaxf(zmax, __shfl_xor_sync(0xffffffffu, zmax, off));
    const float e = fit ? expf(z - zmax) : 0.f;
    float s = e;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    // rank of this orientation: how many fitting orientations beat it
    int rank = 0;
    for (int j = 0; j < 32; ++j) {
        const float zj = __shfl_sync(0xffffffffu, z, j);
        const bool fj = __shfl_sync(0xffffffffu, (int)fit, j) != 0;
        if (fj && (zj > z || (zj == z && j < lane))) ++rank;
    }
    const bool keep = fit && rank < topk;
    float mass = keep ? e / s : 0.f;
    for (int off = 16; off > 0; off >>= 1) mass += __shfl_xor_sync(0xffffffffu, mass, off);
    const bool fallback = mass < margin;
    if (fit && !keep && !fallback) od[lane].skip = 1;
    if (lane == 0 && stats) {
        atomicAdd(&stats[0], 1);
        if (fallback) atomicAdd(&stats[1], 1);
    }
}
