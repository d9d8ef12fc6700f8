// psb_fft.cuh — shared-memory mixed-radix FFT building blocks for sm_100a.
//
// Lines of length N (N = 2^a 3^b 5^c 7^d, N <= PSB_MAX_FFT) live in shared
// memory as float2.  A Stockham auto-sort pass per radix (8, 4, 2, 3, 5, 7)
// reads one buffer and writes the other, so no bit-reversal pass is needed.
// Twiddles come from a table of exp(-2*pi*i*n/N) computed on the host in
// double precision and staged in shared memory by each CTA.
//
// The transforms replace the cuFFT C2C plans of the reference
// (spectral_packing/fft3.cu:1152, 1162, 1168, 1209, 1217, 1269, 1277).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "psb_pdl.cuh"

#define PSB_MAX_FFT 512
#define PSB_MAX_STAGES 12

struct AxisPlan {
    int n;                         // transform length
    int nstages;                   // number of radix passes
    int radix[PSB_MAX_STAGES];     // radix of each pass, applied in order
};

__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 c_mulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// conj(a) * b
__device__ __forceinline__ float2 c_cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float2 c_scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (DIR=-1, forward) or +i (DIR=+1, inverse)
template <int DIR>
__device__ __forceinline__ float2 c_rot(float2 a) {
    return DIR < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

// ---- small DFT kernels (DIR = -1: exp(-2 pi i jk/R), DIR = +1: exp(+...)) ----
template <int DIR>
__device__ __forceinline__ void dft2(float2* v) {
    float2 a = v[0], b = v[1];
    v[0] = c_add(a, b);
    v[1] = c_sub(a, b);
}

template <int DIR>
__device__ __forceinline__ void dft4(float2* v) {
    float2 t0 = c_add(v[0], v[2]), t1 = c_sub(v[0], v[2]);
    float2 t2 = c_add(v[1], v[3]), t3 = c_rot<DIR>(c_sub(v[1], v[3]));
    v[0] = c_add(t0, t2);
    v[2] = c_sub(t0, t2);
    v[1] = c_add(t1, t3);
    v[3] = c_sub(t1, t3);
}

template <int DIR>
__device__ __forceinline__ void dft8(float2* v) {
    const float r = 0.7071067811865476f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    dft4<DIR>(e);
    dft4<DIR>(o);
    // w8^k = exp(DIR * 2 pi i k / 8)
    float2 o1 = make_float2(r * (o[1].x - DIR * o[1].y), r * (o[1].y + DIR * o[1].x));
    float2 o2 = c_rot<DIR>(o[2]);
    float2 o3 = make_float2(r * (-o[3].x - DIR * o[3].y), r * (-o[3].y + DIR * o[3].x));
    v[0] = c_add(e[0], o[0]);
    v[4] = c_sub(e[0], o[0]);
    v[1] = c_add(e[1], o1);
    v[5] = c_sub(e[1], o1);
    v[2] = c_add(e[2], o2);
    v[6] = c_sub(e[2], o2);
    v[3] = c_add(e[3], o3);
    v[7] = c_sub(e[3], o3);
}

template <int DIR>
__device__ __forceinline__ void dft3(float2* v) {
    const float s = 0.8660254037844386f;
    float2 t1 = c_add(v[1], v[2]);
    float2 t2 = c_sub(v[1], v[2]);
    float2 m = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    float2 n = c_rot<DIR>(c_scale(t2, s));
    v[0] = c_add(v[0], t1);
    v[1] = c_add(m, n);
    v[2] = c_sub(m, n);
}

template <int DIR>
__device__ __forceinline__ void dft5(float2* v) {
    const float c1 = 0.30901699437494745f, c2 = -0.8090169943749473f;
    const float s1 = 0.9510565162951535f, s2 = 0.5877852522924732f;
    float2 t1 = c_add(v[1], v[4]), t2 = c_add(v[2], v[3]);
    float2 t3 = c_sub(v[1], v[4]), t4 = c_sub(v[2], v[3]);
    float2 a0 = v[0];
    float2 m1 = make_float2(a0.x + c1 * t1.x + c2 * t2.x, a0.y + c1 * t1.y + c2 * t2.y);
    float2 m2 = make_float2(a0.x + c2 * t1.x + c1 * t2.x, a0.y + c2 * t1.y + c1 * t2.y);
    float2 n1 = c_rot<DIR>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
    float2 n2 = c_rot<DIR>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
    v[0] = make_float2(a0.x + t1.x + t2.x, a0.y + t1.y + t2.y);
    v[1] = c_add(m1, n1);
    v[4] = c_sub(m1, n1);
    v[2] = c_add(m2, n2);
    v[3] = c_sub(m2, n2);
}

template <int DIR>
__device__ __forceinline__ void dft7(float2* v) {
    // c[j][k] = cos(2 pi jk/7), s[j][k] = sin(2 pi jk/7) for j,k in 1..3
    const float C1 = 0.6234898018587336f, C2 = -0.22252093395631434f, C3 = -0.900968867902419f;
    const float S1 = 0.7818314824680298f, S2 = 0.9749279121818236f, S3 = 0.43388373911755823f;
    float2 p1 = c_add(v[1], v[6]), q1 = c_sub(v[1], v[6]);
    float2 p2 = c_add(v[2], v[5]), q2 = c_sub(v[2], v[5]);
    float2 p3 = c_add(v[3], v[4]), q3 = c_sub(v[3], v[4]);
    float2 a0 = v[0];
    // k = 1: cos(1j), sin(1j) ; k = 2: cos(2j) ; k = 3: cos(3j)
    float2 m1 = make_float2(a0.x + C1 * p1.x + C2 * p2.x + C3 * p3.x, a0.y + C1 * p1.y + C2 * p2.y + C3 * p3.y);
    float2 m2 = make_float2(a0.x + C2 * p1.x + C3 * p2.x + C1 * p3.x, a0.y + C2 * p1.y + C3 * p2.y + C1 * p3.y);
    float2 m3 = make_float2(a0.x + C3 * p1.x + C1 * p2.x + C2 * p3.x, a0.y + C3 * p1.y + C1 * p2.y + C2 * p3.y);
    // sin(2 pi jk /7): k=1: S1,S2,S3 ; k=2: S2,-S3,-S1 ; k=3: S3,-S1,S2
    float2 n1 = c_rot<DIR>(make_float2(S1 * q1.x + S2 * q2.x + S3 * q3.x, S1 * q1.y + S2 * q2.y + S3 * q3.y));
    float2 n2 = c_rot<DIR>(make_float2(S2 * q1.x - S3 * q2.x - S1 * q3.x, S2 * q1.y - S3 * q2.y - S1 * q3.y));
    float2 n3 = c_rot<DIR>(make_float2(S3 * q1.x - S1 * q2.x + S2 * q3.x, S3 * q1.y - S1 * q2.y + S2 * q3.y));
    v[0] = make_float2(a0.x + p1.x + p2.x + p3.x, a0.y + p1.y + p2.y + p3.y);
    v[1] = c_add(m1, n1);
    v[6] = c_sub(m1, n1);
    v[2] = c_add(m2, n2);
    v[5] = c_sub(m2, n2);
    v[3] = c_add(m3, n3);
    v[4] = c_sub(m3, n3);
}

// One Stockham pass of radix R over `nlines` lines.
// in/out: line l element e at [l*ls + e]; tw: N forward twiddles.
template <int DIR, int R>
__device__ __forceinline__ void stockham_pass(const float2* __restrict__ in, float2* __restrict__ out,
                                              int nlines, int ls, int N, int Ns, const float2* __restrict__ tw,
                                              int tid, int nthr) {
    const int NR = N / R;
    const int tws = N / (Ns * R);
    const int total = nlines * NR;
    for (int t = tid; t < total; t += nthr) {
        const int line = t / NR;
        const int j = t - line * NR;
        const int k = j % Ns;
        const float2* src = in + line * ls;
        float2* dst = out + line * ls;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[j + r * NR];
        if (k != 0) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = tw[r * k * tws];
                if (DIR > 0) w.y = -w.y;
                v[r] = c_mul(v[r], w);
            }
        }
        if (R == 2) dft2<DIR>(v);
        else if (R == 3) dft3<DIR>(v);
        else if (R == 4) dft4<DIR>(v);
        else if (R == 5) dft5<DIR>(v);
        else if (R == 7) dft7<DIR>(v);
        else if (R == 8) dft8<DIR>(v);
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];
    }
}

// Transform `nlines` lines held in buffer a (b is scratch of the same layout).
// Returns the buffer that holds the result.  All threads of the CTA must call
// it; it ends with a __syncthreads().
template <int DIR>
__device__ float2* smem_fft(float2* a, float2* b, int nlines, int ls, const AxisPlan& p,
                            const float2* tw, int tid, int nthr) {
    int Ns = 1;
    const int N = p.n;
    for (int s = 0; s < p.nstages; ++s) {
        const int R = p.radix[s];
        switch (R) {
            case 2: stockham_pass<DIR, 2>(a, b, nlines, ls, N, Ns, tw, tid, nthr); break;
            case 3: stockham_pass<DIR, 3>(a, b, nlines, ls, N, Ns, tw, tid, nthr); break;
            case 4: stockham_pass<DIR, 4>(a, b, nlines, ls, N, Ns, tw, tid, nthr); break;
            case 5: stockham_pass<DIR, 5>(a, b, nlines, ls, N, Ns, tw, tid, nthr); break;
            case 7: stockham_pass<DIR, 7>(a, b, nlines, ls, N, Ns, tw, tid, nthr); break;
            default: stockham_pass<DIR, 8>(a, b, nlines, ls, N, Ns, tw, tid, nthr); break;
        }
        __syncthreads();
        float2* t = a; a = b; b = t;
        Ns *= R;
    }
    return a;
}

__device__ __forceinline__ void load_twiddles(float2* s_tw, const float2* g_tw, int n, int tid, int nthr) {
    for (int i = tid; i < n; i += nthr) s_tw[i] = g_tw[i];
}
