// psb_fft2.cuh — compile-time-sized FFT passes with large register radices.
//
// A length-N transform is split into two or three Stockham passes of radix
// R (e.g. 240 = 16 x 15, 128 = 16 x 8, 100 = 10 x 10).  Each butterfly of
// radix R is a register DFT (itself a compile-time split into the small
// kernels of psb_fft.cuh), so a 240-point line costs one shared-memory round
// trip instead of four.  The first pass may read straight from global memory
// and the last may hand its outputs to a consumer, so data touches shared
// memory once per pass boundary.
#pragma once
#include "psb_fft.cuh"

// twiddles W_R^i = exp(-2 pi i / R) of the register DFTs, R <= 32, at offset
// R*(R-1)/2 (filled by the host from double precision).
#define PSB_TWR_SIZE 528
__constant__ float2 c_twr[PSB_TWR_SIZE];

constexpr int smallest_factor(int n) {
    for (int p = 2; p * p <= n; ++p)
        if (n % p == 0) return p;
    return n;
}

template <int R, int DIR>
struct RDFT {
    static constexpr int P = (R % 4 == 0 && R > 8) ? 4 : smallest_factor(R);
    static constexpr int Q = R / P;
    static __device__ __forceinline__ void run(float2* v) {
        float2 t[R];
#pragma unroll
        for (int n2 = 0; n2 < Q; ++n2) {
            float2 u[P];
#pragma unroll
            for (int n1 = 0; n1 < P; ++n1) u[n1] = v[Q * n1 + n2];
            RDFT<P, DIR>::run(u);
#pragma unroll
            for (int k1 = 0; k1 < P; ++k1) {
                if ((n2 * k1) % R != 0) {
                    float2 w = c_twr[R * (R - 1) / 2 + (n2 * k1) % R];
                    if (DIR > 0) w.y = -w.y;
                    u[k1] = c_mul(u[k1], w);
                }
                t[n2 * P + k1] = u[k1];
            }
        }
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) {
            float2 w[Q];
#pragma unroll
            for (int n2 = 0; n2 < Q; ++n2) w[n2] = t[n2 * P + k1];
            RDFT<Q, DIR>::run(w);
#pragma unroll
            for (int k2 = 0; k2 < Q; ++k2) v[k1 + P * k2] = w[k2];
        }
    }
};
template <int DIR> struct RDFT<1, DIR> { static __device__ __forceinline__ void run(float2*) {} };
template <int DIR> struct RDFT<2, DIR> { static __device__ __forceinline__ void run(float2* v) { dft2<DIR>(v); } };
template <int DIR> struct RDFT<3, DIR> { static __device__ __forceinline__ void run(float2* v) { dft3<DIR>(v); } };
template <int DIR> struct RDFT<4, DIR> { static __device__ __forceinline__ void run(float2* v) { dft4<DIR>(v); } };
template <int DIR> struct RDFT<5, DIR> { static __device__ __forceinline__ void run(float2* v) { dft5<DIR>(v); } };
template <int DIR> struct RDFT<7, DIR> { static __device__ __forceinline__ void run(float2* v) { dft7<DIR>(v); } };
template <int DIR> struct RDFT<8, DIR> { static __device__ __forceinline__ void run(float2* v) { dft8<DIR>(v); } };

// radix plans of the specialised lengths (two passes; product == N)
template <int N> struct Plan2;
template <> struct Plan2<64> { static constexpr int R0 = 8, R1 = 8; };
template <> struct Plan2<100> { static constexpr int R0 = 10, R1 = 10; };
template <> struct Plan2<128> { static constexpr int R0 = 16, R1 = 8; };
template <> struct Plan2<240> { static constexpr int R0 = 16, R1 = 15; };

__host__ __device__ constexpr bool fast_len(int n) {
    return n == 64 || n == 100 || n == 128 || n == 240;
}

// One Stockham pass of radix R over `nl` lines.  Butterfly b maps to
// (line c, index j): LINE_MAJOR -> consecutive threads walk j of one line,
// else consecutive threads walk lines (column-interleaved, C lines per tile).
// ld(c, n) returns element n of line c; st(c, n, v) stores it.
template <int N, int R, int NS, int DIR, int C, bool LINE_MAJOR, class LD, class ST>
__device__ __forceinline__ void tpass(LD&& ld, ST&& st, int nl, const float2* __restrict__ tw, int tid, int nthr) {
    constexpr int NR = N / R;
    constexpr int TWS = N / (NS * R);
    const int total = (LINE_MAJOR ? nl : C) * NR;
    for (int b = tid; b < total; b += nthr) {
        int c, j;
        if (LINE_MAJOR) {
            c = b / NR;
            j = b - c * NR;
        } else {
            j = b / C;
            c = b - j * C;
            if (c >= nl) continue;
        }
        const int k = j % NS;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = ld(c, j + r * NR);
        if (NS > 1 && k != 0) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = tw[r * k * TWS];
                if (DIR > 0) w.y = -w.y;
                v[r] = c_mul(v[r], w);
            }
        }
        RDFT<R, DIR>::run(v);
        const int base = (j / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) st(c, base + r * NS, v[r]);
    }
}
