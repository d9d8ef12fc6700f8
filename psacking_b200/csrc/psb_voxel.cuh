// psb_voxel.cuh — mesh voxelizer: the caller-side input stage of the packer
// (the reference's voxelize_stl, spectral_packing/bindings.cpp:285-302 and
// packing.cpp:309-588, VoxSurf).
//
// The reference rasterizes every triangle along the three axes in 16-bit
// fixed point: for each pixel centre inside the projected triangle (64-bit
// edge functions) the voxel at the barycentric depth has its axis bit
// flipped; a pixel exactly on an edge counts for one of the two triangles
// sharing it (the one whose edge runs from the lower to the higher vertex
// index).  With the inside fill compiled out (constants.h:9) a voxel is
// occupied when any axis bit is set.  Flips commute, so here one warp per
// (triangle, axis) walks the triangle's pixel box with one lane per pixel and
// flips bits with atomicXor; the result is the reference's.
#pragma once
#include <stdint.h>

#include "psb_pdl.cuh"

#define PSB_FP_POW 16
#define PSB_FP_SCALE (1 << PSB_FP_POW)

// packing.cpp:309-335
__device__ __forceinline__ bool vox_in_triangle(long long i, long long j, const int* p0, const int* p1,
                                                const int* p2, int* depth, int* aligned) {
    const long long d0x = i - p0[0], d0y = j - p0[1];
    const long long d1x = i - p1[0], d1y = j - p1[1];
    const long long d2x = i - p2[0], d2y = j - p2[1];
    const long long e10x = (long long)p1[0] - p0[0], e10y = (long long)p1[1] - p0[1];
    const long long e21x = (long long)p2[0] - p1[0], e21y = (long long)p2[1] - p1[1];
    const long long e02x = (long long)p0[0] - p2[0], e02y = (long long)p0[1] - p2[1];
    const long long c0 = d0x * e10y - d0y * e10x;
    const long long c1 = d1x * e21y - d1y * e21x;
    const long long c2 = d2x * e02y - d2y * e02x;
    const bool inside = (c0 <= 0 && c1 <= 0 && c2 <= 0) || (c0 >= 0 && c1 >= 0 && c2 >= 0);
    *aligned = (c0 == 0) ? 0 : ((c1 == 0) ? 1 : ((c2 == 0) ? 2 : -1));
    if (inside) {
        const long long area = c0 + c1 + c2;
        const long long b0 = (c1 << 10) / area;   // truncating division, as in C++
        const long long b1 = (c2 << 10) / area;
        const long long b2 = (1LL << 10) - b0 - b1;
        *depth = (int)((b0 * p0[2] + b1 * p1[2] + b2 * p2[2]) >> 10);
    }
    return inside;
}

// One warp per (triangle, axis).  pts [n][3] fixed-point vertices, tris [m][3]
// merged vertex indices, vox [X][Y][Z] axis bits.  grid: ceil(3*m / 8), block 256
__global__ void k_voxel_raster(const int* __restrict__ pts, const int* __restrict__ tris, int m, int X, int Y, int Z,
                               unsigned int* __restrict__ vox) {
    pdl_enter();
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= 3 * m) return;
    const int t = w / 3, view = w % 3;
    // swizzles (packing.cpp:337-360): forward maps (x,y,z) to (u,v,depth)
    //   view 0 xyz along z; view 1 yzx along x; view 2 zxy along y
    const int tri[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
    int tp[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int* p = pts + 3 * tri[k];
        if (view == 0) { tp[k][0] = p[0]; tp[k][1] = p[1]; tp[k][2] = p[2]; }
        else if (view == 1) { tp[k][0] = p[1]; tp[k][1] = p[2]; tp[k][2] = p[0]; }
        else { tp[k][0] = p[2]; tp[k][1] = p[0]; tp[k][2] = p[1]; }
    }
    const unsigned int along = view == 0 ? 4u : (view == 1 ? 1u : 2u);
    const long long e10x = tp[1][0] - tp[0][0], e10y = tp[1][1] - tp[0][1];
    const long long e21x = tp[2][0] - tp[1][0], e21y = tp[2][1] - tp[1][1];
    const long long e02x = tp[0][0] - tp[2][0], e02y = tp[0][1] - tp[2][1];
    if ((e10x == 0 && e10y == 0) || (e21x == 0 && e21y == 0) || (e02x == 0 && e02y == 0)) return;
    // the reference forms this determinant from 32-bit int products (v2i),
    // which wrap at these fixed-point magnitudes: a nonzero multiple of 2^32
    // counts as degenerate there, so it is evaluated modulo 2^32 here too
    // (a unit cube at a resolution where 0.95 * res is an integer loses every face)
    if ((unsigned int)e02x * (unsigned int)e10y - (unsigned int)e02y * (unsigned int)e10x == 0u) return;
    const int x0 = min(tp[0][0], min(tp[1][0], tp[2][0])) / PSB_FP_SCALE;
    const int x1 = max(tp[0][0], max(tp[1][0], tp[2][0])) / PSB_FP_SCALE;
    const int y0 = min(tp[0][1], min(tp[1][1], tp[2][1])) / PSB_FP_SCALE;
    const int y1 = max(tp[0][1], max(tp[1][1], tp[2][1])) / PSB_FP_SCALE;
    const int nxp = x1 - x0 + 1;
    const long long npix = (long long)nxp * (y1 - y0 + 1);
    for (long long q = lane; q < npix; q += 32) {
        const int i = x0 + (int)(q % nxp), j = y0 + (int)(q / nxp);
        int depth = 0, aligned = -1;
        if (!vox_in_triangle(((long long)i << PSB_FP_POW) + (1 << (PSB_FP_POW - 1)),
                             ((long long)j << PSB_FP_POW) + (1 << (PSB_FP_POW - 1)), tp[0], tp[1], tp[2], &depth,
                             &aligned))
            continue;
        if (aligned != -1 && !(tri[aligned] < tri[(aligned + 1) % 3])) continue;
        const int d = depth >> PSB_FP_POW;
        int v[3];
        // backward swizzle
        if (view == 0) { v[0] = i; v[1] = j; v[2] = d; }
        else if (view == 1) { v[0] = d; v[1] = i; v[2] = j; }
        else { v[0] = j; v[1] = d; v[2] = i; }
        if (v[0] < 0 || v[1] < 0 || v[2] < 0 || v[0] >= X || v[1] >= Y || v[2] >= Z) continue;
        atomicXor(&vox[((size_t)v[0] * Y + v[1]) * Z + v[2]], along);
    }
}
