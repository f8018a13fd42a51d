// 5DCT deformation d(x,t) = a(t) v(x) + b(t) f(x) applied to a volume
// (the reference's host_deform / kernel_forwardDVF / kernel_deformation,
// src/cu_deform.cu:3-47,66-90, and the first-order host_deform2, :49-64,92-113).
//
// The displacement m = alpha*volume + beta*flow is formed in registers
// (kernel_forwardDVF's three scratch volumes and their cudaMalloc/cudaFree per
// call disappear).  The trilinear gather reads either a persistent 3D texture
// (SrcTex: the texture unit's linear filtering, bit-identical to the
// reference, whose filter weights are not plain products of 8-bit fractions)
// or the linear volume in software with FP32 weights (SrcLinear, the EXACT
// model).  The output keeps the reference's in-slice transposed indexing:
// voxel (ix, iy, iz) of the sampling grid is written at iy + ix*ny + iz*nx*ny
// and samples the source at texture coordinates (iy + my, ix + mx, iz + mz)
// + 0.5 (:85-89).
#pragma once

#include "common.cuh"

namespace mcsart {

template <typename FT> struct Fields {
    const FT *ax, *ay, *az, *bx, *by, *bz;
};

// Sample of `src` for output memory index id (any id in [0, nx*ny*nz)).
// The reference indexes the warp's output in-slice transposed
// (cu_deform.cu:82-85): memory position r = x + y*nx of a slice is treated as
// (ix, iy) = (r / ny, r % ny).  For square slices that is (y, x).
__device__ __forceinline__ void warp_coords(int x, int y, int nx, int ny, int &ix, int &iy) {
    if (nx == ny) {
        ix = y;
        iy = x;
    } else {
        const int r = x + y * nx;
        ix = r / ny;
        iy = r - ix * ny;
    }
}

// Sample of voxel id, whose in-slice transposed coordinates are (ix, iy, iz).
template <typename SRC, typename FT>
__device__ __forceinline__ float warp_sample_at(const SRC &src, const Fields<FT> &f, int64_t id,
                                                int ix, int iy, int iz, int nx, int ny, int nz,
                                                float volume, float flow) {
    // kernel_forwardDVF, cu_deform.cu:74-76
    const float mx = ldv(f.ax, id) * volume + ldv(f.bx, id) * flow;
    const float my = ldv(f.ay, id) * volume + ldv(f.by, id) * flow;
    const float mz = ldv(f.az, id) * volume + ldv(f.bz, id) * flow;
    // kernel_deformation, cu_deform.cu:86-89
    const float xi = iy + 1.0f + my;
    const float yi = ix + 1.0f + mx;
    const float zi = iz + 1.0f + mz;
    return src.fetch(xi - 0.5f, yi - 0.5f, zi - 0.5f, nx, ny, nz);
}

template <typename SRC, typename FT>
__device__ __forceinline__ float warp_sample(const SRC &src, const Fields<FT> &f, int64_t id,
                                             int nx, int ny, int nz, float volume, float flow) {
    const int64_t plane = (int64_t)nx * ny;
    const int iz = (int)(id / plane);
    const int r = (int)(id - (int64_t)iz * plane);
    const int ix = r / ny, iy = r - ix * ny;
    return warp_sample_at(src, f, id, ix, iy, iz, nx, ny, nz, volume, flow);
}

template <typename SRC>
static __global__ void __launch_bounds__(256) deform_kernel(float *out, const SRC src,
                                                            Fields<float> f, int nx, int ny,
                                                            int nz, float volume, float flow) {
    const int64_t n = nvox(nx, ny, nz);
    for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < n;
         id += (int64_t)gridDim.x * blockDim.x)
        out[id] = warp_sample(src, f, id, nx, ny, nz, volume, flow);
}

// deform_kernel with fields and output in a storage type FT (the kernel-level
// form of the driver's 16-bit warps).
template <typename SRC, typename FT>
static __global__ void __launch_bounds__(256) deform_typed_kernel(FT *out, const SRC src,
                                                                  Fields<FT> f, int nx, int ny,
                                                                  int nz, float volume,
                                                                  float flow) {
    const int64_t n = nvox(nx, ny, nz);
    for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < n;
         id += (int64_t)gridDim.x * blockDim.x)
        out[id] = cvt<FT>(warp_sample(src, f, id, nx, ny, nz, volume, flow));
}

// Drop-in kernel_forwardDVF.
static __global__ void __launch_bounds__(256) forward_dvf_kernel(float *mx, float *my, float *mz,
                                                                 Fields<float> f, int64_t n,
                                                                 float volume, float flow) {
    for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < n;
         id += (int64_t)gridDim.x * blockDim.x) {
        mx[id] = f.ax[id] * volume + f.bx[id] * flow;
        my[id] = f.ay[id] * volume + f.by[id] * flow;
        mz[id] = f.az[id] * volume + f.bz[id] * flow;
    }
}

// Drop-in host_deform2 (first-order warp).  Neighbour reads that fall past
// the end of the volume (the +nx neighbour of the last rows of the last slice
// under the transposed index) read 0; the reference reads out of bounds there.
static __global__ void __launch_bounds__(256) deform2_kernel(float *out, const float *in,
                                                             Fields<float> f, int nx, int ny,
                                                             int nz, float volume, float flow) {
    const int64_t n = nvox(nx, ny, nz), plane = (int64_t)nx * ny;
    for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < n;
         id += (int64_t)gridDim.x * blockDim.x) {
        const int iz = (int)(id / plane);
        const int64_t r = id - (int64_t)iz * plane;
        const int ix = (int)(r / ny), iy = (int)(r - (int64_t)ix * ny);
        const float mx = f.ax[id] * volume + f.bx[id] * flow;
        const float my = f.ay[id] * volume + f.by[id] * flow;
        const float mz = f.az[id] * volume + f.bz[id] * flow;
        const float c = in[id];
        auto at = [&](int64_t j) { return j < n ? in[j] : 0.0f; };
        float dx, dy, dz;
        if (ix == nx - 1) dx = 0; else dx = at(id + 1) - c;
        if (iy == ny - 1) dy = 0; else dy = at(id + nx) - c;
        if (iz == nz - 1) dz = 0; else dz = at(id + plane) - c;
        out[id] = c + dy * mx + dx * my + dz * mz;  // cu_deform.cu:112
    }
}

// L2 prefetch for the image pass's warp kernels.  Each voxel's six field
// loads are followed by a dependent texture fetch, so at full occupancy the
// kernels wait on load latency (ncu at 256x256x160: 26 long-scoreboard
// stalls per issue, 4.5 TB/s).  Each block therefore prefetches into L2
// (prefetch.global.L2, no registers, no result changes) the rows of the six
// fields, and optionally of one more volume, that the block
// WARP_PREFETCH_AHEAD blocks later in dispatch order (x fastest, then y, then
// z) will read: one row segment of 32 voxels per thread.  600 blocks is about
// half of those resident at once (8 per SM on 148 SMs); measured at
// 256x256x160: warp_fwd 47.4 to 37.3 ms per step, warp_back_add 59.6 to 55.2
// ms with the fields and to 45.4 ms with the fields and the volume it updates
// (1200 blocks ahead: 37.7 and 55.7; 300: 41.6 and 54.4).  The DVF pass's
// field update, which also writes the fields, was slower with it (97.0 to
// 103.9 ms).
constexpr int WARP_PREFETCH_AHEAD = 600;

// The prefetch for a block of a grid of 32 x TH tiles (gridDim.x x gridDim.y
// per slice, gridDim.z slices); t = the thread's index in the block.
template <typename FT>
__device__ __forceinline__ void prefetch_tile_rows(const Fields<FT> &f, const float *extra,
                                                   int TH, int nx, int ny, int nz, int t) {
    const int64_t gx = gridDim.x, gy = gridDim.y;
    const int64_t b = blockIdx.x + gx * (blockIdx.y + gy * blockIdx.z) + WARP_PREFETCH_AHEAD;
    const int arrays = extra ? 7 : 6;
    if (t >= arrays * TH || b >= gx * gy * gridDim.z) return;
    const int bx = (int)(b % gx), by = (int)((b / gx) % gy), bz = (int)(b / (gx * gy));
    const int a = t / TH, y = by * TH + t % TH, x = bx * 32;
    if (y >= ny || x >= nx || bz >= nz) return;
    const int64_t i = x + (int64_t)y * nx + (int64_t)bz * nx * ny;
    const void *p;
    switch (a) {
        case 0: p = f.ax + i; break;
        case 1: p = f.ay + i; break;
        case 2: p = f.az + i; break;
        case 3: p = f.bx + i; break;
        case 4: p = f.by + i; break;
        case 5: p = f.bz + i; break;
        default: p = extra + i;
    }
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Rows of voxels per thread in the image pass's warp kernels: a block covers
// a 32 x (8 * WARP_ROWS) (x, y) tile of one slice.  2 measured best: 4 rows
// leave a 128x128x96 volume's 1536 blocks in 1.3 waves (warp_fwd 11 % slower
// there), 1 row costs 8 % at 256x256x160.
constexpr int WARP_ROWS = 2;

// SART image pass, forward warp of the current volume into the view's phase:
// dst[id] = warp(src)[id] stored in VT, plus the y-fastest copy
// dstT[iy + ix*ny] of the result (x-fastest reading) for the projector.
// Either output may be nullptr when the view's projector reads only the
// other (all its rays driven along y, or all along x).
// blockDim (32, 8); block covers a 32 x (8 * WR) (x, y) tile of slice
// blockIdx.z.
// WR: rows of voxels per thread (the launch shape the driver's tuning may
// choose; the same bits for every value).
template <typename SRC, typename FT, typename VT, int WR = WARP_ROWS>
static __global__ void __launch_bounds__(256) warp_fwd_kernel(VT *dst, VT *dstT, const SRC src,
                                                              Fields<FT> f, int nx, int ny,
                                                              int nz, float volume, float flow) {
    constexpr int TH = 8 * WR;
    __shared__ float tile[TH][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * TH, iz = blockIdx.z;
    const int64_t slice = (int64_t)iz * nx * ny;
    const int xm = x0 + tx;
    prefetch_tile_rows(f, nullptr, TH, nx, ny, nz, ty * 32 + tx);
#pragma unroll
    for (int k = 0; k < WR; k++) {
        const int ly = ty + 8 * k, ym = y0 + ly;
        float v = 0.0f;
        if (xm < nx && ym < ny) {
            const int64_t id = xm + (int64_t)ym * nx + slice;
            int ix, iy;
            warp_coords(xm, ym, nx, ny, ix, iy);
            v = warp_sample_at(src, f, id, ix, iy, iz, nx, ny, nz, volume, flow);
            if (dst) dst[id] = cvt<VT>(v);
        }
        tile[ly][tx] = v;
    }
    if (dstT == nullptr) return;  // uniform over the block
    __syncthreads();
    // transposed store: runs of TH consecutive iy per ix
    const int t = ty * 32 + tx;
#pragma unroll
    for (int k = 0; k < WR; k++) {
        const int e = t + 256 * k, lx = e / TH, ly = e % TH;
        const int xmT = x0 + lx, ymT = y0 + ly;
        if (xmT < nx && ymT < ny) dstT[ymT + (int64_t)xmT * ny + slice] = cvt<VT>(tile[ly][lx]);
    }
}

// SART image pass, backward warp of the normalised correction and update:
// img[id] += lambda * warp(src)[id]  (AUMISART.cu:222-223).  With a surface,
// the updated voxel is also written to the 3D array the next forward warp
// samples through the texture unit.
// blockDim (32, 8), 32 x (8 * WR) tiles of slice blockIdx.z.
template <typename SRC, typename FT, int WR = WARP_ROWS>
static __global__ void __launch_bounds__(256) warp_back_add_kernel(
    float *img, cudaSurfaceObject_t img_surf, const SRC src, Fields<FT> f, int nx, int ny,
    int nz, float volume, float flow, float lambda) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int xm = blockIdx.x * 32 + tx, iz = blockIdx.z;
    const int64_t slice = (int64_t)iz * nx * ny;
    prefetch_tile_rows(f, img, 8 * WR, nx, ny, nz, ty * 32 + tx);  // and the volume's rows
    if (xm >= nx) return;
#pragma unroll
    for (int k = 0; k < WR; k++) {
        const int ym = blockIdx.y * (8 * WR) + ty + 8 * k;
        if (ym >= ny) break;
        const int64_t id = xm + (int64_t)ym * nx + slice;
        int ix, iy;
        warp_coords(xm, ym, nx, ny, ix, iy);
        const float w = warp_sample_at(src, f, id, ix, iy, iz, nx, ny, nz, volume, flow);
        const float v = __fmaf_rn(w, lambda, img[id]);  // cu_add.cu:17
        img[id] = v;
        if (img_surf)
            surf3Dwrite(v, img_surf, xm * (int)sizeof(float), ym, iz, cudaBoundaryModeZero);
    }
}

// Inverse of the warp's displacement, for square slices (nx == ny), where
// the reference's warp (cu_deform.cu:79-90) samples memory position
// q = (X, Y, Z) of its source at q + D(q) with D = (my, mx, mz)(q) (the
// in-slice transposed index swaps the first two components).  The inverse
// N(q) = -D(q + N(q)) is found by fixed-point iteration from N = 0 with exact
// FP32 trilinear samples of m (clamped at the edges, as the texture), and
// returned in the forward layout: ox = N_Y, oy = N_X, oz = N_Z, so that a
// warp with displacement (ox, oy, oz) undoes the warp with (mx, my, mz).
// blockDim (32, 8), 32x8 tiles of slice blockIdx.z.
static __global__ void __launch_bounds__(256) invert_dvf_kernel(
    float *ox, float *oy, float *oz, const float *mx, const float *my, const float *mz, int nx,
    int ny, int nz, int iters) {
    const int X = blockIdx.x * 32 + threadIdx.x, Y = blockIdx.y * 8 + threadIdx.y, Z = blockIdx.z;
    if (X >= nx || Y >= ny) return;
    const SrcLinear<float> sx{my}, sy{mx}, sz{mz};
    float NX = 0.0f, NY = 0.0f, NZ = 0.0f;
    for (int k = 0; k < iters; k++) {
        const float px = (float)X + 0.5f + NX, py = (float)Y + 0.5f + NY, pz = (float)Z + 0.5f + NZ;
        const float dX = sx.fetch(px, py, pz, nx, ny, nz);
        const float dY = sy.fetch(px, py, pz, nx, ny, nz);
        const float dZ = sz.fetch(px, py, pz, nx, ny, nz);
        NX = -dX;
        NY = -dY;
        NZ = -dZ;
    }
    const int64_t id = X + (int64_t)Y * nx + (int64_t)Z * nx * ny;
    ox[id] = NY;
    oy[id] = NX;
    oz[id] = NZ;
}

// warp_back_add_kernel with an explicit displacement (mx, my, mz) instead of
// alpha * volume + beta * flow: img += lambda * src sampled at the warped
// position (square slices).  blockDim (32, 8), 32x32 tiles of slice blockIdx.z.
template <typename SRC>
static __global__ void __launch_bounds__(256) warp_back_add_disp_kernel(
    float *img, cudaSurfaceObject_t img_surf, const SRC src, const float *mx, const float *my,
    const float *mz, int nx, int ny, int nz, float lambda) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int xm = blockIdx.x * 32 + tx, iz = blockIdx.z;
    const int64_t slice = (int64_t)iz * nx * ny;
    if (xm >= nx) return;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int ym = blockIdx.y * 32 + ty + 8 * k;
        if (ym >= ny) break;
        const int64_t id = xm + (int64_t)ym * nx + slice;
        int ix, iy;
        warp_coords(xm, ym, nx, ny, ix, iy);
        const float xi = iy + 1.0f + my[id], yi = ix + 1.0f + mx[id], zi = iz + 1.0f + mz[id];
        const float w = src.fetch(xi - 0.5f, yi - 0.5f, zi - 0.5f, nx, ny, nz);
        const float v = __fmaf_rn(w, lambda, img[id]);  // cu_add.cu:17
        img[id] = v;
        if (img_surf)
            surf3Dwrite(v, img_surf, xm * (int)sizeof(float), ym, iz, cudaBoundaryModeZero);
    }
}

}  // namespace mcsart
