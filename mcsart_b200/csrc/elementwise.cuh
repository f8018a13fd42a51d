// Elementwise and stencil steps of the SART/motion loop: the reference's
// cu_add.cu, cu_initial.cu, cu_division.cu, cu_multiple.cu, cu_update_udvf.cu
// and mex_diff.cu kernels (drop-in forms), plus the fused motion-pass kernels
// the engine's driver uses instead of chains of them.
#pragma once

#include "backprojector.cuh"
#include "common.cuh"
#include "warp.cuh"

namespace mcsart {

#define MC_GRID_STRIDE(n)                                                                      \
    for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < (n);                \
         id += (int64_t)gridDim.x * blockDim.x)

struct Vox {
    int ix, iy, iz;
};
__device__ __forceinline__ Vox vox_of(int64_t id, int nx, int ny) {
    const int64_t plane = (int64_t)nx * ny;
    Vox v;
    v.iz = (int)(id / plane);
    const int64_t r = id - (int64_t)v.iz * plane;
    v.iy = (int)(r / nx);
    v.ix = (int)(r - (int64_t)v.iy * nx);
    return v;
}

// Forward difference along ind, 0 on the last plane (cu_add.cu:37-57).
template <typename T>
__device__ __forceinline__ float fwd_diff(const T *img0, int64_t id, const Vox &v, int nx, int ny,
                                          int nz, int ind) {
    switch (ind) {
        case 1: return (v.ix == nx - 1) ? 0.0f : ldv(img0, id + 1) - ldv(img0, id);
        case 2: return (v.iy == ny - 1) ? 0.0f : ldv(img0, id + nx) - ldv(img0, id);
        case 3: return (v.iz == nz - 1) ? 0.0f : ldv(img0, id + (int64_t)nx * ny) - ldv(img0, id);
        default: return 0.0f;
    }
}

// cu_add.cu:9-18
static __global__ void add_kernel(float *img1, const float *img, int64_t n, float weight) {
    MC_GRID_STRIDE(n) { img1[id] = __fmaf_rn(img[id], weight, img1[id]); }
}

// cu_add.cu:28-59: img1[id] += img[iy + ix*ny + iz*nx*ny] * weight * d_ind img0
static __global__ void add2_kernel(float *img1, const float *img, int nx, int ny, int nz,
                            const float *img0, float weight, int ind) {
    const int64_t n = nvox(nx, ny, nz);
    MC_GRID_STRIDE(n) {
        const Vox v = vox_of(id, nx, ny);
        const float df = fwd_diff(img0, id, v, nx, ny, nz, ind);
        const int64_t t = v.iy + (int64_t)v.ix * ny + (int64_t)v.iz * nx * ny;
        img1[id] = __fmaf_rn(img[t] * weight, df, img1[id]);
    }
}

// cu_initial.cu:10-17
static __global__ void initial_kernel(float *img, int64_t n, float value) {
    MC_GRID_STRIDE(n) { img[id] = value; }
}

// cu_initial.cu:27-49
static __global__ void initial2_kernel(float *img, int nx, int ny, int nz, const float *img0,
                                float volume, float flow) {
    const int64_t n = nvox(nx, ny, nz);
    MC_GRID_STRIDE(n) {
        const Vox v = vox_of(id, nx, ny);
        const float dfx = fwd_diff(img0, id, v, nx, ny, nz, 1);
        const float dfy = fwd_diff(img0, id, v, nx, ny, nz, 2);
        const float dfz = fwd_diff(img0, id, v, nx, ny, nz, 3);
        img[id] = (dfx + dfy + dfz) * (volume + flow);
    }
}

// cu_division.cu:11-25
static __global__ void division_kernel(float *img1, const float *img, int64_t n) {
    MC_GRID_STRIDE(n) {
        float q = img1[id] / img[id];
        if (isnan(q) || isinf(q)) q = 0.0f;
        img1[id] = q;
    }
}

// cu_multiple.cu:11-43
static __global__ void multiple_kernel(float *img1, int nx, int ny, int nz, const float *img0,
                                float weight, int ind) {
    const int64_t n = nvox(nx, ny, nz);
    MC_GRID_STRIDE(n) {
        const Vox v = vox_of(id, nx, ny);
        img1[id] *= weight * fwd_diff(img0, id, v, nx, ny, nz, ind);
    }
}

// cu_update_udvf.cu:11-62.  b pairs alpha_y/beta_y with the x gradient and
// alpha_x/beta_x with the y gradient (:45-50) while the update adds the x
// component to alpha_x (:55), exactly as the reference does.
static __global__ void update_udvf_kernel(float *ax, float *ay, float *az, float *bx, float *by,
                                   float *bz, const float *img, const float *img0,
                                   float volume_diff, float flow_diff, int nx, int ny, int nz) {
    const int64_t n = nvox(nx, ny, nz);
    MC_GRID_STRIDE(n) {
        const Vox v = vox_of(id, nx, ny);
        const float dfI = img0[id] - img[id];
        const float dfx = fwd_diff(img, id, v, nx, ny, nz, 1);
        const float dfy = fwd_diff(img, id, v, nx, ny, nz, 2);
        const float dfz = fwd_diff(img, id, v, nx, ny, nz, 3);
        const float cax = dfx * volume_diff, cay = dfy * volume_diff, caz = dfz * volume_diff;
        const float cbx = dfx * flow_diff, cby = dfy * flow_diff, cbz = dfz * flow_diff;
        const float w = cax * cax + cay * cay + caz * caz + cbx * cbx + cby * cby + cbz * cbz;
        const float a_x = ay[id], a_y = ax[id], a_z = az[id];
        const float b_x = by[id], b_y = bx[id], b_z = bz[id];
        float b = dfI - cax * a_x - cay * a_y - caz * a_z - cbx * b_x - cby * b_y - cbz * b_z;
        if (w == 0) continue;
        b /= w;
        ax[id] += 1.0f / 6 * b * cax;
        ay[id] += 1.0f / 6 * b * cay;
        az[id] += 1.0f / 6 * b * caz;
        bx[id] += 1.0f / 6 * b * cbx;
        by[id] += 1.0f / 6 * b * cby;
        bz[id] += 1.0f / 6 * b * cbz;
    }
}

// mex_diff.cu:75-113: backward difference, 0 on both faces.
static __global__ void diff_kernel(float *img1, const float *img, int nx, int ny, int nz, int ind) {
    const int64_t n = nvox(nx, ny, nz);
    MC_GRID_STRIDE(n) {
        const Vox v = vox_of(id, nx, ny);
        float r;
        switch (ind) {
            case 1: r = (v.ix == nx - 1 || v.ix == 0) ? 0.0f : img[id] - img[id - 1]; break;
            case 2: r = (v.iy == ny - 1 || v.iy == 0) ? 0.0f : img[id] - img[id - nx]; break;
            case 3:
                r = (v.iz == nz - 1 || v.iz == 0) ? 0.0f : img[id] - img[id - (int64_t)nx * ny];
                break;
            default: continue;
        }
        img1[id] = r;
    }
}

// --------------------------------------------------------- fused kernels
// Storage-type copy of an FP32 volume.
template <typename DT> __global__ void cast_kernel(DT *dst, const float *src, int64_t n) {
    MC_GRID_STRIDE(n) { dst[id] = cvt<DT>(src[id]); }
}

// y-fastest copy of an x-fastest volume: dstT[iy + ix*ny] = src[ix + iy*nx].
// blockDim (32, 8), 32x32 tiles of slice blockIdx.z.
template <typename ST, typename DT>
static __global__ void __launch_bounds__(256) transpose_kernel(DT *dstT, const ST *src, int nx, int ny) {
    __shared__ float tile[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    const int64_t slice = (int64_t)blockIdx.z * nx * ny;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int ly = ty + 8 * k;
        const int ix = x0 + tx, iy = y0 + ly;
        tile[ly][tx] = (ix < nx && iy < ny) ? ldv(src, ix + (int64_t)iy * nx + slice) : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int lx = ty + 8 * k;
        const int ix = x0 + lx, iy = y0 + tx;
        if (ix < nx && iy < ny) dstT[iy + (int64_t)ix * ny + slice] = cvt<DT>(tile[tx][lx]);
    }
}

// Loads the 32x32 tile of a field read at the transposed index
// t = iy + ix*ny + iz*nx*ny for the block's (x, y) tile into tile[lx][ly].
template <typename T>
__device__ __forceinline__ void load_tile_T(float (*tile)[33], const T *src, int x0, int y0,
                                            int nx, int ny, int64_t slice) {
    const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int lx = ty + 8 * k, ix = x0 + lx, iy = y0 + tx;
        tile[lx][tx] = (ix < nx && iy < ny) ? ldv(src, iy + (int64_t)ix * ny + slice) : 0.0f;
    }
}

// Motion pass, AUMISART.cu:252-258 and :267 fused: for the current view
//   img0 = sum over the six (field, gradient) pairs of F[t]*w*d img
//   ones = (dx + dy + dz img) * (-vd + -fd)
// each written x-fastest (img0, ones) and as a y-fastest copy (img0T,
// onesT) for the projector; either pair may be nullptr when the view's
// projector reads only the other.  PAIR: img0 and ones interleaved in img0
// (img0[2i], img0[2i + 1]) and img0T, for the projector's paired load; ones
// and onesT unused.
template <typename FT, typename VT, bool PAIR = false>
static __global__ void __launch_bounds__(256) motion_prep_kernel(VT *img0, VT *img0T, VT *ones,
                                                          VT *onesT, const float *img,
                                                          Fields<FT> f, int nx, int ny, int nz,
                                                          float vd, float fd) {
    __shared__ float ft[6][32][33];
    __shared__ float o0[32][33], o1[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32, iz = blockIdx.z;
    const int64_t slice = (int64_t)iz * nx * ny;
    load_tile_T(ft[0], f.ay, x0, y0, nx, ny, slice);
    load_tile_T(ft[1], f.ax, x0, y0, nx, ny, slice);
    load_tile_T(ft[2], f.az, x0, y0, nx, ny, slice);
    load_tile_T(ft[3], f.by, x0, y0, nx, ny, slice);
    load_tile_T(ft[4], f.bx, x0, y0, nx, ny, slice);
    load_tile_T(ft[5], f.bz, x0, y0, nx, ny, slice);
    __syncthreads();
    const int ix = x0 + tx;
    const float s_ones = (-vd) + (-fd);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int ly = ty + 8 * k, iy = y0 + ly;
        float a = 0.0f, b = 0.0f;
        if (ix < nx && iy < ny) {
            const int64_t id = ix + (int64_t)iy * nx + slice;
            const Vox v{ix, iy, iz};
            const float dfx = fwd_diff(img, id, v, nx, ny, nz, 1);
            const float dfy = fwd_diff(img, id, v, nx, ny, nz, 2);
            const float dfz = fwd_diff(img, id, v, nx, ny, nz, 3);
            // host_initial(img0, 0) then six host_add2 in the reference's order
            a = __fmaf_rn(ft[0][tx][ly] * vd, dfx, a);
            a = __fmaf_rn(ft[1][tx][ly] * vd, dfy, a);
            a = __fmaf_rn(ft[2][tx][ly] * vd, dfz, a);
            a = __fmaf_rn(ft[3][tx][ly] * fd, dfx, a);
            a = __fmaf_rn(ft[4][tx][ly] * fd, dfy, a);
            a = __fmaf_rn(ft[5][tx][ly] * fd, dfz, a);
            b = (dfx + dfy + dfz) * s_ones;  // cu_initial.cu:48
            if (img0) {
                if (PAIR) {
                    stv2(img0, id, a, b);
                } else {
                    img0[id] = cvt<VT>(a);
                    ones[id] = cvt<VT>(b);
                }
            }
        }
        o0[ly][tx] = a;
        o1[ly][tx] = b;
    }
    if (img0T == nullptr) return;  // uniform over the block
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int lx = ty + 8 * k, ixT = x0 + lx, iyT = y0 + tx;
        if (ixT < nx && iyT < ny) {
            const int64_t t = iyT + (int64_t)ixT * ny + slice;
            if (PAIR) {
                stv2(img0T, t, o0[tx][lx], o1[tx][lx]);
            } else {
                img0T[t] = cvt<VT>(o0[tx][lx]);
                onesT[t] = cvt<VT>(o1[tx][lx]);
            }
        }
    }
}

// Motion pass field update, AUMISART.cu:272-277 fused: with q = img_temp read
// at the transposed index, alpha_y += q*nvd*dx img, alpha_x += q*nvd*dy img,
// alpha_z += q*nvd*dz img, and the same for beta with nfd.
template <typename FT>
static __global__ void __launch_bounds__(256) field_update_kernel(FT *ax, FT *ay, FT *az, FT *bx, FT *by,
                                                           FT *bz, const float *img_temp,
                                                           const float *img, int nx, int ny,
                                                           int nz, float nvd, float nfd) {
    __shared__ float qt[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32, iz = blockIdx.z;
    const int64_t slice = (int64_t)iz * nx * ny;
    load_tile_T(qt, img_temp, x0, y0, nx, ny, slice);
    __syncthreads();
    const int ix = x0 + tx;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int ly = ty + 8 * k, iy = y0 + ly;
        if (ix < nx && iy < ny) {
            const int64_t id = ix + (int64_t)iy * nx + slice;
            const Vox v{ix, iy, iz};
            const float dfx = fwd_diff(img, id, v, nx, ny, nz, 1);
            const float dfy = fwd_diff(img, id, v, nx, ny, nz, 2);
            const float dfz = fwd_diff(img, id, v, nx, ny, nz, 3);
            const float q = qt[tx][ly];
            ay[id] = cvt<FT>(__fmaf_rn(q * nvd, dfx, ldv(ay, id)));
            ax[id] = cvt<FT>(__fmaf_rn(q * nvd, dfy, ldv(ax, id)));
            az[id] = cvt<FT>(__fmaf_rn(q * nvd, dfz, ldv(az, id)));
            by[id] = cvt<FT>(__fmaf_rn(q * nfd, dfx, ldv(by, id)));
            bx[id] = cvt<FT>(__fmaf_rn(q * nfd, dfy, ldv(bx, id)));
            bz[id] = cvt<FT>(__fmaf_rn(q * nfd, dfz, ldv(bz, id)));
        }
    }
}

// field_update_kernel for view v followed by motion_prep_kernel for the next
// view, in one pass over the fields (square slices, nx == ny).  The block of
// output tile A = (x0, y0) updates the fields on the transposed memory tile
// A^T, which is exactly the set motion_prep reads for A, keeps the updated
// values in shared memory and then computes img0 / ones of tile A for the
// next view.  Every field voxel is updated by exactly one block, and the
// arithmetic is that of the two kernels, so the results are bitwise theirs.
// EARLY (a launch shape the driver's tuning may choose): every thread loads
// its 4 x 6 field values first, before the ratio tile and its barrier, so
// that 24 loads per thread are in flight at once (more registers, fewer
// resident blocks); otherwise the fields are loaded voxel by voxel.
// PAIR: img0 and ones interleaved, as in motion_prep_kernel.
// BP: the view's backprojection ratio of tile A (the DVF pass's
// host_backprojection and host_division, src/AUMISART.cu:95-100 / :265-270) is
// computed here from `bp` (its (residual, initial2-projection) pairs and
// column data, one slice) with the backprojector's own per-voxel code,
// instead of being read from img_temp: the field update of a tile needs the
// ratio of that tile only, so the ratio never goes to memory, and blocks
// gathering from the detector (bound by instruction issue) share the SMs
// with blocks streaming the fields (bound by memory latency).  PROVEN: as in
// bp_kernel.  The ratio's bits are the backprojector kernel's.
template <typename FT, typename VT, bool EARLY = false, bool PAIR = false, bool BP = false,
          bool PROVEN = false>
static __global__ void __launch_bounds__(256) field_update_prep_kernel(
    FT *ax, FT *ay, FT *az, FT *bx, FT *by, FT *bz, const float *img_temp, const float *img,
    int nx, int ny, int nz, float nvd, float nfd, VT *img0, VT *img0T, VT *ones, VT *onesT,
    float vd, float fd, const BPArgs bp) {
    __shared__ float ft[6][32][33];
    __shared__ float rt[32][33];
    __shared__ float o0[32][33], o1[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32, iz = blockIdx.z;
    const int64_t slice = (int64_t)iz * nx * ny;
    if (BP) {
        // The block's own field rows (tile A^T) and volume rows (A^T and A)
        // are prefetched into L2 before the backprojection gather, which
        // then covers their memory latency: one 32-voxel row per thread
        // (6 x 32 field rows, 2 x 32 volume rows).  Measured at 256x256x160:
        // 151.4 to 141.9 ms per step (fields alone 145.3).
        const int t = ty * 32 + tx, r = t % 32, w = t / 32;
        const void *p = nullptr;
        if (w < 7) {  // rows of A^T: memory rows x0 + r, columns from y0
            if (x0 + r < ny && y0 < nx) {
                const int64_t i = y0 + (int64_t)(x0 + r) * nx + slice;
                switch (w) {
                    case 0: p = ax + i; break;
                    case 1: p = ay + i; break;
                    case 2: p = az + i; break;
                    case 3: p = bx + i; break;
                    case 4: p = by + i; break;
                    case 5: p = bz + i; break;
                    default: p = img + i;
                }
            }
        } else if (y0 + r < ny && x0 < nx) {  // volume rows of A
            p = img + x0 + (int64_t)(y0 + r) * nx + slice;
        }
        if (p) asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
    // the field values at this thread's 4 voxels of A^T (EARLY)
    float fe[EARLY ? 4 : 1][6];
    if (EARLY) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int lx = ty + 8 * k, xp = y0 + tx, yp = x0 + lx;
            const bool in = xp < nx && yp < ny;
            const int64_t id = in ? xp + (int64_t)yp * nx + slice : 0;
            fe[k][0] = in ? ldv(ay, id) : 0.0f;
            fe[k][1] = in ? ldv(ax, id) : 0.0f;
            fe[k][2] = in ? ldv(az, id) : 0.0f;
            fe[k][3] = in ? ldv(by, id) : 0.0f;
            fe[k][4] = in ? ldv(bx, id) : 0.0f;
            fe[k][5] = in ? ldv(bz, id) : 0.0f;
        }
    }
    // ratio on tile A, x-fastest: rt[y - y0][x - x0]
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int ly = ty + 8 * k, xx = x0 + tx, yy = y0 + ly;
        float q = 0.0f;
        if (xx < nx && yy < ny) {
            if (BP) {
                float a0 = 0.0f, a1 = 0.0f;
                bp_gather_view<2, PROVEN, 1>(bp, bp.angle, nullptr, bp.pair, xx, yy, iz, &a0,
                                             &a1);
                q = a0 / a1;                           // cu_division.cu:20
                if (isnan(q) || isinf(q)) q = 0.0f;    // :21-24
            } else {
                q = img_temp[xx + (int64_t)yy * nx + slice];
            }
        }
        rt[ly][tx] = q;
    }
    __syncthreads();
    // field update on A^T: voxel (x', y') = (y0 + tx, x0 + lx); its q is the
    // ratio at the transposed index, i.e. at (x0 + lx, y0 + tx) of tile A
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int lx = ty + 8 * k, xp = y0 + tx, yp = x0 + lx;
        float n[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (xp < nx && yp < ny) {
            const int64_t id = xp + (int64_t)yp * nx + slice;
            const Vox v{xp, yp, iz};
            const float dfx = fwd_diff(img, id, v, nx, ny, nz, 1);
            const float dfy = fwd_diff(img, id, v, nx, ny, nz, 2);
            const float dfz = fwd_diff(img, id, v, nx, ny, nz, 3);
            const float q = rt[tx][lx];
            const float fay = EARLY ? fe[k % (EARLY ? 4 : 1)][0] : ldv(ay, id);
            const float fax = EARLY ? fe[k % (EARLY ? 4 : 1)][1] : ldv(ax, id);
            const float faz = EARLY ? fe[k % (EARLY ? 4 : 1)][2] : ldv(az, id);
            const float fby = EARLY ? fe[k % (EARLY ? 4 : 1)][3] : ldv(by, id);
            const float fbx = EARLY ? fe[k % (EARLY ? 4 : 1)][4] : ldv(bx, id);
            const float fbz = EARLY ? fe[k % (EARLY ? 4 : 1)][5] : ldv(bz, id);
            const FT nay = cvt<FT>(__fmaf_rn(q * nvd, dfx, fay));
            const FT nax = cvt<FT>(__fmaf_rn(q * nvd, dfy, fax));
            const FT naz = cvt<FT>(__fmaf_rn(q * nvd, dfz, faz));
            const FT nby = cvt<FT>(__fmaf_rn(q * nfd, dfx, fby));
            const FT nbx = cvt<FT>(__fmaf_rn(q * nfd, dfy, fbx));
            const FT nbz = cvt<FT>(__fmaf_rn(q * nfd, dfz, fbz));
            ay[id] = nay; ax[id] = nax; az[id] = naz;
            by[id] = nby; bx[id] = nbx; bz[id] = nbz;
            n[0] = tof(nay); n[1] = tof(nax); n[2] = tof(naz);
            n[3] = tof(nby); n[4] = tof(nbx); n[5] = tof(nbz);
        }
#pragma unroll
        for (int c = 0; c < 6; c++) ft[c][lx][tx] = n[c];
    }
    __syncthreads();
    // motion_prep_kernel for tile A with the next view's weights
    const int ix = x0 + tx;
    const float s_ones = (-vd) + (-fd);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int ly = ty + 8 * k, iy = y0 + ly;
        float a = 0.0f, b = 0.0f;
        if (ix < nx && iy < ny) {
            const int64_t id = ix + (int64_t)iy * nx + slice;
            const Vox v{ix, iy, iz};
            const float dfx = fwd_diff(img, id, v, nx, ny, nz, 1);
            const float dfy = fwd_diff(img, id, v, nx, ny, nz, 2);
            const float dfz = fwd_diff(img, id, v, nx, ny, nz, 3);
            a = __fmaf_rn(ft[0][tx][ly] * vd, dfx, a);
            a = __fmaf_rn(ft[1][tx][ly] * vd, dfy, a);
            a = __fmaf_rn(ft[2][tx][ly] * vd, dfz, a);
            a = __fmaf_rn(ft[3][tx][ly] * fd, dfx, a);
            a = __fmaf_rn(ft[4][tx][ly] * fd, dfy, a);
            a = __fmaf_rn(ft[5][tx][ly] * fd, dfz, a);
            b = (dfx + dfy + dfz) * s_ones;  // cu_initial.cu:48
            if (img0) {
                if (PAIR) {
                    stv2(img0, id, a, b);
                } else {
                    img0[id] = cvt<VT>(a);
                    ones[id] = cvt<VT>(b);
                }
            }
        }
        o0[ly][tx] = a;
        o1[ly][tx] = b;
    }
    if (img0T == nullptr) return;  // uniform over the block
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int lx = ty + 8 * k, ixT = x0 + lx, iyT = y0 + tx;
        if (ixT < nx && iyT < ny) {
            const int64_t t = iyT + (int64_t)ixT * ny + slice;
            if (PAIR) {
                stv2(img0T, t, o0[tx][lx], o1[tx][lx]);
            } else {
                img0T[t] = cvt<VT>(o0[tx][lx]);
                onesT[t] = cvt<VT>(o1[tx][lx]);
            }
        }
    }
}

// Norm ratios ||r_v|| / ||b_v|| from per-block partials (fixed order); one
// warp per view.  Replaces the two cublasSnrm2 calls per view.
static __global__ void norm_finalize_kernel(float *norm_out, const double2 *part, int n_blocks,
                                     const int *views, int n) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n) return;
    const double2 *p = part + (int64_t)w * n_blocks;
    double sb = 0.0, sr = 0.0;
    for (int i = lane; i < n_blocks; i += 32) {
        sb += p[i].x;
        sr += p[i].y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        sb += __shfl_down_sync(0xffffffffu, sb, off);
        sr += __shfl_down_sync(0xffffffffu, sr, off);
    }
    if (lane == 0) norm_out[views[w]] = (float)(sqrt(sr) / sqrt(sb));
}

}  // namespace mcsart
