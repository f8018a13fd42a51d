// Gather-form backprojector (the reference's kernel_backprojection,
// src/cu_backprojection.cu:49-170), restructured for B200.
//
// Reference semantics kept exactly: voxel centre with integer nx/2 (:66-68);
// six boundary points, i.e. an axis-aligned unit square in the rotated frame
// plus the voxel's top and bottom (:82-97); magnification SD/(x+SO) (:105-122);
// bounding box in detector index units a/da - ai + 0.5 (:135-138); unnormalised
// overlap weights wa*wb (:150-168); __sinf/__cosf of the angle (:62-63).
// The projection is read straight from global memory: the reference's texture
// fetch happens at texel centres (:167) and so returns the texel itself, with
// denormal texels read as signed zeros (tex_texel; the projector applies it
// to the pairs it writes for this kernel), which removes the per-call
// cudaMalloc3DArray + copy (:10-37).
//
// Restructured for the hardware: one thread per column of BP_NZ voxels (no
// atomics, so runs are bitwise reproducible), 32-wide rows of voxels per warp
// for coalesced stores and a shared-memory transpose when the y-fastest copy
// of the volume must be kept current; two projections (SART residual and ones-projection, packed as
// float2) are gathered with one set of weights and the SART division
// (src/cu_division.cu:20-24) and update (src/cu_add.cu:17) run in the epilogue.
#pragma once

#include "common.cuh"

namespace mcsart {

enum BPMode { BP_PLAIN = 0, BP_DIV = 1, BP_DIV_ADD = 2 };

// In-plane part of the footprint of voxel column (ix, iy): the same for every
// z (src/cu_backprojection.cu:66-67,80-122,135-136).
struct BPColumn {
    float amin, amax;  // detector column box, index units
    float rl, rr, r0;  // magnifications SD/(x+SO) at the three distances
};

// PROVEN: bp_geom_proven(g) holds, so every division below has its operands
// in mk_div's checked range and takes the branch-free form without tests.
template <bool PROVEN>
__device__ __forceinline__ BPColumn bp_column(int ix, int iy, float cphi, float sphi,
                                              const Geom &g) {
    const float xc = (float)ix - g.nx / 2 + 0.5f;
    const float yc = (float)iy - g.ny / 2 + 0.5f;
    // rotated voxel centre; the boundary points differ by +-0.5 from it.  The
    // products are fused explicitly in the order that reproduces the
    // reference kernel bit for bit (":80-95" as compiled), so that the result
    // does not depend on how the compiler contracts after unrolling.
    const float t = __fmaf_rn(yc, sphi, __fmul_rn(xc, cphi));
    const float u = __fmaf_rn(yc, cphi, __fmul_rn(-xc, sphi));
    const float tl = t - 0.5f, tr = t + 0.5f, ul = u - 0.5f, ur = u + 0.5f;
    BPColumn c;
    if (PROVEN) {
        const float dl = tl + g.SO, dr = tr + g.SO, d0 = t + g.SO;
        c.rl = mk_div(g.SD, dl, mk_recip(dl));
        c.rr = mk_div(g.SD, dr, mk_recip(dr));
        c.r0 = mk_div(g.SD, d0, mk_recip(d0));
    } else {
        c.rl = g.SD / (tl + g.SO);  // points ll and lr
        c.rr = g.SD / (tr + g.SO);  // points rr and rl
        c.r0 = g.SD / (t + g.SO);   // top and bottom
    }
    const float all = c.rl * ul, alr = c.rl * ur, arr = c.rr * ur, arl = c.rr * ul, at = c.r0 * u;
    const float amax = fmaxf(fmaxf(fmaxf(all, arr), fmaxf(alr, arl)), at);
    const float amin = fminf(fminf(fminf(all, arr), fminf(alr, arl)), at);
    const float ya = mk_recip(g.da);
    float qmax = mk_div(amax, g.da, ya), qmin = mk_div(amin, g.da, ya);
    if (!PROVEN && !(mk_den_ok(g.da) && mk_num_ok(amax) && mk_num_ok(amin))) {
        qmax = amax / g.da;
        qmin = amin / g.da;
    }
    c.amax = qmax - g.ai + 0.5f;
    c.amin = qmin - g.ai + 0.5f;
    return c;
}

// Axial part for slice iz (:68,96-97,115-122,137-138): detector row box.
template <bool PROVEN>
__device__ __forceinline__ void bp_rows(const BPColumn &c, int iz, const Geom &g, float &bmin,
                                        float &bmax) {
    const float zc = (float)iz - g.nz / 2 + 0.5f;
    const float bl = c.rl * zc, br = c.rr * zc, bt = c.r0 * (zc + 0.5f), bb = c.r0 * (zc - 0.5f);
    const float hi = fmaxf(fmaxf(fmaxf(bl, br), fmaxf(bl, br)), fmaxf(bt, bb));
    const float lo = fminf(fminf(fminf(bl, br), fminf(bl, br)), fminf(bt, bb));
    const float y = mk_recip(g.db);
    float qhi = mk_div(hi, g.db, y), qlo = mk_div(lo, g.db, y);
    if (!PROVEN && !(mk_den_ok(g.db) && mk_num_ok(hi) && mk_num_ok(lo))) {
        qhi = hi / g.db;
        qlo = lo / g.db;
    }
    bmax = qhi - g.bi + 0.5f;
    bmin = qlo - g.bi + 0.5f;
}

// Whether the geometry alone puts every division of bp_column / bp_rows in
// mk_div's checked range (divisor in [2^-20, 2^20), numerator +0 or in
// [2^-80, 2^80]), for every voxel and angle:
//  * |t| <= nx/2 + ny/2 + 2 for a voxel centre (|sin|, |cos| <= 1), so the
//    magnification divisors t -+ 0.5 + SO lie in [SO - R, SO + R] and the
//    magnifications r = SD / divisor in [rmin, rmax];
//  * the column box ends are corner products r * (u -+ 0.5) (the centre
//    product r0 * u lies between them): u -+ 0.5 is +0 or at least 2^-25 in
//    magnitude (an exact difference of floats near 0.5 when it is small);
//  * the row box ends are r times a half-integer, or r0 times an integer,
//    which is +0 or at least 1 in magnitude.
// None of these is -0.  Bounds carry a margin of 2^-10 for rounding and for
// the intrinsic sine and cosine.
inline bool bp_geom_proven(const Geom &g) {
    const double R = ((double)(g.nx / 2) + (double)(g.ny / 2) + 3.0) * (1.0 + 0x1p-10);
    const double dlo = (double)g.SO - R, dhi = (double)g.SO + R;
    if (!(dlo >= 0x1p-19 && dhi < 0x1p19)) return false;
    const double rmin = (double)g.SD / dhi * (1.0 - 0x1p-10);
    const double rmax = (double)g.SD / dlo * (1.0 + 0x1p-10);
    const double extent = R + (double)(g.nz / 2) + 4.0;
    return g.SD >= 0x1p-79 && g.SD <= 0x1p79 && g.da >= 0x1p-19 && g.da < 0x1p19 &&
           g.db >= 0x1p-19 && g.db < 0x1p19 && rmin * 0x1p-26 >= 0x1p-79 &&
           rmax * extent <= 0x1p79;
}

struct BPArgs {
    const float *proj;    // K == 1
    const float2 *pair;   // K == 2: (residual, ones-projection)
    Geom g;
    float angle;
    float lambda;
    float *out;           // BP_PLAIN / BP_DIV: output (nullable in BP_DIV); BP_DIV_ADD:
                          // volume updated in place
    float *outT;          // BP_DIV_ADD: y-fastest copy refreshed alongside (nullable)
    cudaSurfaceObject_t outSurf;  // BP_DIV: 3D array receiving the ratio (0 = none)
    // Several views per launch (K == 2): n_views views of an ordered subset,
    // angles[v] (device) and pair + v*na*nb.  BP_DIV writes view v's ratio to
    // out + v*V and outSurfs[v]; BP_DIV_ADD adds lambda times the sum of the
    // views' ratios (summed in view order) to out.  n_views <= 1 with
    // angles == nullptr is the single view at `angle`.
    int n_views;
    const float *angles;
    cudaSurfaceObject_t outSurfs[16];
    // the views' column data (bp_column for every (ix, iy), index
    // ix + iy*nx, view v of the launch at + v*nx*ny), computed by the
    // projector launch before this one; nullptr = compute it here
    const float4 *colA;  // amin, amax, rl, rr
    const float *colB;   // r0
};
constexpr int BP_MAX_VIEWS = 16;

// Voxel columns per block: 32 (x) by BP_ROWS (y), BP_NZ slices per thread.
#ifndef MCSART_BP_NZ
#define MCSART_BP_NZ 2
#endif
// 4 rows: 128-thread blocks fill the SMs' slots in fewer partial waves than
// 256-thread ones (9 resident per SM at 56 registers); 2.5 % less
// backprojector time than 32 x 8 at both benchmark sizes.
constexpr int BP_ROWS = 4;
constexpr int BP_NZ = MCSART_BP_NZ;
// Row weights kept in registers per slice; footprints taller than this many
// detector rows take the general loop (3 measured 12 % slower at 256x256x160:
// about a fifth of the voxels need 4 rows there).
constexpr int BP_WB = 4;
// Resident 256-thread blocks per SM the register budget must allow (the
// launch-bounds minimum): for the single-view kernel with FP32 geometry and
// up to 2 voxels per thread 5, i.e. at most 48 registers, which it fits
// without spilling (10 resident 128-thread blocks instead of 9 at 55
// registers): backprojector time -1 % at 256x256x160; 6 (40 registers)
// spills and was 3 % slower.  The several-view form (75 registers) was 5 %
// slower per view under the same bound and keeps its own allocation.
template <bool GEO64, bool MULTI, int NZ> constexpr int bp_min_blocks() {
    return (!GEO64 && !MULTI && NZ <= 2) ? 5 : 1;
}

// Overlap-weighted gather of one view for the NZ voxels (ix, iy, z0 ..)
// of a thread: acc0 (and acc1 with K == 2) get the view's terms in the
// reference's order (detector column outer, row inner, acc = fma(wa*wb, p,
// acc), :150-168).  The column box and the column weights wa are shared by the
// voxels of a thread, the row weights wb are computed once per voxel.
template <int K, bool PROVEN, int NZ = BP_NZ>
__device__ __forceinline__ void bp_gather_view(const BPArgs &p, float angle, const float *proj,
                                               const float2 *pair, int ix, int iy, int z0,
                                               float *acc0, float *acc1, int view = 0) {
    const Geom &g = p.g;
    const int na = g.na;
    BPColumn col;
    if (p.colA != nullptr) {
        const int64_t c = ix + ((int64_t)iy + (int64_t)view * g.ny) * g.nx;
        const float4 a = __ldg(p.colA + c);
        col.amin = a.x;
        col.amax = a.y;
        col.rl = a.z;
        col.rr = a.w;
        col.r0 = __ldg(p.colB + c);
    } else {
        const float sphi = __sinf(angle), cphi = __cosf(angle);
        col = bp_column<PROVEN>(ix, iy, cphi, sphi, g);
    }
    // rows of each slice: first row, count (BP_WB + 1 = more than BP_WB),
    // row weights, box
    int ib0[NZ], nbk[NZ];
    float wb[NZ][BP_WB], bmn[NZ], bmx[NZ];
#pragma unroll
    for (int k = 0; k < NZ; k++) {
        nbk[k] = 0;
        ib0[k] = 0;
        bmn[k] = 0.0f;
        bmx[k] = 0.0f;
#pragma unroll
        for (int j = 0; j < BP_WB; j++) wb[k][j] = 0.0f;
        const int iz = z0 + k;
        if (iz < g.nz) {
            bp_rows<PROVEN>(col, iz, g, bmn[k], bmx[k]);
            const float blim = ((float)g.nb < bmx[k]) ? (float)g.nb : bmx[k];  // MIN(nb, b_max)
            ib0[k] = max(0, (int)floorf(fmaxf(bmn[k], -1.0f)));
            // rows ib >= ib0 with (float)ib < blim, i.e. ib < ceil(blim)
            // (blim <= nb, so every row index is exact in float; a NaN
            // converts to 0 and gives no rows, as the loop test would)
            nbk[k] = min(BP_WB + 1, max(0, (int)ceilf(blim) - ib0[k]));
#pragma unroll
            for (int j = 0; j < BP_WB; j++) {
                const int ib = ib0[k] + j;
                wb[k][j] = fminf(ib + 1.0f, bmx[k]) - fmaxf(ib + 0.0f, bmn[k]);
            }
        }
    }
    const float alim = ((float)na < col.amax) ? (float)na : col.amax;  // MIN(na, a_max)
    const int ia0 = max(0, (int)floorf(fmaxf(col.amin, -1.0f)));
    for (int ia = ia0; (float)ia < alim; ia++) {
        const float wa = fminf(ia + 1.0f, col.amax) - fmaxf(ia + 0.0f, col.amin);
#pragma unroll
        for (int k = 0; k < NZ; k++) {
            if (nbk[k] <= BP_WB) {
#pragma unroll
                for (int j = 0; j < BP_WB; j++) {
                    if (j < nbk[k]) {
                        const float w = __fmul_rn(wa, wb[k][j]);
                        const int pix = ia + (ib0[k] + j) * na;
                        if (K == 1) {
                            acc0[k] = __fmaf_rn(w, tex_texel(__ldg(proj + pix)), acc0[k]);
                        } else {
                            const float2 v = __ldg(pair + pix);
                            acc0[k] = __fmaf_rn(w, v.x, acc0[k]);
                            acc1[k] = __fmaf_rn(w, v.y, acc1[k]);
                        }
                    }
                }
            } else {
                const float blim = ((float)g.nb < bmx[k]) ? (float)g.nb : bmx[k];
                for (int ib = ib0[k]; (float)ib < blim; ib++) {
                    const float w =
                        __fmul_rn(wa, fminf(ib + 1.0f, bmx[k]) - fmaxf(ib + 0.0f, bmn[k]));
                    const int pix = ia + ib * na;
                    if (K == 1) {
                        acc0[k] = __fmaf_rn(w, tex_texel(__ldg(proj + pix)), acc0[k]);
                    } else {
                        const float2 v = __ldg(pair + pix);
                        acc0[k] = __fmaf_rn(w, v.x, acc0[k]);
                        acc1[k] = __fmaf_rn(w, v.y, acc1[k]);
                    }
                }
            }
        }
    }
}

// FP64 geometry (options.geom64): the footprint of bp_column / bp_rows
// (src/cu_backprojection.cu:66-168) with every coordinate, box edge and
// overlap weight in FP64 and the rotation by the FP64 sine and cosine of the
// angle; the projection's terms (K == 1) or the residual's (K == 2) are
// accumulated in FP32 (acc0), the normaliser's (the projection of a
// ones-volume, the SART column sum; K == 2) in FP64 (acc1).  Same order of
// terms as bp_gather_view.
template <int K, int NZ = BP_NZ>
__device__ __forceinline__ void bp_gather_view64(const BPArgs &p, float angle, const float *proj,
                                                 const float2 *pair, int ix, int iy, int z0,
                                                 float *acc0, double *acc1) {
    const Geom &g = p.g;
    const double SO = g.SO, SD = g.SD, da = g.da, db = g.db;
    double sphi, cphi;
    sincos((double)angle, &sphi, &cphi);
    const double xc = (double)ix - g.nx / 2 + 0.5, yc = (double)iy - g.ny / 2 + 0.5;
    const double t = xc * cphi + yc * sphi, u = -xc * sphi + yc * cphi;
    const double rl = SD / (t - 0.5 + SO), rr = SD / (t + 0.5 + SO), r0 = SD / (t + SO);
    const double all = rl * (u - 0.5), alr = rl * (u + 0.5);
    const double arr = rr * (u + 0.5), arl = rr * (u - 0.5), at = r0 * u;
    const double amax = fmax(fmax(fmax(all, arr), fmax(alr, arl)), at) / da - g.ai + 0.5;
    const double amin = fmin(fmin(fmin(all, arr), fmin(alr, arl)), at) / da - g.ai + 0.5;
    const int ia0 = max(0, (int)floor(fmax(amin, -1.0)));
    const int ia1 = (int)ceil(fmin(amax, (double)g.na));  // columns ia < ia1
#pragma unroll
    for (int k = 0; k < NZ; k++) {
        const int iz = z0 + k;
        if (iz >= g.nz) continue;
        const double zc = (double)iz - g.nz / 2 + 0.5;
        const double bl = rl * zc, br = rr * zc, bt = r0 * (zc + 0.5), bb = r0 * (zc - 0.5);
        const double bmax = fmax(fmax(bl, br), fmax(bt, bb)) / db - g.bi + 0.5;
        const double bmin = fmin(fmin(bl, br), fmin(bt, bb)) / db - g.bi + 0.5;
        const int ib0 = max(0, (int)floor(fmax(bmin, -1.0)));
        const int ib1 = (int)ceil(fmin(bmax, (double)g.nb));
        for (int ia = ia0; ia < ia1; ia++) {
            const double wa = fmin(ia + 1.0, amax) - fmax((double)ia, amin);
            for (int ib = ib0; ib < ib1; ib++) {
                const double w = wa * (fmin(ib + 1.0, bmax) - fmax((double)ib, bmin));
                if (K == 1) {
                    acc0[k] = __fmaf_rn((float)w, __ldg(proj + ia + (int64_t)ib * g.na), acc0[k]);
                } else {
                    const float2 v = __ldg(pair + ia + (int64_t)ib * g.na);
                    acc0[k] = __fmaf_rn((float)w, v.x, acc0[k]);
                    acc1[k] = fma(w, (double)v.y, acc1[k]);
                }
            }
        }
    }
}

// blockDim = (32, BP_ROWS); each thread backprojects the BP_NZ voxels
// (ix, iy, z0 .. z0 + BP_NZ - 1), z0 = blockIdx.z * BP_NZ, for every view of
// the launch.
// MULTI = false: one view (the reference's loop); the view loop and the
// per-view outputs exist only in the ordered-subset instantiation, so that
// the single-view kernel keeps its registers (and resident blocks).
// GEO64: FP64 geometry and normaliser (bp_gather_view64; one view).
// NZ (voxels per thread along z) and ROWS (voxel rows per block) are the
// launch shape the driver's tuning may choose; every shape gives the same
// bits (each voxel's terms and their order do not depend on it).
template <int K, int MODE, bool MULTI = false, bool PROVEN = false, bool GEO64 = false,
          int NZ = BP_NZ, int ROWS = BP_ROWS>
__global__ void __launch_bounds__(256, (bp_min_blocks<GEO64, MULTI, NZ>())) bp_kernel(const BPArgs p) {
    __shared__ float tile[NZ][ROWS][33];
    const Geom &g = p.g;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * ROWS, z0 = blockIdx.z * NZ;
    const int ix = x0 + tx, iy = y0 + ty;
    const bool active = ix < g.nx && iy < g.ny;
    const int64_t plane = (int64_t)g.nx * g.ny, V = plane * g.nz, NP = (int64_t)g.na * g.nb;
    const int nv = MULTI ? p.n_views : 1;

    float qsum[NZ];
#pragma unroll
    for (int k = 0; k < NZ; k++) qsum[k] = 0.0f;
    for (int v = 0; v < nv; v++) {
        float acc0[NZ], acc1[NZ];
#pragma unroll
        for (int k = 0; k < NZ; k++) { acc0[k] = 0.0f; acc1[k] = 0.0f; }
        const float angle = MULTI ? p.angles[v] : p.angle;
        double acc64[NZ];
        if (GEO64) {
            static_assert(!GEO64 || !MULTI, "FP64 geometry: one view per launch");
#pragma unroll
            for (int k = 0; k < NZ; k++) acc64[k] = 0.0;
            if (active) bp_gather_view64<K, NZ>(p, angle, p.proj, p.pair, ix, iy, z0, acc0, acc64);
        } else if (active) {
            bp_gather_view<K, PROVEN, NZ>(p, angle, p.proj, p.pair + v * NP, ix, iy, z0, acc0,
                                          acc1, v);
        }
#pragma unroll
        for (int k = 0; k < NZ; k++) {
            const int iz = z0 + k;
            if (!(active && iz < g.nz)) continue;
            const int64_t id = ix + (int64_t)iy * g.nx + iz * plane;
            if (MODE == BP_PLAIN) {
                p.out[id] = acc0[k];
                continue;
            }
            float q = GEO64 ? (float)((double)acc0[k] / acc64[k])
                            : acc0[k] / acc1[k];    // cu_division.cu:20
            if (isnan(q) || isinf(q)) q = 0.0f;     // :21-24
            if (MODE == BP_DIV) {
                if (p.out) p.out[id + v * V] = q;
                const cudaSurfaceObject_t s = MULTI ? p.outSurfs[v] : p.outSurf;
                if (s) surf3Dwrite(q, s, ix * (int)sizeof(float), iy, iz, cudaBoundaryModeZero);
            } else {
                qsum[k] = (!MULTI || v == 0) ? q : qsum[k] + q;  // subset: summed in view order
            }
        }
    }
    if (MODE != BP_DIV_ADD) return;
#pragma unroll
    for (int k = 0; k < NZ; k++) {
        const int iz = z0 + k;
        float val = 0.0f;
        if (active && iz < g.nz) {
            const int64_t id = ix + (int64_t)iy * g.nx + iz * plane;
            val = __fmaf_rn(qsum[k], p.lambda, p.out[id]);  // cu_add.cu:17
            p.out[id] = val;
        }
        tile[k][ty][tx] = val;
    }
    if (p.outT != nullptr) {
        __syncthreads();
        // transposed store outT[iy + ix*ny + iz*nx*ny]: ROWS consecutive iy per ix
        const int t = ty * 32 + tx;
        const int lx = t / ROWS, ly = t % ROWS;
        const int ixT = x0 + lx, iyT = y0 + ly;
        if (ixT < g.nx && iyT < g.ny) {
#pragma unroll
            for (int k = 0; k < NZ; k++) {
                const int iz = z0 + k;
                if (iz < g.nz) p.outT[iyT + (int64_t)ixT * g.ny + iz * plane] = tile[k][ly][lx];
            }
        }
    }
}

}  // namespace mcsart
