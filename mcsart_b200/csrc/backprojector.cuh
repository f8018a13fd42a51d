// Gather-form backprojector (the reference's kernel_backprojection,
// src/cu_backprojection.cu:49-170), restructured for B200.
//
// Reference semantics kept exactly: voxel centre with integer nx/2 (:66-68);
// six boundary points, i.e. an axis-aligned unit square in the rotated frame
// plus the voxel's top and bottom (:82-97); magnification SD/(x+SO) (:105-122);
// bounding box in detector index units a/da - ai + 0.5 (:135-138); unnormalised
// overlap weights wa*wb (:150-168); __sinf/__cosf of the angle (:62-63).
// The projection is read straight from global memory: the reference's texture
// fetch happens at texel centres (:167) and so returns the texel itself, which
// removes the per-call cudaMalloc3DArray + copy (:10-37).
//
// Restructured for the hardware: one thread per voxel (no atomics, so runs are
// bitwise reproducible), 32x32 voxel tiles per block for coalesced stores and
// a shared-memory transpose when the y-fastest copy of the volume must be kept
// current; two projections (SART residual and ones-projection, packed as
// float2) are gathered with one set of weights and the SART division
// (src/cu_division.cu:20-24) and update (src/cu_add.cu:17) run in the epilogue.
#pragma once

#include "common.cuh"

namespace mcsart {

enum BPMode { BP_PLAIN = 0, BP_DIV = 1, BP_DIV_ADD = 2 };

struct BPBox {
    float amin, amax, bmin, bmax;
};

// src/cu_backprojection.cu:66-138 for voxel (ix, iy, iz).
__device__ __forceinline__ BPBox bp_box(int ix, int iy, int iz, float cphi, float sphi,
                                        const Geom &g) {
    const float xc = (float)ix - g.nx / 2 + 0.5f;
    const float yc = (float)iy - g.ny / 2 + 0.5f;
    const float zc = (float)iz - g.nz / 2 + 0.5f;
    // rotated voxel centre; the boundary points differ by +-0.5 from it.  The
    // products are fused explicitly in the order that reproduces the
    // reference kernel bit for bit (":80-95" as compiled), so that the result
    // does not depend on how the compiler contracts after unrolling.
    const float t = __fmaf_rn(yc, sphi, __fmul_rn(xc, cphi));
    const float u = __fmaf_rn(yc, cphi, __fmul_rn(-xc, sphi));
    const float tl = t - 0.5f, tr = t + 0.5f, ul = u - 0.5f, ur = u + 0.5f;
    const float rl = g.SD / (tl + g.SO);  // points ll and lr
    const float rr = g.SD / (tr + g.SO);  // points rr and rl
    const float r0 = g.SD / (t + g.SO);   // top and bottom
    const float all = rl * ul, alr = rl * ur, arr = rr * ur, arl = rr * ul, at = r0 * u;
    const float bl = rl * zc, br = rr * zc, bt = r0 * (zc + 0.5f), bb = r0 * (zc - 0.5f);
    float amax = fmaxf(fmaxf(fmaxf(all, arr), fmaxf(alr, arl)), at);
    float amin = fminf(fminf(fminf(all, arr), fminf(alr, arl)), at);
    float bmax = fmaxf(fmaxf(fmaxf(bl, br), fmaxf(bl, br)), fmaxf(bt, bb));
    float bmin = fminf(fminf(fminf(bl, br), fminf(bl, br)), fminf(bt, bb));
    BPBox box;
    box.amax = amax / g.da - g.ai + 0.5f;
    box.amin = amin / g.da - g.ai + 0.5f;
    box.bmax = bmax / g.db - g.bi + 0.5f;
    box.bmin = bmin / g.db - g.bi + 0.5f;
    return box;
}

// Overlap-weighted gather of K projections over the box (:150-168).
template <int K>
__device__ __forceinline__ void bp_gather(const BPBox &bx, const float *p1, const float2 *p2,
                                          const Geom &g, float *acc) {
    const float alim = ((float)g.na < bx.amax) ? (float)g.na : bx.amax;  // MIN(na, a_max)
    const float blim = ((float)g.nb < bx.bmax) ? (float)g.nb : bx.bmax;
    const int ia0 = max(0, (int)floorf(fmaxf(bx.amin, -1.0f)));
    const int ib0 = max(0, (int)floorf(fmaxf(bx.bmin, -1.0f)));
    for (int ia = ia0; (float)ia < alim; ia++) {
        const float wa = fminf(ia + 1.0f, bx.amax) - fmaxf(ia + 0.0f, bx.amin);
        for (int ib = ib0; (float)ib < blim; ib++) {
            const float wb = fminf(ib + 1.0f, bx.bmax) - fmaxf(ib + 0.0f, bx.bmin);
            const float w = wa * wb;
            const int64_t pix = ia + (int64_t)ib * g.na;
            if (K == 1) {
                acc[0] = __fmaf_rn(w, __ldg(p1 + pix), acc[0]);
            } else {
                const float2 v = __ldg(p2 + pix);
                acc[0] = __fmaf_rn(w, v.x, acc[0]);
                acc[1] = __fmaf_rn(w, v.y, acc[1]);
            }
        }
    }
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
};

// blockDim = (32, 8); each block covers a 32x32 (x, y) tile of slice blockIdx.z.
template <int K, int MODE>
__global__ void __launch_bounds__(256) bp_kernel(const BPArgs p) {
    __shared__ float tile[32][33];
    const Geom &g = p.g;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32, iz = blockIdx.z;
    const int ix = x0 + tx;
    const float sphi = __sinf(p.angle), cphi = __cosf(p.angle);
    const int64_t slice = (int64_t)iz * g.nx * g.ny;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int ly = ty + 8 * k, iy = y0 + ly;
        float val = 0.0f;
        if (ix < g.nx && iy < g.ny) {
            const BPBox box = bp_box(ix, iy, iz, cphi, sphi, g);
            float acc[2] = {0.0f, 0.0f};
            bp_gather<K>(box, p.proj, p.pair, g, acc);
            const int64_t id = ix + (int64_t)iy * g.nx + slice;
            if (MODE == BP_PLAIN) {
                val = acc[0];
                p.out[id] = val;
            } else {
                float q = acc[0] / acc[1];              // cu_division.cu:20
                if (isnan(q) || isinf(q)) q = 0.0f;     // :21-24
                if (MODE == BP_DIV) {
                    val = q;
                    if (p.out) p.out[id] = val;
                    if (p.outSurf)
                        surf3Dwrite(val, p.outSurf, ix * (int)sizeof(float), iy, iz,
                                    cudaBoundaryModeZero);
                } else {
                    val = __fmaf_rn(q, p.lambda, p.out[id]);  // cu_add.cu:17
                    p.out[id] = val;
                }
            }
        }
        if (MODE == BP_DIV_ADD) tile[ly][tx] = val;
    }
    if (MODE == BP_DIV_ADD && p.outT != nullptr) {
        __syncthreads();
        // transposed store: outT[iy + ix*ny + iz*nx*ny]
        const int iyT = y0 + tx;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int lx = ty + 8 * k, ixT = x0 + lx;
            if (ixT < g.nx && iyT < g.ny) p.outT[iyT + (int64_t)ixT * g.ny + slice] = tile[tx][lx];
        }
    }
}

}  // namespace mcsart
