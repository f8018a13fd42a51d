// Distance-driven forward projector (the reference's kernel_projection,
// src/cu_projection.cu:15-145), restructured for B200.
//
// Reference semantics kept exactly: per-ray driving axis |x21| > |y21| (:39);
// the four in-plane edge ratios yl/xl, yl/xr, yr/xl, yr/xr and their min/max
// (:54-64); axial edges zl/x21, zr/x21 (:71-77); integer ny/2, nz/2 offsets
// against float nx/2 (:52,55,72); overlap weights normalised by the footprint
// width (:83,86); loops clamped to the volume.
//
// Restructured for the hardware:
//   * one thread per ray (the reference runs 4 redundant threads per ray that
//     race on a non-atomic +=);
//   * the slabs of a ray are split across `groups` warps of a block and
//     recombined in a fixed order through shared memory (deterministic);
//   * the loop-invariant ratios are hoisted out of the slab loop;
//   * x-driven rays read a y-fastest copy of the volume so that the 32 lanes
//     of a warp (adjacent detector columns) gather adjacent addresses;
//   * up to three volumes are projected with one set of weights, the
//     projection of a ones-volume (sum of weights) comes for free, and the
//     SART residual, its norm partial sums and the packing for the
//     backprojector are done in the epilogue.
#pragma once

#include "backprojector.cuh"
#include "common.cuh"

namespace mcsart {

enum FPMode { FP_PLAIN = 0, FP_IMAGE = 1, FP_MOTION = 2 };

struct RayGeom {
    float r0, r1, r2, r3;  // in-plane edge ratios
    float rz0, rz1;        // axial edge ratios
    float u_off;           // source coordinate along the in-plane axis (y1 or x1)
    float u_half;          // (float)(nu/2), integer division
    float d_half;          // (float)nd/2, float division
    float src_d;           // source coordinate along the driving axis (x1 or y1)
    int nd, nu;
    bool xdrive;
};

// src/cu_projection.cu:23-39,48-51,67-68,101-104,120-121 for ray (ia, ib).
// Every operation is pinned with an explicit rounding intrinsic: which
// products the compiler fuses into fma's otherwise depends on the surrounding
// code.  The fused forms below are the ones whose results equal the
// reference kernel's bit for bit; they were selected by running every
// combination of candidate forms against the rebuilt reference on ~300k rays
// (3 geometries, 30 angles, both driving axes): x2 and y2 fuse the product
// with cos, the edge offsets (da/2)*sin, (da/2)*cos fuse into the edges, the
// axial edges are z2 -+ db/2 after rounding z2, the source offset is
// subtracted unfused.
__device__ __forceinline__ RayGeom ray_geom(float cphi, float sphi, int ia, int ib,
                                            const Geom &g) {
    const float x1 = -__fmul_rn(g.SO, cphi), y1 = -__fmul_rn(g.SO, sphi);
    const float x20 = __fsub_rn(g.SD, g.SO);
    const float y20 = __fmul_rn(__fadd_rn((float)ia, g.ai), g.da);
    const float x2 = __fmaf_rn(x20, cphi, -__fmul_rn(y20, sphi));
    const float y2 = __fmaf_rn(y20, cphi, __fmul_rn(x20, sphi));
    const float z2 = __fmul_rn(__fadd_rn((float)ib, g.bi), g.db);  // z21 = z2 - z1, z1 = 0
    const float x21 = __fsub_rn(x2, x1), y21 = __fsub_rn(y2, y1);
    RayGeom r;
    r.xdrive = fabsf(x21) > fabsf(y21);
    const float hda = __fdiv_rn(g.da, 2.0f), hdb = __fdiv_rn(g.db, 2.0f);
    const float xl = __fmaf_rn(-hda, sphi, x21), xr = __fmaf_rn(hda, sphi, x21);
    const float yl = __fmaf_rn(-hda, cphi, y21), yr = __fmaf_rn(hda, cphi, y21);
    const float zl = __fsub_rn(z2, hdb), zr = __fadd_rn(z2, hdb);
    if (r.xdrive) {
        r.r0 = __fdiv_rn(yl, xl); r.r1 = __fdiv_rn(yl, xr);
        r.r2 = __fdiv_rn(yr, xl); r.r3 = __fdiv_rn(yr, xr);
        r.rz0 = __fdiv_rn(zl, x21); r.rz1 = __fdiv_rn(zr, x21);
        r.u_off = y1; r.u_half = (float)(g.ny / 2);
        r.d_half = __fdiv_rn((float)g.nx, 2.0f); r.src_d = x1;
        r.nd = g.nx; r.nu = g.ny;
    } else {
        r.r0 = __fdiv_rn(xl, yl); r.r1 = __fdiv_rn(xl, yr);
        r.r2 = __fdiv_rn(xr, yl); r.r3 = __fdiv_rn(xr, yr);
        r.rz0 = __fdiv_rn(zl, y21); r.rz1 = __fdiv_rn(zr, y21);
        r.u_off = x1; r.u_half = (float)(g.nx / 2);
        r.d_half = __fdiv_rn((float)g.ny, 2.0f); r.src_d = y1;
        r.nd = g.ny; r.nu = g.nx;
    }
    return r;
}

template <typename VT, int K> struct FPVolumes {
    const VT *std[K];  // x-fastest volumes
    const VT *tr[K];   // y-fastest copies (tr[k][iy + ix*ny + iz*nx*ny]) or nullptr
};

// The K volumes' values at voxel offset a into t[0..K-1]: one load per
// volume, or (PAIR, three volumes) the second and third interleaved in one
// array, base[1][2a], base[1][2a + 1], read with one two-element load.
template <int K, bool PAIR, typename VT>
__device__ __forceinline__ void fp_voxel(const VT *const *base, int64_t a, float *t) {
    static_assert(!PAIR || K == 3, "paired volumes come with three volumes");
    if (PAIR) {
        t[0] = ldv(base[0], a);
        const float2 q = ldv2(base[1], a);
        t[1] = q.x;
        t[2] = q.y;
    } else {
#pragma unroll
        for (int k = 0; k < K; k++) t[k] = ldv(base[k], a);
    }
}

// Ray-sum order.  SUM_REF accumulates every voxel term straight into the ray
// sum in the reference's order (slabs, then in-plane, then axial index,
// acc = fma(v*w_u, w_z, acc), cu_projection.cu:81-88), so that results are
// bitwise those of the reference kernel.  SUM_PLAIN / SUM_KAHAN first sum the
// (at most a few) terms of one slab and then add the slab sum to the ray sum,
// plainly or with Kahan compensation; they allow the slabs of a ray to be
// split across warps.
enum SumMode { SUM_REF = 0, SUM_PLAIN = 1, SUM_KAHAN = 2 };

// Accumulates the footprint of slabs [d0, d1) of one ray into s[0..K-1]
// (volume sums) and sw (sum of weights = projection of a ones-volume).
template <int K, bool ONES, int SUM, typename VT>
__device__ __forceinline__ void ray_slabs(const RayGeom &r, const FPVolumes<VT, K> &v,
                                          const Geom &g, int d0, int d1, float *s, float &sw) {
    const VT *base[K];
    int64_t su, sd;
    const int64_t sz = (int64_t)g.nx * g.ny;
    if (r.xdrive) {
        if (v.tr[0] != nullptr) {
#pragma unroll
            for (int k = 0; k < K; k++) base[k] = v.tr[k];
            su = 1; sd = g.ny;
        } else {
#pragma unroll
            for (int k = 0; k < K; k++) base[k] = v.std[k];
            su = g.nx; sd = 1;
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; k++) base[k] = v.std[k];
        su = 1; sd = g.nx;
    }
    const float z_half = (float)(g.nz / 2);
    float acc[K], cmp[K], accw = 0.0f, cmpw = 0.0f;
#pragma unroll
    for (int k = 0; k < K; k++) { acc[k] = 0.0f; cmp[k] = 0.0f; }

    for (int d = d0; d < d1; d++) {
        // :52 / :105
        const float dc = __fsub_rn(__fsub_rn(__fadd_rn((float)d, 0.5f), r.d_half), r.src_d);
        // :54-61 / :107-114 ("ratio * xc + y1 + ny / 2")
        const float c0 = __fadd_rn(__fmaf_rn(r.r0, dc, r.u_off), r.u_half);
        const float c1 = __fadd_rn(__fmaf_rn(r.r1, dc, r.u_off), r.u_half);
        const float c2 = __fadd_rn(__fmaf_rn(r.r2, dc, r.u_off), r.u_half);
        const float c3 = __fadd_rn(__fmaf_rn(r.r3, dc, r.u_off), r.u_half);
        const float ui1 = fminf(fminf(c0, c1), fminf(c2, c3));
        const float ui2 = fmaxf(fmaxf(c0, c1), fmaxf(c2, c3));
        // :71-77 / :124-130 ("ratio * xc + z1 + nz / 2", z1 = 0)
        const float cz0 = __fadd_rn(__fmul_rn(r.rz0, dc), z_half);
        const float cz1 = __fadd_rn(__fmul_rn(r.rz1, dc), z_half);
        const float zi1 = fminf(cz0, cz1), zi2 = fmaxf(cz0, cz1);
        const int U1 = (int)floorf(ui1), U2 = (int)floorf(ui2);
        const int Z1 = (int)floorf(zi1), Z2 = (int)floorf(zi2);
        const float du = __fsub_rn(ui2, ui1), dz = __fsub_rn(zi2, zi1);
        if (SUM == SUM_REF && U2 - U1 <= 1 && Z2 - Z1 <= 1) {
            // The footprint fits a 2x2 voxel window (U1, U1+1) x (Z1, Z1+1): the
            // reference's loops visit its in-volume members in this order, so
            // evaluating the four candidates with predication gives the same
            // sequence of fma's, without data-dependent trip counts.
            const bool u0 = U1 >= 0 && U1 <= r.nu - 1;
            const bool u1 = U1 + 1 <= U2 && U1 + 1 >= 0 && U1 + 1 <= r.nu - 1;
            const bool z0 = Z1 >= 0 && Z1 <= g.nz - 1;
            const bool z1 = Z1 + 1 <= Z2 && Z1 + 1 >= 0 && Z1 + 1 <= g.nz - 1;
            const float fu0 = (float)U1, fu1 = (float)(U1 + 1);
            const float fz0 = (float)Z1, fz1 = (float)(Z1 + 1);
            const float wu0 = __fdiv_rn(__fsub_rn(fminf(__fadd_rn(fu0, 1.0f), ui2), fmaxf(fu0, ui1)), du);
            const float wu1 = __fdiv_rn(__fsub_rn(fminf(__fadd_rn(fu1, 1.0f), ui2), fmaxf(fu1, ui1)), du);
            const float wz0 = __fdiv_rn(__fsub_rn(fminf(__fadd_rn(fz0, 1.0f), zi2), fmaxf(fz0, zi1)), dz);
            const float wz1 = __fdiv_rn(__fsub_rn(fminf(__fadd_rn(fz1, 1.0f), zi2), fmaxf(fz1, zi1)), dz);
            // in-bounds addresses for every candidate (unused ones are not read)
            const int cu0 = min(max(U1, 0), r.nu - 1), cu1 = min(max(U1 + 1, 0), r.nu - 1);
            const int cz0 = min(max(Z1, 0), g.nz - 1), cz1 = min(max(Z1 + 1, 0), g.nz - 1);
            const int64_t r0 = (int64_t)cu0 * su + (int64_t)d * sd;
            const int64_t r1 = (int64_t)cu1 * su + (int64_t)d * sd;
            const int64_t a00 = r0 + (int64_t)cz0 * sz, a01 = r0 + (int64_t)cz1 * sz;
            const int64_t a10 = r1 + (int64_t)cz0 * sz, a11 = r1 + (int64_t)cz1 * sz;
#pragma unroll
            for (int k = 0; k < K; k++) {
                if (u0 && z0) acc[k] = __fmaf_rn(__fmul_rn(ldv(base[k], a00), wu0), wz0, acc[k]);
                if (u0 && z1) acc[k] = __fmaf_rn(__fmul_rn(ldv(base[k], a01), wu0), wz1, acc[k]);
                if (u1 && z0) acc[k] = __fmaf_rn(__fmul_rn(ldv(base[k], a10), wu1), wz0, acc[k]);
                if (u1 && z1) acc[k] = __fmaf_rn(__fmul_rn(ldv(base[k], a11), wu1), wz1, acc[k]);
            }
            if (ONES) {
                if (u0 && z0) accw = __fmaf_rn(wu0, wz0, accw);
                if (u0 && z1) accw = __fmaf_rn(wu0, wz1, accw);
                if (u1 && z0) accw = __fmaf_rn(wu1, wz0, accw);
                if (u1 && z1) accw = __fmaf_rn(wu1, wz1, accw);
            }
            continue;
        }
        const int u_lo = max(0, U1), u_hi = min(r.nu - 1, U2);
        const int z_lo = max(0, Z1), z_hi = min(g.nz - 1, Z2);
        if (u_lo > u_hi || z_lo > z_hi) continue;
        float ss[K], ssw = 0.0f;
#pragma unroll
        for (int k = 0; k < K; k++) ss[k] = 0.0f;
        for (int u = u_lo; u <= u_hi; u++) {
            // :83 / :136
            const float wu = __fdiv_rn(__fsub_rn(fminf(__fadd_rn((float)u, 1.0f), ui2), fmaxf((float)u, ui1)), du);
            const int64_t row = (int64_t)u * su + (int64_t)d * sd;
            for (int z = z_lo; z <= z_hi; z++) {
                // :86 / :139
                const float wz = __fdiv_rn(__fsub_rn(fminf(__fadd_rn((float)z, 1.0f), zi2), fmaxf((float)z, zi1)), dz);
                const int64_t a = row + (int64_t)z * sz;
                if (SUM == SUM_REF) {
#pragma unroll
                    for (int k = 0; k < K; k++)
                        acc[k] = __fmaf_rn(__fmul_rn(ldv(base[k], a), wu), wz, acc[k]);  // :87 / :140
                    if (ONES) accw = __fmaf_rn(wu, wz, accw);
                } else {
#pragma unroll
                    for (int k = 0; k < K; k++) ss[k] = __fmaf_rn(__fmul_rn(ldv(base[k], a), wu), wz, ss[k]);
                    if (ONES) ssw = __fmaf_rn(wu, wz, ssw);
                }
            }
        }
        if (SUM == SUM_REF) continue;
#pragma unroll
        for (int k = 0; k < K; k++) {
            if (SUM == SUM_KAHAN) {
                const float y = ss[k] - cmp[k];
                const float t = acc[k] + y;
                cmp[k] = (t - acc[k]) - y;
                acc[k] = t;
            } else {
                acc[k] += ss[k];
            }
        }
        if (ONES) {
            if (SUM == SUM_KAHAN) {
                const float y = ssw - cmpw;
                const float t = accw + y;
                cmpw = (t - accw) - y;
                accw = t;
            } else {
                accw += ssw;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < K; k++) s[k] = acc[k];
    sw = accw;
}

// ------------------------------------------------------------------------
// FP64 geometry (options.geom64, with the split summation modes): the same
// footprint formulas as ray_geom / ray_slabs (src/cu_projection.cu:23-144),
// every boundary coordinate and overlap weight in FP64; the volume terms
// v * w are accumulated in FP32 (plainly or Kahan-compensated), the weight
// sum (the projection of a ones-volume, the SART row normaliser) in FP64.
struct RayGeom64 {
    double r0, r1, r2, r3, rz0, rz1;
    double u_off, u_half, d_half, src_d;
    int nd, nu;
    bool xdrive;
};

__device__ __forceinline__ RayGeom64 ray_geom64(double cphi, double sphi, int ia, int ib,
                                                const Geom &g) {
    const double SO = g.SO, SD = g.SD, da = g.da, db = g.db;
    const double x1 = -SO * cphi, y1 = -SO * sphi;  // :25-26
    const double x20 = SD - SO, y20 = ((double)ia + (double)g.ai) * da;
    const double x2 = x20 * cphi - y20 * sphi, y2 = y20 * cphi + x20 * sphi;
    const double z2 = ((double)ib + (double)g.bi) * db;
    const double x21 = x2 - x1, y21 = y2 - y1;
    RayGeom64 r;
    r.xdrive = fabs(x21) > fabs(y21);  // :39
    const double hda = da / 2.0, hdb = db / 2.0;
    const double xl = x21 - hda * sphi, xr = x21 + hda * sphi;
    const double yl = y21 - hda * cphi, yr = y21 + hda * cphi;
    const double zl = z2 - hdb, zr = z2 + hdb;
    if (r.xdrive) {
        r.r0 = yl / xl; r.r1 = yl / xr; r.r2 = yr / xl; r.r3 = yr / xr;
        r.rz0 = zl / x21; r.rz1 = zr / x21;
        r.u_off = y1; r.u_half = (double)(g.ny / 2);
        r.d_half = (double)g.nx / 2.0; r.src_d = x1;
        r.nd = g.nx; r.nu = g.ny;
    } else {
        r.r0 = xl / yl; r.r1 = xl / yr; r.r2 = xr / yl; r.r3 = xr / yr;
        r.rz0 = zl / y21; r.rz1 = zr / y21;
        r.u_off = x1; r.u_half = (double)(g.nx / 2);
        r.d_half = (double)g.ny / 2.0; r.src_d = y1;
        r.nd = g.ny; r.nu = g.nx;
    }
    return r;
}

// Slabs [d0, d1) of one ray with FP64 geometry: s[k] (FP32 sums of the
// volumes' terms) and sw (FP64 sum of the weights).
template <int K, bool ONES, int SUM, typename VT>
__device__ __forceinline__ void ray_slabs64(const RayGeom64 &r, const FPVolumes<VT, K> &v,
                                            const Geom &g, int d0, int d1, float *s, double &sw) {
    const VT *base[K];
    int64_t su, sd;
    const int64_t sz = (int64_t)g.nx * g.ny;
    if (r.xdrive && v.tr[0] != nullptr) {
#pragma unroll
        for (int k = 0; k < K; k++) base[k] = v.tr[k];
        su = 1; sd = g.ny;
    } else {
#pragma unroll
        for (int k = 0; k < K; k++) base[k] = v.std[k];
        if (r.xdrive) { su = g.nx; sd = 1; } else { su = 1; sd = g.nx; }
    }
    const double z_half = (double)(g.nz / 2);
    float acc[K], cmp[K];
#pragma unroll
    for (int k = 0; k < K; k++) { acc[k] = 0.0f; cmp[k] = 0.0f; }
    double accw = 0.0;
    for (int d = d0; d < d1; d++) {
        const double dc = ((double)d + 0.5) - r.d_half - r.src_d;  // :52 / :105
        const double c0 = r.r0 * dc + r.u_off + r.u_half, c1 = r.r1 * dc + r.u_off + r.u_half;
        const double c2 = r.r2 * dc + r.u_off + r.u_half, c3 = r.r3 * dc + r.u_off + r.u_half;
        const double ui1 = fmin(fmin(c0, c1), fmin(c2, c3));
        const double ui2 = fmax(fmax(c0, c1), fmax(c2, c3));
        const double cz0 = r.rz0 * dc + z_half, cz1 = r.rz1 * dc + z_half;  // :71-77
        const double zi1 = fmin(cz0, cz1), zi2 = fmax(cz0, cz1);
        // loop bounds clamped to the volume before the integer conversion
        const int u_lo = max(0, (int)floor(fmax(ui1, -1.0)));
        const int u_hi = min(r.nu - 1, (int)floor(fmin(ui2, (double)r.nu)));
        const int z_lo = max(0, (int)floor(fmax(zi1, -1.0)));
        const int z_hi = min(g.nz - 1, (int)floor(fmin(zi2, (double)g.nz)));
        if (u_lo > u_hi || z_lo > z_hi) continue;
        const double du = ui2 - ui1, dz = zi2 - zi1;
        float ss[K];
#pragma unroll
        for (int k = 0; k < K; k++) ss[k] = 0.0f;
        for (int u = u_lo; u <= u_hi; u++) {
            const double wu = (fmin(u + 1.0, ui2) - fmax((double)u, ui1)) / du;  // :83 / :136
            const int64_t row = (int64_t)u * su + (int64_t)d * sd;
            for (int z = z_lo; z <= z_hi; z++) {
                const double wz = (fmin(z + 1.0, zi2) - fmax((double)z, zi1)) / dz;  // :86 / :139
                const double w = wu * wz;
                const float wf = (float)w;
                const int64_t a = row + (int64_t)z * sz;
#pragma unroll
                for (int k = 0; k < K; k++) ss[k] = __fmaf_rn(ldv(base[k], a), wf, ss[k]);
                if (ONES) accw += w;
            }
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            if (SUM == SUM_KAHAN) {
                const float y = ss[k] - cmp[k];
                const float t = acc[k] + y;
                cmp[k] = (t - acc[k]) - y;
                acc[k] = t;
            } else {
                acc[k] += ss[k];
            }
        }
    }
#pragma unroll
    for (int k = 0; k < K; k++) s[k] = acc[k];
    sw = accw;
}

template <typename VT, int K, typename MT = VT> struct FPArgs {
    FPVolumes<VT, K> vol;
    Geom g;
    float angle;            // used when angles == nullptr
    const float *angles;    // per-view angles (device), view = blockIdx.z
    int mode;
    // FP_PLAIN: out[view*na*nb + ia + ib*na] = s0
    float *out;
    // FP_IMAGE / FP_MOTION
    const MT *meas;     // measured projection of this view
    float *resid;       // residual output (nullable)
    float2 *bp_in;      // (residual, ones-projection) pairs for the backprojector
    double2 *norm_part; // per-block (sum b^2, sum r^2)
    // several views per launch (fp_ref_kernel, view = blockIdx.z): meas,
    // resid and bp_in advance by na*nb per view, norm_part by the blocks of
    // one view, and the volumes by vol_stride elements per view (0: every
    // view projects the same volumes)
    int64_t vol_stride;
    // when set, also write each view's backprojector column data (bp_column
    // for every (ix, iy), index ix + iy*nx, view j of a several-view launch at
    // + j*nx*ny) for the backprojector launch that follows
    float4 *bpcolA;  // amin, amax, rl, rr
    float *bpcolB;   // r0
};

// ------------------------------------------------------------------------
// Column-shared projector for the reference summation order (SUM_REF).
//
// Every ray of one detector column ia has the same in-plane geometry: the
// driving axis, the four edge ratios and so, per slab, the in-plane voxel
// range U1..U2 and weights w_u (only the axial part depends on the row ib,
// through z2).  A block of FPC_COLS columns x FPC_ROWS rows computes the
// in-plane part once per (column, slab) into shared memory (SlabC: weights,
// slab distance, clamped voxel-row offsets, visit flags), FPC_CHUNK slabs at
// a time, and every ray then adds its axial part and its terms in the
// reference's order.  The per-ray arithmetic is unchanged, so the sums are
// bitwise those of the per-ray form (and of the reference kernel).
#ifndef MCSART_FP_COLS
#define MCSART_FP_COLS 16
#endif
#ifndef MCSART_FP_ROWS
#define MCSART_FP_ROWS 8
#endif
constexpr int FPC_COLS = MCSART_FP_COLS, FPC_ROWS = MCSART_FP_ROWS;
constexpr int FPC_THREADS = FPC_COLS * FPC_ROWS;
// at least 512 threads per SM: lets the compiler use up to 128 registers
constexpr int FPC_MIN_BLOCKS = 512 / FPC_THREADS;
// Slabs per table fill (a 32 KB table per block; 64 measured 1 % faster than
// 32 at both benchmark sizes).
constexpr int FPC_CHUNK = 64;
// Slabs per group in the 2x2 fast path: with three volumes 4 (more loads in
// flight within the 128-register budget: the DVF pass's projector 6 % faster
// than with 2), with one volume 2 (4 spills inside the 80 registers that keep
// 6 blocks per SM).
template <int K> constexpr int fp_group() { return K >= 3 ? 4 : 2; }

// In-plane footprint of one slab.  U2 - U1 <= 1: (a, b) = weights of voxels
// U1 and U1 + 1; otherwise (a, b) = (ui1, ui2), the footprint edges.
struct SlabU {
    int U1, U2;
    float a, b;
};

// :52 / :105: distance of slab d's centre from the source along the driving
// axis (d < 2^20, validate_geom: mk_i2f is exact).
__device__ __forceinline__ float slab_dc(const RayGeom &r, int d) {
    return __fsub_rn(__fsub_rn(__fadd_rn(mk_i2f(d), 0.5f), r.d_half), r.src_d);
}

// :52-63 / :105-116 for slab d of the ray's column.
__device__ __forceinline__ SlabU slab_u(const RayGeom &r, int d) {
    const float dc = slab_dc(r, d);
    const float c0 = __fadd_rn(__fmaf_rn(r.r0, dc, r.u_off), r.u_half);
    const float c1 = __fadd_rn(__fmaf_rn(r.r1, dc, r.u_off), r.u_half);
    const float c2 = __fadd_rn(__fmaf_rn(r.r2, dc, r.u_off), r.u_half);
    const float c3 = __fadd_rn(__fmaf_rn(r.r3, dc, r.u_off), r.u_half);
    const float ui1 = fminf(fminf(c0, c1), fminf(c2, c3));
    const float ui2 = fmaxf(fmaxf(c0, c1), fmaxf(c2, c3));
    SlabU e;
    float fu0, fu1;
    if (fabsf(ui1) < MK_MAGIC_RANGE && fabsf(ui2) < MK_MAGIC_RANGE) {
        e.U1 = mk_floor(ui1, fu0);
        e.U2 = mk_floor_i(ui2);
        fu1 = __fadd_rn(fu0, 1.0f);  // (float)(U1 + 1), exact below 2^22
    } else {
        e.U1 = (int)floorf(ui1);
        e.U2 = (int)floorf(ui2);
        fu0 = (float)e.U1;
        fu1 = (float)(e.U1 + 1);
    }
    if (e.U2 - e.U1 <= 1) {
        const float du = __fsub_rn(ui2, ui1);  // :83 / :136
        const float n0 = __fsub_rn(fminf(__fadd_rn(fu0, 1.0f), ui2), fmaxf(fu0, ui1));
        const float n1 = __fsub_rn(fminf(__fadd_rn(fu1, 1.0f), ui2), fmaxf(fu1, ui1));
        const float y = mk_recip(du);
        e.a = mk_div(n0, du, y);
        e.b = mk_div(n1, du, y);
        if (!(mk_den_ok(du) && mk_num_ok(n0) && mk_num_ok(n1))) {
            e.a = __fdiv_rn(n0, du);
            e.b = __fdiv_rn(n1, du);
        }
    } else {
        e.a = ui1;
        e.b = ui2;
    }
    return e;
}

// What every ray of one detector column shares for slab d, kept in shared
// memory: slab_u's footprint, the slab distance dc, the clamped offsets of
// the window's two in-plane voxel rows (cu * su + d * sd) and which of the two
// the reference's loops visit (:80-82 / :133-135).
struct __align__(16) SlabC {
    int r0, r1;
    float a, b;  // SlabU's
    float dc;
    int U1, U2;
    int flags;   // SC_U0 | SC_U1 | SC_NARROW (U2 - U1 <= 1) | SC_UANY
};
// SC_UANY: the reference's in-plane loop over max(0, U1) .. min(nu-1, U2) is
// not empty (:80-81 / :133-134)
constexpr int SC_U0 = 1, SC_U1 = 2, SC_NARROW = 4, SC_UANY = 8;

__device__ __forceinline__ SlabC slab_c(const RayGeom &r, int d, int su, int sd) {
    const SlabU e = slab_u(r, d);
    SlabC c;
    c.a = e.a;
    c.b = e.b;
    c.U1 = e.U1;
    c.U2 = e.U2;
    c.dc = slab_dc(r, d);
    const int U1 = e.U1, U2 = e.U2;
    const bool u0 = U1 >= 0 && U1 <= r.nu - 1;
    const bool u1 = U1 + 1 <= U2 && U1 + 1 >= 0 && U1 + 1 <= r.nu - 1;
    c.flags = (u0 ? SC_U0 : 0) | (u1 ? SC_U1 : 0) | (U2 - U1 <= 1 ? SC_NARROW : 0) |
              (U2 >= 0 && U1 <= r.nu - 1 ? SC_UANY : 0);
    const int cu0 = min(max(U1, 0), r.nu - 1), cu1 = min(max(U1 + 1, 0), r.nu - 1);
    c.r0 = cu0 * su + d * sd;
    c.r1 = cu1 * su + d * sd;
    return c;
}

// A 2x2 footprint window (U1, U1+1) x (Z1, Z1+1) of one slab: weights,
// clamped (always in-bounds) addresses and which of the four voxels the
// reference's loops visit (:80-88 / :133-141).
struct SlabZ {
    float wu0, wu1, wz0, wz1;
    int a00, a01, a10, a11;
    bool p00, p01, p10, p11;
};

// Axial part of slab d for this ray; true (and w filled) if the footprint is
// a 2x2 window whose weights the branch-free division computed exactly.
// zsafe: the ray's axial coordinates stay inside the range of the
// magic-number floor (otherwise the caller takes the general path).  CHECK:
// test the division's operand range here; without it the caller has shown it
// for every slab of the ray (ray_axial).  CLAMP: the four candidates'
// addresses are clamped to the volume, so that they can be loaded before the
// predicates are known; otherwise they are exact only where their predicate
// holds, and the caller loads under the predicate.  Voxel indices are
// 32-bit: volumes are validated to hold fewer than 2^31 voxels (the
// reference indexes with int as well).
template <bool CHECK, bool CLAMP = true>
__device__ __forceinline__ bool slab_window(const RayGeom &r, const Geom &g, const SlabC &c, int sz,
                                            float z_half, bool zsafe, SlabZ &w) {
    // :71-77 / :124-130 ("ratio * xc + z1 + nz / 2", z1 = 0)
    const float cz0 = __fadd_rn(__fmul_rn(r.rz0, c.dc), z_half);
    const float cz1 = __fadd_rn(__fmul_rn(r.rz1, c.dc), z_half);
    const float zi1 = fminf(cz0, cz1), zi2 = fmaxf(cz0, cz1);
    float fz0;
    const int Z1 = mk_floor(zi1, fz0);
    const float fz1 = __fadd_rn(fz0, 1.0f), fz2 = __fadd_rn(fz1, 1.0f);
    const float dz = __fsub_rn(zi2, zi1);
    // Z2 = floor(zi2) is Z1 (zi2 < Z1 + 1) or Z1 + 1 (zi2 < Z1 + 2) for a
    // window of at most two slices: compared against the exact floats
    // Z1 + 1, Z1 + 2 (zsafe: |zi| < 2^19)
    const bool two = zi2 >= fz1, narrow = zi2 < fz2;
    const unsigned nz = (unsigned)g.nz;
    // the reference's axial loop visits Z1 and (when Z2 = Z1 + 1) Z1 + 1,
    // clamped to the volume (:80-82 / :133-135)
    const bool u0 = c.flags & SC_U0, u1 = c.flags & SC_U1;
    const bool z0 = (unsigned)Z1 < nz;
    const bool z1 = two && (unsigned)Z1 + 1u < nz;
    w.p00 = u0 && z0;
    w.p01 = u0 && z1;
    w.p10 = u1 && z0;
    w.p11 = u1 && z1;
    w.wu0 = c.a;
    w.wu1 = c.b;
    const float n0 = __fsub_rn(fminf(fz1, zi2), fmaxf(fz0, zi1));
    const float n1 = __fsub_rn(fminf(fz2, zi2), fmaxf(fz1, zi1));
    const float y = mk_recip(dz);
    w.wz0 = mk_div(n0, dz, y);
    w.wz1 = mk_div(n1, dz, y);
    const bool exact = CHECK ? (mk_den_ok(dz) && mk_num_ok(n0) && mk_num_ok(n1)) : true;
    if (CLAMP) {
        const int cz0i = min(max(Z1, 0), g.nz - 1), cz1i = min(max(Z1 + 1, 0), g.nz - 1);
        w.a00 = c.r0 + cz0i * sz;
        w.a01 = c.r0 + cz1i * sz;
        w.a10 = c.r1 + cz0i * sz;
        w.a11 = c.r1 + cz1i * sz;
    } else {  // (unsigned: wraps instead of overflowing where Z1 is out of range)
        const unsigned zo = (unsigned)Z1 * (unsigned)sz;
        w.a00 = (int)((unsigned)c.r0 + zo);
        w.a01 = (int)((unsigned)w.a00 + (unsigned)sz);
        w.a10 = (int)((unsigned)c.r1 + zo);
        w.a11 = (int)((unsigned)w.a10 + (unsigned)sz);
    }
    // outside the division's checked range the caller takes the general path
    return (c.flags & SC_NARROW) && narrow && exact && zsafe;
}

// Per-ray facts about the axial footprint over all the ray's slabs, bounded
// from the ray's constants with rounding margins: the slab distance dc runs
// monotonically over [dc(0), dc(nd - 1)] and cz = rz * dc + nz/2 is linear in
// it, computed with an error below 2^-23 * max|cz|.
//  zsafe: |cz| < 2^19, inside the magic-number floor's range, so that also
//         dz = zi2 - zi1 < 2^20;
//  exact: additionally dc keeps one sign, dz >= 2^-19 (|rz1 - rz0| * |dc|
//         less the rounding) and no cz comes within 2^-50 of zero.  Then
//         every slab's division operands are in mk_div's checked range: dz is
//         in [2^-20, 2^20); n0 is either dz or (Z1 + 1) - zi1, a positive
//         multiple of ulp(zi1) >= 2^-73; n1, used only when Z2 = Z1 + 1, is
//         zi2 - (Z1 + 1), zero or a positive multiple of ulp(zi2); cz is
//         never -0, so neither is -0.  (n1 when Z2 = Z1 is never used.)
struct RayAxial {
    bool zsafe, exact;
};
__device__ __forceinline__ RayAxial ray_axial(const RayGeom &r, float z_half) {
    const float dc_lo = __fsub_rn(__fsub_rn(0.5f, r.d_half), r.src_d) - 1.0f;
    const float dc_hi = __fsub_rn(__fsub_rn((float)r.nd - 0.5f, r.d_half), r.src_d) + 1.0f;
    const float dmax = fmaxf(fabsf(dc_lo), fabsf(dc_hi));
    const float rmax = fmaxf(fabsf(r.rz0), fabsf(r.rz1));
    const float zmax = rmax * dmax + fabsf(z_half) + 1.0f;
    const float err = zmax * 0x1p-21f;  // >= 4 ulp of any cz, covers these bounds' rounding
    RayAxial a;
    a.zsafe = zmax + err < 0x1p19f;
    const bool one_sign = dc_lo > 0.0f || dc_hi < 0.0f;
    const float dmin = fminf(fabsf(dc_lo), fabsf(dc_hi));
    const float drz = fabsf(r.rz1 - r.rz0);
    const float dz_min = (drz * dmin - 2.0f * err) * (1.0f - 0x1p-20f);
    // the range of each cz over the ray, from its ends
    const float e0a = fmaf(r.rz0, dc_lo, z_half), e0b = fmaf(r.rz0, dc_hi, z_half);
    const float e1a = fmaf(r.rz1, dc_lo, z_half), e1b = fmaf(r.rz1, dc_hi, z_half);
    const float tiny = 0x1p-50f + err;
    const bool off0 = fminf(e0a, e0b) > tiny || fmaxf(e0a, e0b) < -tiny;
    const bool off1 = fminf(e1a, e1b) > tiny || fmaxf(e1a, e1b) < -tiny;
    a.exact = a.zsafe && one_sign && dz_min >= 0x1p-19f && off0 && off1;
    return a;
}

// The slabs d of a ray whose axial footprint can meet the volume: a superset
// of {d : max(cz0, cz1) >= 0 and min(cz0, cz1) < nz}, outside which the
// reference's axial loop over max(0, Z1) .. min(nz-1, Z2) is empty
// (:80-82 / :133-135) and the slab adds nothing.  Worked from the exact lines
// c_k(dc) = rz_k * dc + nz/2 of the ray's own (float) constants with a
// tolerance of 1/64 voxel, far above the difference of their float
// evaluation (a few ulp of values below 2^20); each condition's set of dc is
// a union of half-lines whose hull is taken, and the intersection of the
// hulls is mapped to slab indices with one slab of margin on either side.
// Returns lo > hi when no slab can contribute.
__device__ __forceinline__ void ray_zrange(const RayGeom &r, float z_half, int nz, int &lo,
                                           int &hi) {
    const double tol = 1.0 / 64.0, zh = z_half, rz[2] = {r.rz0, r.rz1};
    const double inf = 1e300;
    // hull of F1 = U_k {rz_k dc >= -tol - zh}: [lo1, hi1]
    double lo1 = inf, hi1 = -inf;
    // hull of F2 = U_k {rz_k dc < nz + tol - zh}: [lo2, hi2]
    double lo2 = inf, hi2 = -inf;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const double a = rz[k];
        const double t1 = (-tol - zh) / a, t2 = ((double)nz + tol - zh) / a;
        if (a > 0.0) {
            lo1 = fmin(lo1, t1); hi1 = inf;    // [t1, inf)
            lo2 = -inf; hi2 = fmax(hi2, t2);   // (-inf, t2)
        } else if (a < 0.0) {
            lo1 = -inf; hi1 = fmax(hi1, t1);   // (-inf, t1]
            lo2 = fmin(lo2, t2); hi2 = inf;    // (t2, inf)
        } else {  // constant zh: inside [0, nz)
            lo1 = -inf; hi1 = inf;
            lo2 = -inf; hi2 = inf;
        }
    }
    const double dlo = fmax(lo1, lo2), dhi = fmin(hi1, hi2);
    // slab d has dc = d + 0.5 - d_half - src_d (up to the rounding of
    // those floats)
    const double off = (double)r.d_half + (double)r.src_d - 0.5;
    const double a = fmax(dlo + off, -2.0), b = fmin(dhi + off, (double)r.nd + 1.0);
    if (!(a <= b)) {  // also NaN
        lo = 1;
        hi = 0;
        return;
    }
    lo = max(0, (int)floor(a) - 1);
    hi = min(r.nd - 1, (int)ceil(b) + 1);
}

// One slab of one ray, any footprint: the 2x2 window with predication or the
// reference's loops (:80-88 / :133-141).
template <int K, bool ONES, typename VT, bool CHECK, bool PAIR = false>
__device__ __forceinline__ void fp_slab(const RayGeom &r, const Geom &g, const SlabC &e, int d,
                                        const VT *const *base, int su, int sd, int sz,
                                        float z_half, bool zsafe, float *acc, float &accw) {
    SlabZ w;
    // (every load below is under its voxel's predicate)
    if (slab_window<CHECK, false>(r, g, e, sz, z_half, zsafe, w)) {
        // each volume's terms in the window's order (the volumes' sums are
        // independent, so visiting the voxels outermost keeps every order)
        float t[K];
        if (w.p00) {
            fp_voxel<K, PAIR>(base, w.a00, t);
#pragma unroll
            for (int k = 0; k < K; k++) acc[k] = __fmaf_rn(__fmul_rn(t[k], w.wu0), w.wz0, acc[k]);
        }
        if (w.p01) {
            fp_voxel<K, PAIR>(base, w.a01, t);
#pragma unroll
            for (int k = 0; k < K; k++) acc[k] = __fmaf_rn(__fmul_rn(t[k], w.wu0), w.wz1, acc[k]);
        }
        if (w.p10) {
            fp_voxel<K, PAIR>(base, w.a10, t);
#pragma unroll
            for (int k = 0; k < K; k++) acc[k] = __fmaf_rn(__fmul_rn(t[k], w.wu1), w.wz0, acc[k]);
        }
        if (w.p11) {
            fp_voxel<K, PAIR>(base, w.a11, t);
#pragma unroll
            for (int k = 0; k < K; k++) acc[k] = __fmaf_rn(__fmul_rn(t[k], w.wu1), w.wz1, acc[k]);
        }
        if (ONES) {
            if (w.p00) accw = __fmaf_rn(w.wu0, w.wz0, accw);
            if (w.p01) accw = __fmaf_rn(w.wu0, w.wz1, accw);
            if (w.p10) accw = __fmaf_rn(w.wu1, w.wz0, accw);
            if (w.p11) accw = __fmaf_rn(w.wu1, w.wz1, accw);
        }
        return;
    }
    const float cz0 = __fadd_rn(__fmul_rn(r.rz0, e.dc), z_half);
    const float cz1 = __fadd_rn(__fmul_rn(r.rz1, e.dc), z_half);
    const float zi1 = fminf(cz0, cz1), zi2 = fmaxf(cz0, cz1);
    const int Z1 = (int)floorf(zi1), Z2 = (int)floorf(zi2);
    const float dz = __fsub_rn(zi2, zi1);
    const int U1 = e.U1, U2 = e.U2;
    const bool fast_u = U2 - U1 <= 1;
    const int u_lo = max(0, U1), u_hi = min(r.nu - 1, U2);
    const int z_lo = max(0, Z1), z_hi = min(g.nz - 1, Z2);
    const float ui1 = e.a, ui2 = e.b;
    const float du = fast_u ? 0.0f : __fsub_rn(ui2, ui1);
    for (int u = u_lo; u <= u_hi; u++) {
        const float wu = fast_u ? (u == U1 ? e.a : e.b)
                                : __fdiv_rn(__fsub_rn(fminf(__fadd_rn((float)u, 1.0f), ui2),
                                                      fmaxf((float)u, ui1)), du);
        const int rowa = u * su + d * sd;
        for (int z = z_lo; z <= z_hi; z++) {
            const float wz = __fdiv_rn(__fsub_rn(fminf(__fadd_rn((float)z, 1.0f), zi2),
                                                 fmaxf((float)z, zi1)), dz);
            const int a = rowa + z * sz;
            float t[K];
            fp_voxel<K, PAIR>(base, a, t);
#pragma unroll
            for (int k = 0; k < K; k++) acc[k] = __fmaf_rn(__fmul_rn(t[k], wu), wz, acc[k]);
            if (ONES) accw = __fmaf_rn(wu, wz, accw);
        }
    }
}

// The windows of slabs d0+j .. d0+j+G-1 of a ray and the 4*K voxel
// values of each (addresses are clamped, so every load is in bounds and can
// be issued before the predicates are known; loading under the predicates
// from unclamped addresses measured 2-3 % slower at 256x256x160); true if
// all of them are exact 2x2 windows.
template <int K, int G, bool CHECK, typename VT, bool PAIR = false>
__device__ __forceinline__ bool fp_group_load(const RayGeom &r, const Geom &g,
                                              const SlabC (*sm_c)[FPC_COLS], int col, int j, int sz,
                                              const VT *const *base, float z_half, bool zsafe,
                                              SlabZ *w,
                                              float (*v)[K][4]) {
    bool all_fast = true;
#pragma unroll
    for (int q = 0; q < G; q++)
        all_fast &= slab_window<CHECK>(r, g, sm_c[j + q][col], sz, z_half, zsafe, w[q]);
#pragma unroll
    for (int q = 0; q < G; q++) {
        const int a[4] = {w[q].a00, w[q].a01, w[q].a10, w[q].a11};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            float t[K];
            fp_voxel<K, PAIR>(base, a[i], t);
#pragma unroll
            for (int k = 0; k < K; k++) v[q][k][i] = t[k];
        }
    }
    return all_fast;
}

// The terms of one group in the reference's order: from the loaded windows
// when all are 2x2 (fast), else slab by slab on the general path.
template <int K, int G, bool ONES, typename VT, bool CHECK, bool PAIR = false>
__device__ __forceinline__ void fp_group_sum(const RayGeom &r, const Geom &g,
                                             const SlabC (*sm_c)[FPC_COLS], int col, int j, int d0,
                                             const VT *const *base, int su, int sd, int sz,
                                             float z_half, bool zsafe, bool fast, const SlabZ *w,
                                             const float (*v)[K][4], float *acc, float &accw) {
    if (!fast) {
#pragma unroll 1
        for (int q = 0; q < G; q++)
            fp_slab<K, ONES, VT, CHECK, PAIR>(r, g, sm_c[j + q][col], d0 + j + q, base, su, sd, sz,
                                              z_half, zsafe, acc, accw);
        return;
    }
#pragma unroll
    for (int q = 0; q < G; q++) {
        const SlabZ &x = w[q];
        if (K == 1 && ONES) {
            // one volume and the weight sum: the two chains interleaved term
            // by term (measured faster here; the per-volume order below is
            // faster with three volumes)
            if (x.p00) {
                acc[0] = __fmaf_rn(__fmul_rn(v[q][0][0], x.wu0), x.wz0, acc[0]);
                accw = __fmaf_rn(x.wu0, x.wz0, accw);
            }
            if (x.p01) {
                acc[0] = __fmaf_rn(__fmul_rn(v[q][0][1], x.wu0), x.wz1, acc[0]);
                accw = __fmaf_rn(x.wu0, x.wz1, accw);
            }
            if (x.p10) {
                acc[0] = __fmaf_rn(__fmul_rn(v[q][0][2], x.wu1), x.wz0, acc[0]);
                accw = __fmaf_rn(x.wu1, x.wz0, accw);
            }
            if (x.p11) {
                acc[0] = __fmaf_rn(__fmul_rn(v[q][0][3], x.wu1), x.wz1, acc[0]);
                accw = __fmaf_rn(x.wu1, x.wz1, accw);
            }
            continue;
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            if (x.p00) acc[k] = __fmaf_rn(__fmul_rn(v[q][k][0], x.wu0), x.wz0, acc[k]);
            if (x.p01) acc[k] = __fmaf_rn(__fmul_rn(v[q][k][1], x.wu0), x.wz1, acc[k]);
            if (x.p10) acc[k] = __fmaf_rn(__fmul_rn(v[q][k][2], x.wu1), x.wz0, acc[k]);
            if (x.p11) acc[k] = __fmaf_rn(__fmul_rn(v[q][k][3], x.wu1), x.wz1, acc[k]);
        }
        if (ONES) {
            if (x.p00) accw = __fmaf_rn(x.wu0, x.wz0, accw);
            if (x.p01) accw = __fmaf_rn(x.wu0, x.wz1, accw);
            if (x.p10) accw = __fmaf_rn(x.wu1, x.wz0, accw);
            if (x.p11) accw = __fmaf_rn(x.wu1, x.wz1, accw);
        }
    }
}

// Slabs d0 + j0 .. d0 + jend - 1 of a ray from the shared table (j0 is the
// same for the whole warp).  Groups of G slabs: the windows and loads of a
// whole group are issued together before its terms enter the sums in the
// reference's order, so that a warp waits for memory once per group instead
// of per slab.  A group whose footprints are not all 2x2 windows takes the
// general per-slab path.
template <int K, int G, bool ONES, typename VT, bool CHECK, bool PAIR = false>
__device__ __forceinline__ void fp_chunk(const RayGeom &r, const Geom &g,
                                         const SlabC (*sm_c)[FPC_COLS], int col, int j0, int jend,
                                         int d0, const VT *const *base, int su, int sd, int sz,
                                         float z_half, bool zsafe, float *acc, float &accw) {
    int j = j0;
    for (; j + G <= jend; j += G) {
        SlabZ w[G];
        float v[G][K][4];
        const bool fast = fp_group_load<K, G, CHECK, VT, PAIR>(r, g, sm_c, col, j, sz, base,
                                                            z_half, zsafe, w, v);
        fp_group_sum<K, G, ONES, VT, CHECK, PAIR>(r, g, sm_c, col, j, d0, base, su, sd, sz,
                                               z_half, zsafe, fast, w, v, acc, accw);
    }
    for (; j < jend; j++)
        fp_slab<K, ONES, VT, CHECK, PAIR>(r, g, sm_c[j][col], d0 + j, base, su, sd, sz, z_half,
                                          zsafe, acc, accw);
}

// blockDim = FPC_THREADS: thread t is column t % FPC_COLS, row t / FPC_COLS;
// gridDim = (ceil(na/FPC_COLS), ceil(nb/FPC_ROWS), views).
// MULTI = true: several views per launch (ordered subsets, kernel-level
// multi-view projection), view = blockIdx.z with the per-view offsets of
// FPArgs; false: one view per launch without them.
// Row block i of n in dispatch order, from the middle of the detector
// outwards (m, m+1, m-1, m+2, ...): central rays cross the whole volume,
// outer ones fewer slabs (ray_zrange), so the longest blocks start first and
// the short ones fill the last wave.
__device__ __forceinline__ int middle_out(int i, int n) {
    const int m = (n - 1) / 2;
    return (i & 1) ? m + (i + 1) / 2 : m - i / 2;
}

// Whether a launch of bx x by projector blocks is resident at once with
// FPC_MIN_BLOCKS blocks per SM (so that the larger register budget of deeper
// slab groups costs no occupancy).
inline bool fp_one_wave(const mcsart_ctx *ctx, unsigned bx, unsigned by) {
    return ctx->sms > 0 && (int64_t)bx * by <= (int64_t)FPC_MIN_BLOCKS * ctx->sms;
}

// Resident blocks per SM the register budget must allow: one volume, 6 (at
// most 80 registers, which the kernel fits without spilling); three volumes,
// FPC_MIN_BLOCKS.  Large detectors fill every SM, and there the one-volume
// projector runs 6 blocks per SM instead of 5 (4.6 % less projector time at
// 512x384 rays per view; unchanged at 256x192, where fewer blocks exist).
// G = 4 slab groups keep more loads in flight and need the 128-register
// budget; the one-volume projector takes them when every block of the launch
// is resident at once (fp_one_wave), where the register budget costs no
// occupancy.
constexpr int FPC_MIN_BLOCKS_K1 = 6;
// MINB: resident blocks per SM the register budget must allow (the launch
// shape the driver's tuning may choose, with G; every choice gives the same
// bits).
// PAIR (three volumes): the second and third volumes interleaved in one
// array, vol.std[1] / vol.tr[1] (fp_voxel).
template <int K, bool ONES, typename VT, typename MT = VT, bool MULTI = false,
          int G = fp_group<K>(), int MINB = (K == 1 && G == 2) ? FPC_MIN_BLOCKS_K1 : FPC_MIN_BLOCKS,
          bool PAIR = false>
__global__ void __launch_bounds__(FPC_THREADS, MINB) fp_ref_kernel(const FPArgs<VT, K, MT> p) {
    __shared__ SlabC sm_c[FPC_CHUNK][FPC_COLS];
    __shared__ double2 sm_norm[FPC_THREADS / 32];
    __shared__ int sm_wr[FPC_THREADS / 32][2];  // each warp's slab range
    __shared__ int sm_ur[2];                    // the chunk's in-plane slab range
    const Geom &g = p.g;
    const int t = threadIdx.x, col = t % FPC_COLS, row = t / FPC_COLS;
    const int by = middle_out(blockIdx.y, gridDim.y);  // this block's row block
    const int ia = blockIdx.x * FPC_COLS + col, ib = by * FPC_ROWS + row;
    const bool col_ok = ia < g.na;
    const bool active = col_ok && ib < g.nb;
    const float angle = p.angles ? p.angles[blockIdx.z] : p.angle;
    const float cphi = cosf(angle), sphi = sinf(angle);  // :23-24
    // rows past the detector still compute their column's in-plane part
    const RayGeom r = ray_geom(cphi, sphi, col_ok ? ia : 0, min(ib, g.nb - 1), g);

    const VT *base[K];
    int su, sd;
    const int sz = g.nx * g.ny;
    const int64_t voff = MULTI ? (int64_t)blockIdx.z * p.vol_stride : 0;
    if (r.xdrive) {
        if (p.vol.tr[0] != nullptr) {
#pragma unroll
            for (int k = 0; k < K; k++) base[k] = p.vol.tr[k] + voff;
            su = 1; sd = g.ny;
        } else {
#pragma unroll
            for (int k = 0; k < K; k++) base[k] = p.vol.std[k] + voff;
            su = g.nx; sd = 1;
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; k++) base[k] = p.vol.std[k] + voff;
        su = 1; sd = g.nx;
    }
    const float z_half = (float)(g.nz / 2);
    float acc[K], accw = 0.0f;
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = 0.0f;

    // warps whose rays all have proven division operands skip the per-slab
    // range checks (warp-uniform, so neither form diverges)
    const RayAxial ax = ray_axial(r, z_half);
    const bool warp_exact = __all_sync(0xffffffffu, !active || ax.exact);
    // Slabs that can add to some ray of the warp: the union of the rays'
    // axial ranges (ray_zrange); the block visits the union of its warps'.
    // Outside them, and outside the slabs where some column of the block
    // meets the volume in-plane (SC_UANY), the reference's loops are empty.
    int zlo = 1, zhi = 0;
    if (active) ray_zrange(r, z_half, g.nz, zlo, zhi);
    if (zlo > zhi) {
        zlo = INT_MAX;
        zhi = INT_MIN;
    }
    const int wlo = __reduce_min_sync(0xffffffffu, zlo), whi = __reduce_max_sync(0xffffffffu, zhi);
    if ((t & 31) == 0) {
        sm_wr[t >> 5][0] = wlo;
        sm_wr[t >> 5][1] = whi;
    }
    __syncthreads();
    int blo = INT_MAX, bhi = INT_MIN;
#pragma unroll
    for (int w = 0; w < FPC_THREADS / 32; w++) {
        blo = min(blo, sm_wr[w][0]);
        bhi = max(bhi, sm_wr[w][1]);
    }
    const int first = blo <= bhi ? blo - blo % FPC_CHUNK : 0;
    for (int d0 = first; d0 <= bhi; d0 += FPC_CHUNK) {
        for (int j = row; j < FPC_CHUNK; j += FPC_ROWS) {
            const int d = d0 + j;
            SlabC e;
            e.r0 = 0; e.r1 = 0; e.a = 0.0f; e.b = 0.0f; e.dc = 0.0f;
            e.U1 = 0; e.U2 = -1; e.flags = 0;
            if (col_ok && d < r.nd) e = slab_c(r, d, su, sd);
            sm_c[j][col] = e;
        }
        __syncthreads();
        if (t < 32) {  // the chunk's slabs where some column meets the volume in-plane
            unsigned m[FPC_CHUNK / 32];
#pragma unroll
            for (int h = 0; h < FPC_CHUNK / 32; h++) {
                bool any = false;
#pragma unroll
                for (int c = 0; c < FPC_COLS; c++) any |= (sm_c[h * 32 + t][c].flags & SC_UANY) != 0;
                m[h] = __ballot_sync(0xffffffffu, any);
            }
            if (t == 0) {
                int lo = FPC_CHUNK, hi = -1;
#pragma unroll
                for (int h = FPC_CHUNK / 32 - 1; h >= 0; h--)
                    if (m[h]) lo = h * 32 + __ffs(m[h]) - 1;
#pragma unroll
                for (int h = 0; h < FPC_CHUNK / 32; h++)
                    if (m[h]) hi = h * 32 + 31 - __clz(m[h]);
                sm_ur[0] = lo;
                sm_ur[1] = hi;
            }
        }
        __syncthreads();
        // (an empty warp range is wlo = INT_MAX > whi = INT_MIN)
        const int j0 = wlo <= whi ? max(sm_ur[0], wlo - d0) : 0;
        const int jend = (active && wlo <= whi) ? min(min(sm_ur[1], whi - d0) + 1, r.nd - d0) : 0;
        if (warp_exact)
            fp_chunk<K, G, ONES, VT, false, PAIR>(r, g, sm_c, col, max(j0, 0), jend, d0, base, su,
                                               sd, sz, z_half, ax.zsafe, acc, accw);
        else
            fp_chunk<K, G, ONES, VT, true, PAIR>(r, g, sm_c, col, max(j0, 0), jend, d0, base, su,
                                              sd, sz, z_half, ax.zsafe, acc, accw);
        __syncthreads();
    }

    if (p.bpcolA != nullptr) {
        // the following backprojector's per-column part, with its own sine
        // and cosine of the angle (src/cu_backprojection.cu:62-63): the same
        // device code, so the same bits as computing it there; spread over
        // all threads of the view's blocks
        const float bs = __sinf(angle), bc = __cosf(angle);
        const int64_t ncol = (int64_t)g.nx * g.ny;
        const int64_t coff = MULTI ? (int64_t)blockIdx.z * ncol : 0;
        const int64_t nthr = (int64_t)gridDim.x * gridDim.y * FPC_THREADS;
        for (int64_t c = ((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * FPC_THREADS + t; c < ncol;
             c += nthr) {
            const BPColumn col = bp_column<false>((int)(c % g.nx), (int)(c / g.nx), bc, bs, g);
            p.bpcolA[coff + c] = make_float4(col.amin, col.amax, col.rl, col.rr);
            p.bpcolB[coff + c] = col.r0;
        }
    }

    const int64_t pix = ia + (int64_t)ib * g.na;
    const int64_t vpix = MULTI ? pix + (int64_t)blockIdx.z * g.na * g.nb : pix;  // this view's cell
    double nb2 = 0.0, nr2 = 0.0;
    if (active) {
        if (p.mode == FP_PLAIN) {
            p.out[vpix] = acc[0];
        } else {
            const float b = ldv(p.meas, vpix);
            // AUMISART.cu:206 host_add(proj, proj_temp, -1): proj += proj_temp * -1
            float res = __fmaf_rn(acc[0], -1.0f, b);
            float ones = ONES ? accw : 0.0f;
            if (p.mode == FP_MOTION) {
                res = __fmaf_rn(acc[K > 1 ? 1 : 0], 1.0f, res);  // AUMISART.cu:260, + FP(img0)
                if (K >= 3) ones = acc[K - 1];                   // FP(initial2(...)), :267-268
            }
            if (p.resid) p.resid[vpix] = res;
            // the backprojector's operands as the reference's texture reads
            // them; resid and the norms keep the residual itself
            p.bp_in[vpix] = make_float2(tex_texel(res), tex_texel(ones));
            nb2 = (double)b * (double)b;
            nr2 = (double)res * (double)res;
        }
    }
    if (p.mode == FP_PLAIN) return;
    // block partial of the two squared norms, fixed-order reduction
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        nb2 += __shfl_down_sync(0xffffffffu, nb2, off);
        nr2 += __shfl_down_sync(0xffffffffu, nr2, off);
    }
    if ((t & 31) == 0) sm_norm[t >> 5] = make_double2(nb2, nr2);
    __syncthreads();
    if (t == 0) {
        double tb = 0.0, tr = 0.0;
        for (int w = 0; w < FPC_THREADS / 32; w++) {
            tb += sm_norm[w].x;
            tr += sm_norm[w].y;
        }
        const int64_t vblk = MULTI ? (int64_t)blockIdx.z * gridDim.x * gridDim.y : 0;
        p.norm_part[vblk + by * gridDim.x + blockIdx.x] = make_double2(tb, tr);
    }
}

// Per-ray projector, used for the split summation modes (the engine launches
// fp_ref_kernel for SUM_REF).
// Launch shapes.  SUM_REF: blockDim (32, 8), one ray per thread, 32 columns x
// 8 rows per block, gridDim (ceil(na/32), ceil(nb/8), views).  Split modes:
// blockDim (32, groups), threadIdx.y = slab group of the same 32 rays,
// gridDim (ceil(na/32), nb, views).
// GEO64: FP64 geometry and weight sum (ray_geom64 / ray_slabs64); split
// summation modes only.
template <int K, bool ONES, int SUM, typename VT, typename MT = VT, bool GEO64 = false>
__global__ void __launch_bounds__(256) fp_kernel(const FPArgs<VT, K, MT> p) {
    static_assert(!GEO64 || SUM != SUM_REF, "FP64 geometry needs a split summation mode");
    constexpr int NS = K + (ONES ? 1 : 0);
    extern __shared__ float sm_fp[];  // split modes: [groups][NS][32]
    __shared__ double2 sm_norm[8];
    __shared__ double sm_w64[GEO64 ? 8 : 1][32];  // GEO64: the groups' FP64 weight sums
    const int lane = threadIdx.x;
    const Geom &g = p.g;
    const int ia = blockIdx.x * 32 + lane;
    const int ib = (SUM == SUM_REF) ? blockIdx.y * 8 + threadIdx.y : blockIdx.y;
    const bool active = ia < g.na && ib < g.nb;
    float s[K], sw = 0.0f;
    double sw64 = 0.0;
#pragma unroll
    for (int k = 0; k < K; k++) s[k] = 0.0f;
    if (active) {
        const float angle = p.angles ? p.angles[blockIdx.z] : p.angle;
        if (GEO64) {
            double sd, cd;
            sincos((double)angle, &sd, &cd);
            const RayGeom64 r = ray_geom64(cd, sd, ia, ib, g);
            const int groups = blockDim.y, grp = threadIdx.y;
            const int per = (r.nd + groups - 1) / groups;
            const int d0 = grp * per, d1 = min(r.nd, d0 + per);
            ray_slabs64<K, ONES, SUM, VT>(r, p.vol, g, d0, d1, s, sw64);
        } else {
            const float cphi = cosf(angle), sphi = sinf(angle);  // :23-24
            const RayGeom r = ray_geom(cphi, sphi, ia, ib, g);
            if (SUM == SUM_REF) {
                ray_slabs<K, ONES, SUM, VT>(r, p.vol, g, 0, r.nd, s, sw);
            } else {
                const int groups = blockDim.y, grp = threadIdx.y;
                const int per = (r.nd + groups - 1) / groups;
                const int d0 = grp * per, d1 = min(r.nd, d0 + per);
                ray_slabs<K, ONES, SUM, VT>(r, p.vol, g, d0, d1, s, sw);
            }
        }
    }
    if (SUM != SUM_REF) {
        const int grp = threadIdx.y, groups = blockDim.y;
#pragma unroll
        for (int k = 0; k < K; k++) sm_fp[(grp * NS + k) * 32 + lane] = s[k];
        if (ONES) sm_fp[(grp * NS + K) * 32 + lane] = sw;
        if (GEO64) sm_w64[grp][lane] = sw64;
        __syncthreads();
        if (grp != 0) return;
        // fixed-order combination of the slab groups
        for (int q = 1; q < groups; q++) {
#pragma unroll
            for (int k = 0; k < K; k++) s[k] += sm_fp[(q * NS + k) * 32 + lane];
            if (ONES) sw += sm_fp[(q * NS + K) * 32 + lane];
            if (GEO64) sw64 += sm_w64[q][lane];
        }
        if (GEO64) sw = (float)sw64;
    }
    const int64_t pix = ia + (int64_t)ib * g.na;
    double nb2 = 0.0, nr2 = 0.0;
    if (active) {
        if (p.mode == FP_PLAIN) {
            p.out[pix + (int64_t)blockIdx.z * g.na * g.nb] = s[0];
        } else {
            const float b = ldv(p.meas, pix);
            // AUMISART.cu:206 host_add(proj, proj_temp, -1): proj += proj_temp * -1
            float res = __fmaf_rn(s[0], -1.0f, b);
            float ones = ONES ? sw : 0.0f;
            if (p.mode == FP_MOTION) {
                res = __fmaf_rn(s[1], 1.0f, res);  // AUMISART.cu:260, + FP(img0)
                if (K >= 3) ones = s[2];            // FP(initial2(...)), :267-268
            }
            if (p.resid) p.resid[pix] = res;
            p.bp_in[pix] = make_float2(tex_texel(res), tex_texel(ones));
            nb2 = (double)b * (double)b;
            nr2 = (double)res * (double)res;
        }
    }
    if (p.mode == FP_PLAIN) return;
    // block partial of the two squared norms, fixed-order reduction
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        nb2 += __shfl_down_sync(0xffffffffu, nb2, off);
        nr2 += __shfl_down_sync(0xffffffffu, nr2, off);
    }
    if (SUM != SUM_REF) {  // only warp 0 is left
        if (lane == 0) p.norm_part[blockIdx.y * gridDim.x + blockIdx.x] = make_double2(nb2, nr2);
        return;
    }
    if (lane == 0) sm_norm[threadIdx.y] = make_double2(nb2, nr2);
    __syncthreads();
    if (threadIdx.y == 0 && lane == 0) {
        double tb = 0.0, tr = 0.0;
        for (int w = 0; w < (int)blockDim.y; w++) {
            tb += sm_norm[w].x;
            tr += sm_norm[w].y;
        }
        p.norm_part[blockIdx.y * gridDim.x + blockIdx.x] = make_double2(tb, tr);
    }
}

}  // namespace mcsart
