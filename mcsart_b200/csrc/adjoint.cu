// mcsart_backprojection_adjoint: the exact adjoint (transpose) of the engine's
// distance-driven projector (mcsart_projection, the reference's
// kernel_projection, src/cu_projection.cu:7-145).  The reference's own
// backprojector (src/cu_backprojection.cu) is a different operator: it maps
// voxel boundaries onto the detector, while the projector maps detector cell
// boundaries onto slab planes.  A matched pair makes SART's update a true
// gradient step and lets dot-product tests hold.
//
// Deterministic gather, no floating-point atomics.  Per view:
//  1. every ray's geometry (ray_geom): the column's in-plane part and the
//     ray's axial ratios rz0, rz1;
//  2. every column's in-plane footprint per slab (slab_u) and, for each
//     (driving axis, slab, in-plane voxel), the range of columns whose
//     footprint covers it (integer min / max atomics, order-independent);
//  3. per voxel: for the covering columns and the rows whose axial footprint
//     can reach the voxel (the footprint centre is linear in the row), the
//     projector's own weights w_u, w_z, recomputed with the same operations,
//     and acc = fma(p * w_u, w_z, acc) in a fixed order (x-driven columns,
//     then y-driven; columns, then rows, ascending).
#include <climits>

#include "common.cuh"
#include "projector.cuh"

#define MC_EXPORT extern "C" __attribute__((visibility("default")))

namespace mcsart {

static __global__ void adj_rays_kernel(RayGeom *cols, float2 *rz, float angle, Geom g) {
    const int ia = blockIdx.x * blockDim.x + threadIdx.x, ib = blockIdx.y;
    if (ia >= g.na) return;
    const float cphi = cosf(angle), sphi = sinf(angle);  // as the projector
    const RayGeom r = ray_geom(cphi, sphi, ia, ib, g);
    rz[ia + (int64_t)ib * g.na] = make_float2(r.rz0, r.rz1);
    if (ib == 0) cols[ia] = r;
}

static __global__ void adj_range_init_kernel(int2 *range, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        range[i] = make_int2(INT_MAX, -1);
}

// range[(axis * nmax + d) * nmax + u] = (first, last) column covering in-plane
// voxel u of slab d, axis 1 = x-driven columns.
static __global__ void adj_slabs_kernel(const RayGeom *cols, SlabU *slabs, int2 *range, Geom g,
                                        int nmax) {
    const int ia = blockIdx.x * blockDim.x + threadIdx.x, d = blockIdx.y;
    if (ia >= g.na) return;
    const RayGeom r = cols[ia];
    if (d >= r.nd) return;
    const SlabU e = slab_u(r, d);
    slabs[(int64_t)ia * nmax + d] = e;
    const int axis = r.xdrive ? 1 : 0;
    const int u0 = max(0, e.U1), u1 = min(r.nu - 1, e.U2);
    for (int u = u0; u <= u1; u++) {
        int2 *c = range + ((int64_t)axis * nmax + d) * nmax + u;
        atomicMin(&c->x, ia);
        atomicMax(&c->y, ia);
    }
}

// blockDim (32, 8): one voxel per thread, x fastest.
static __global__ void __launch_bounds__(256) adj_gather_kernel(
    float *img, const float *proj, const RayGeom *cols, const float2 *rz, const SlabU *slabs,
    const int2 *range, Geom g, int nmax) {
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y,
              z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    const float z_half = (float)(g.nz / 2), fz = (float)z;
    const int na = g.na, nb = g.nb;
    float acc = 0.0f;
    for (int axis = 1; axis >= 0; axis--) {
        const int d = axis ? x : y, u = axis ? y : x;
        const int2 cr = range[((int64_t)axis * nmax + d) * nmax + u];
        for (int ia = cr.x; ia <= cr.y; ia++) {
            const RayGeom r = cols[ia];
            if ((r.xdrive ? 1 : 0) != axis || d >= r.nd) continue;
            const SlabU e = slabs[(int64_t)ia * nmax + d];
            if (u < max(0, e.U1) || u > min(r.nu - 1, e.U2)) continue;
            // the projector's in-plane weight of voxel u (slab_u, fp_slab)
            float wu;
            if (e.U2 - e.U1 <= 1) {
                wu = u == e.U1 ? e.a : e.b;
            } else {
                const float ui1 = e.a, ui2 = e.b;
                wu = __fdiv_rn(__fsub_rn(fminf(__fadd_rn((float)u, 1.0f), ui2), fmaxf((float)u, ui1)),
                               __fsub_rn(ui2, ui1));
            }
            const float dc = __fsub_rn(__fsub_rn(__fadd_rn((float)d, 0.5f), r.d_half), r.src_d);
            // rows whose axial footprint can reach z: its centre is linear in
            // the row; the bound is widened by two rows and every candidate is
            // tested exactly below
            int ib_lo = 0, ib_hi = nb - 1;
            if (nb > 1) {
                const float2 q0 = rz[ia], q1 = rz[ia + (int64_t)(nb - 1) * na];
                const float c0 = 0.5f * (q0.x + q0.y) * dc + z_half;
                const float c1 = 0.5f * (q1.x + q1.y) * dc + z_half;
                const float s = (c1 - c0) / (float)(nb - 1);
                const float h = 0.5f * fabsf((q0.y - q0.x) * dc) + 0.5f;
                if (fabsf(s) > 1e-6f) {
                    const float ta = (fz + 0.5f - h - c0) / s, tb = (fz + 0.5f + h - c0) / s;
                    const float lo = fminf(ta, tb) - 2.0f, hi = fmaxf(ta, tb) + 2.0f;
                    if (hi < 0.0f || lo > (float)(nb - 1)) continue;
                    ib_lo = max(0, (int)floorf(fmaxf(lo, 0.0f)));
                    ib_hi = min(nb - 1, (int)ceilf(fminf(hi, (float)(nb - 1))));
                }
            }
            for (int ib = ib_lo; ib <= ib_hi; ib++) {
                const float2 q = rz[ia + (int64_t)ib * na];
                // the projector's axial footprint (slab_window, fp_slab)
                const float cz0 = __fadd_rn(__fmul_rn(q.x, dc), z_half);
                const float cz1 = __fadd_rn(__fmul_rn(q.y, dc), z_half);
                const float zi1 = fminf(cz0, cz1), zi2 = fmaxf(cz0, cz1);
                const int Z1 = (int)floorf(zi1), Z2 = (int)floorf(zi2);
                if (z < max(0, Z1) || z > min(g.nz - 1, Z2)) continue;
                const float wz = __fdiv_rn(__fsub_rn(fminf(__fadd_rn(fz, 1.0f), zi2), fmaxf(fz, zi1)),
                                           __fsub_rn(zi2, zi1));
                acc = __fmaf_rn(__fmul_rn(__ldg(proj + ia + (int64_t)ib * na), wu), wz, acc);
            }
        }
    }
    img[x + (int64_t)y * g.nx + (int64_t)z * g.nx * g.ny] = acc;
}

}  // namespace mcsart

using namespace mcsart;

MC_EXPORT int mcsart_backprojection_adjoint(mcsart_ctx *ctx, float *d_img, const float *d_proj,
                                            float angle, float SO, float SD, float da, int na,
                                            float ai, float db, int nb, float bi, int nx, int ny,
                                            int nz) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(d_proj && d_img, "d_proj and d_img must be non-NULL");
    Geom g;
    g.SO = SO; g.SD = SD; g.da = da; g.ai = ai; g.db = db; g.bi = bi;
    g.na = na; g.nb = nb; g.nx = nx; g.ny = ny; g.nz = nz;
    MC_TRY(validate_geom(g));
    const int nmax = std::max(nx, ny);
    void *w_cols, *w_rz, *w_slabs, *w_range;
    MC_TRY(workspace(ctx, "adj_cols", (size_t)na * sizeof(RayGeom), &w_cols));
    MC_TRY(workspace(ctx, "adj_rz", (size_t)na * nb * sizeof(float2), &w_rz));
    MC_TRY(workspace(ctx, "adj_slabs", (size_t)na * nmax * sizeof(SlabU), &w_slabs));
    const int64_t n_range = 2LL * nmax * nmax;
    MC_TRY(workspace(ctx, "adj_range", (size_t)n_range * sizeof(int2), &w_range));
    RayGeom *cols = (RayGeom *)w_cols;
    float2 *rz = (float2 *)w_rz;
    SlabU *slabs = (SlabU *)w_slabs;
    int2 *range = (int2 *)w_range;
    MC_LAUNCH(ctx, adj_rays_kernel, dim3(div_up(na, 128), nb), 128, 0, cols, rz, angle, g);
    MC_LAUNCH(ctx, adj_range_init_kernel, (unsigned)std::min<int64_t>(div_up(n_range, 256), 4096),
              256, 0, range, n_range);
    MC_LAUNCH(ctx, adj_slabs_kernel, dim3(div_up(na, 128), nmax), 128, 0, cols, slabs, range, g,
              nmax);
    MC_LAUNCH(ctx, adj_gather_kernel, dim3(div_up(nx, 32), div_up(ny, 8), nz), dim3(32, 8), 0,
              d_img, d_proj, cols, rz, slabs, range, g, nmax);
    return finish(ctx, "mcsart_backprojection_adjoint");
}
