// Kernel-level C ABI: one entry point per reference launcher (include/mcsart.h).
#include <algorithm>

#include "backprojector.cuh"
#include "common.cuh"
#include "elementwise.cuh"
#include "projector.cuh"
#include "sart.cuh"
#include "warp.cuh"

#define MC_EXPORT extern "C" __attribute__((visibility("default")))

namespace mcsart {

// Slab groups per ray: enough warps for ~4 waves of 48 warps on 148 SMs,
// at least 8 slabs per group, at most 8 groups.
int fp_auto_groups(int64_t ray_blocks, int n_slabs) {
    const int64_t target = 148LL * 48 * 2;
    int s = 1;
    while (s < 8 && ray_blocks * s < target && n_slabs / (2 * s) >= 8) s *= 2;
    return s;
}

// True if any ray of the view is x-driven (|x21| > |y21|, cu_projection.cu:39),
// evaluated with the float arithmetic of the kernel's ray setup.
bool view_has_xdrive(float angle, const Geom &g) {
    const float cphi = cosf(angle), sphi = sinf(angle);
    const float x1 = -g.SO * cphi, y1 = -g.SO * sphi;
    const float x20 = g.SD - g.SO;
    for (int ia = 0; ia < g.na; ia++) {
        const float y20 = (ia + g.ai) * g.da;
        const float x21 = (x20 * cphi - y20 * sphi) - x1;
        const float y21 = (x20 * sphi + y20 * cphi) - y1;
        // host and device cos/sin may differ in the last bit: be conservative
        if (fabsf(x21) >= 0.999f * fabsf(y21)) return true;
    }
    return false;
}

// Which volume copies a view's projector reads: x-driven rays read the
// y-fastest copy, y-driven rays the x-fastest one.  Evaluated with the float
// arithmetic of the kernel's ray set-up and a margin for the last bit of the
// host's and the device's sine and cosine, so a column near the switch
// counts for both.
void view_drive_axes(float angle, const Geom &g, bool *any_x, bool *any_y) {
    const float cphi = cosf(angle), sphi = sinf(angle);
    const float x1 = -g.SO * cphi, y1 = -g.SO * sphi;
    const float x20 = g.SD - g.SO;
    *any_x = *any_y = false;
    for (int ia = 0; ia < g.na; ia++) {
        const float y20 = (ia + g.ai) * g.da;
        const float x21 = (x20 * cphi - y20 * sphi) - x1;
        const float y21 = (x20 * sphi + y20 * cphi) - y1;
        if (fabsf(x21) >= 0.999f * fabsf(y21)) *any_x = true;
        if (fabsf(y21) >= 0.999f * fabsf(x21)) *any_y = true;
    }
}

template <int K>
int launch_fp_plain(mcsart_ctx *ctx, float *d_proj, const float *d_img, const float *d_imgT,
                    float angle, const float *d_angles, int n_views, const Geom &g) {
    FPArgs<float, K> a{};
    a.vol.std[0] = d_img;
    a.vol.tr[0] = d_imgT;
    a.g = g;
    a.angle = angle;
    a.angles = d_angles;
    a.mode = FP_PLAIN;
    a.out = d_proj;
    // the reference's summation order: bitwise the reference kernel's output
    const dim3 grid(div_up(g.na, FPC_COLS), div_up(g.nb, FPC_ROWS), n_views);
    // several views (mcsart_projection_views): the multi-view instantiation
    if (n_views > 1)
        MC_LAUNCH(ctx, (fp_ref_kernel<K, false, float, float, true>), grid, dim3(FPC_THREADS), 0, a);
    else
        MC_LAUNCH(ctx, (fp_ref_kernel<K, false, float>), grid, dim3(FPC_THREADS), 0, a);
    return MCSART_OK;
}

int transpose_f32(mcsart_ctx *ctx, float *dstT, const float *src, int nx, int ny, int nz) {
    const dim3 grid(div_up(nx, 32), div_up(ny, 32), nz), block(32, 8);
    MC_LAUNCH(ctx, (transpose_kernel<float, float>), grid, block, 0, dstT, src, nx, ny);
    return MCSART_OK;
}

unsigned stream_blocks(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return (unsigned)std::min<int64_t>(b, 148LL * 16);
}

}  // namespace mcsart

using namespace mcsart;

static Geom make_geom(float SO, float SD, float da, int na, float ai, float db, int nb, float bi,
                      int nx, int ny, int nz) {
    Geom g;
    g.SO = SO; g.SD = SD; g.da = da; g.ai = ai; g.db = db; g.bi = bi;
    g.na = na; g.nb = nb; g.nx = nx; g.ny = ny; g.nz = nz;
    return g;
}

MC_EXPORT int mcsart_projection(mcsart_ctx *ctx, float *d_proj, const float *d_img, float angle,
                                float SO, float SD, float da, int na, float ai, float db, int nb,
                                float bi, int nx, int ny, int nz) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(d_proj && d_img, "d_proj and d_img must be non-NULL");
    const Geom g = make_geom(SO, SD, da, na, ai, db, nb, bi, nx, ny, nz);
    MC_TRY(validate_geom(g));
    const float *imgT = nullptr;
    if (view_has_xdrive(angle, g)) {
        void *ws;
        MC_TRY(workspace(ctx, "fp_volT", nvox(nx, ny, nz) * sizeof(float), &ws));
        MC_TRY(transpose_f32(ctx, (float *)ws, d_img, nx, ny, nz));
        imgT = (const float *)ws;
    }
    MC_TRY(launch_fp_plain<1>(ctx, d_proj, d_img, imgT, angle, nullptr, 1, g));
    return finish(ctx, "mcsart_projection");
}

MC_EXPORT int mcsart_projection_views(mcsart_ctx *ctx, float *d_proj, const float *d_img,
                                      const float *h_angles, int n_views, float SO, float SD,
                                      float da, int na, float ai, float db, int nb, float bi,
                                      int nx, int ny, int nz) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(d_proj && d_img && h_angles, "d_proj, d_img and h_angles must be non-NULL");
    MC_REQUIRE(n_views > 0 && n_views <= 65535, "n_views must be in [1, 65535]");
    const Geom g = make_geom(SO, SD, da, na, ai, db, nb, bi, nx, ny, nz);
    MC_TRY(validate_geom(g));
    void *wsT, *wsA;
    MC_TRY(workspace(ctx, "fp_volT", nvox(nx, ny, nz) * sizeof(float), &wsT));
    MC_TRY(workspace(ctx, "fp_angles", (size_t)n_views * sizeof(float), &wsA));
    MC_CHECK_CUDA(cudaMemcpyAsync(wsA, h_angles, (size_t)n_views * sizeof(float),
                                  cudaMemcpyHostToDevice, ctx->stream));
    MC_TRY(transpose_f32(ctx, (float *)wsT, d_img, nx, ny, nz));
    MC_TRY(launch_fp_plain<1>(ctx, d_proj, d_img, (const float *)wsT, 0.0f, (const float *)wsA,
                              n_views, g));
    // the angle staging buffer must outlive the launch before the host array is reused
    MC_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    return finish(ctx, "mcsart_projection_views");
}

MC_EXPORT int mcsart_backprojection(mcsart_ctx *ctx, float *d_img, const float *d_proj,
                                    float angle, float SO, float SD, float da, int na, float ai,
                                    float db, int nb, float bi, int nx, int ny, int nz) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(d_proj && d_img, "d_proj and d_img must be non-NULL");
    const Geom g = make_geom(SO, SD, da, na, ai, db, nb, bi, nx, ny, nz);
    MC_TRY(validate_geom(g));
    BPArgs a{};
    a.proj = d_proj;
    a.g = g;
    a.angle = angle;
    a.out = d_img;
    const dim3 grid(div_up(nx, 32), div_up(ny, BP_ROWS), div_up(nz, BP_NZ)), block(32, BP_ROWS);
    if (bp_geom_proven(g))
        MC_LAUNCH(ctx, (bp_kernel<1, BP_PLAIN, false, true>), grid, block, 0, a);
    else
        MC_LAUNCH(ctx, (bp_kernel<1, BP_PLAIN>), grid, block, 0, a);
    return finish(ctx, "mcsart_backprojection");
}

static int deform_common(mcsart_ctx *ctx, bool first_order, float *d_img1, const float *d_img,
                         int nx, int ny, int nz, float volume, float flow, const float *ax,
                         const float *ay, const float *az, const float *bx, const float *by,
                         const float *bz) {
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(d_img1 && d_img && ax && ay && az && bx && by && bz,
               "volume and field pointers must be non-NULL");
    const int64_t n = nvox(nx, ny, nz);
    const Fields<float> f{ax, ay, az, bx, by, bz};
    const unsigned blocks = stream_blocks(n);
    if (!first_order && ctx->interp == MCSART_INTERP_TEXTURE) {
        // the reference samples a texture over a copy of the input
        // (cu_deform.cu:13-38); here the 3D array persists across calls
        if (!ctx->driver) ctx->driver.reset(new DriverState());
        TexVol &tv = ctx->driver->tv_deform;
        MC_TRY(tv.ensure(nx, ny, nz));
        MC_TRY(tv.upload(d_img, ctx->stream));
        MC_LAUNCH(ctx, deform_kernel<SrcTex>, blocks, 256, 0, d_img1, SrcTex{tv.tex}, f, nx, ny,
                  nz, volume, flow);
        return MCSART_OK;
    }
    const float *src = d_img;
    if (d_img1 == d_img) {  // the reference samples a copy (cu_deform.cu:13-23)
        void *ws;
        MC_TRY(workspace(ctx, "deform_src", n * sizeof(float), &ws));
        MC_CHECK_CUDA(cudaMemcpyAsync(ws, d_img, n * sizeof(float), cudaMemcpyDeviceToDevice,
                                      ctx->stream));
        src = (const float *)ws;
    }
    if (first_order) {
        MC_LAUNCH(ctx, deform2_kernel, blocks, 256, 0, d_img1, src, f, nx, ny, nz, volume, flow);
    } else {
        MC_LAUNCH(ctx, deform_kernel<SrcLinear<float>>, blocks, 256, 0, d_img1,
                  SrcLinear<float>{src}, f, nx, ny, nz, volume, flow);
    }
    return MCSART_OK;
}

MC_EXPORT int mcsart_deform(mcsart_ctx *ctx, float *d_img1, const float *d_img, int nx, int ny,
                            int nz, float volume, float flow, const float *ax, const float *ay,
                            const float *az, const float *bx, const float *by, const float *bz) {
    clear_error();
    MC_TRY(deform_common(ctx, false, d_img1, d_img, nx, ny, nz, volume, flow, ax, ay, az, bx, by,
                         bz));
    return finish(ctx, "mcsart_deform");
}

MC_EXPORT int mcsart_deform2(mcsart_ctx *ctx, float *d_img1, const float *d_img, int nx, int ny,
                             int nz, float volume, float flow, const float *ax, const float *ay,
                             const float *az, const float *bx, const float *by, const float *bz) {
    clear_error();
    MC_TRY(deform_common(ctx, true, d_img1, d_img, nx, ny, nz, volume, flow, ax, ay, az, bx, by,
                         bz));
    return finish(ctx, "mcsart_deform2");
}

MC_EXPORT int mcsart_forward_dvf(mcsart_ctx *ctx, float *mx, float *my, float *mz,
                                 const float *ax, const float *ay, const float *az,
                                 const float *bx, const float *by, const float *bz, float volume,
                                 float flow, int nx, int ny, int nz) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(mx && my && mz && ax && ay && az && bx && by && bz, "pointers must be non-NULL");
    const int64_t n = nvox(nx, ny, nz);
    const Fields<float> f{ax, ay, az, bx, by, bz};
    MC_LAUNCH(ctx, forward_dvf_kernel, stream_blocks(n), 256, 0, mx, my, mz, f, n, volume, flow);
    return finish(ctx, "mcsart_forward_dvf");
}

MC_EXPORT int mcsart_invert_dvf(mcsart_ctx *ctx, float *inv_x, float *inv_y, float *inv_z,
                                const float *ax, const float *ay, const float *az,
                                const float *bx, const float *by, const float *bz, float volume,
                                float flow, int nx, int ny, int nz, int n_iter) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(inv_x && inv_y && inv_z && ax && ay && az && bx && by && bz,
               "pointers must be non-NULL");
    MC_REQUIRE(nx == ny, "the warp is a displacement field only for square slices (nx == ny)");
    MC_REQUIRE(n_iter >= 1 && n_iter <= 64, "n_iter must be in [1, 64]");
    const int64_t n = nvox(nx, ny, nz);
    void *ws;
    MC_TRY(workspace(ctx, "inv_m", 3 * n * sizeof(float), &ws));
    float *m = (float *)ws;
    const Fields<float> f{ax, ay, az, bx, by, bz};
    MC_LAUNCH(ctx, forward_dvf_kernel, stream_blocks(n), 256, 0, m, m + n, m + 2 * n, f, n, volume,
              flow);
    MC_LAUNCH(ctx, invert_dvf_kernel, dim3(div_up(nx, 32), div_up(ny, 8), nz), dim3(32, 8), 0,
              inv_x, inv_y, inv_z, m, m + n, m + 2 * n, nx, ny, nz, n_iter);
    return finish(ctx, "mcsart_invert_dvf");
}

MC_EXPORT int mcsart_add(mcsart_ctx *ctx, float *img1, const float *img, int nx, int ny, int nz,
                         float weight) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(img1 && img, "pointers must be non-NULL");
    const int64_t n = nvox(nx, ny, nz);
    MC_LAUNCH(ctx, add_kernel, stream_blocks(n), 256, 0, img1, img, n, weight);
    return finish(ctx, "mcsart_add");
}

MC_EXPORT int mcsart_add2(mcsart_ctx *ctx, float *img1, const float *img, int nx, int ny, int nz,
                          const float *img0, float weight, int ind) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(img1 && img && img0, "pointers must be non-NULL");
    MC_REQUIRE(ind >= 1 && ind <= 3, "ind must be 1, 2 or 3 (got %d)", ind);
    MC_LAUNCH(ctx, add2_kernel, stream_blocks(nvox(nx, ny, nz)), 256, 0, img1, img, nx, ny, nz,
              img0, weight, ind);
    return finish(ctx, "mcsart_add2");
}

MC_EXPORT int mcsart_initial(mcsart_ctx *ctx, float *img, int nx, int ny, int nz, float value) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(img, "img must be non-NULL");
    const int64_t n = nvox(nx, ny, nz);
    MC_LAUNCH(ctx, initial_kernel, stream_blocks(n), 256, 0, img, n, value);
    return finish(ctx, "mcsart_initial");
}

MC_EXPORT int mcsart_initial2(mcsart_ctx *ctx, float *img, int nx, int ny, int nz,
                              const float *img0, float volume, float flow) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(img && img0, "pointers must be non-NULL");
    MC_LAUNCH(ctx, initial2_kernel, stream_blocks(nvox(nx, ny, nz)), 256, 0, img, nx, ny, nz, img0,
              volume, flow);
    return finish(ctx, "mcsart_initial2");
}

MC_EXPORT int mcsart_division(mcsart_ctx *ctx, float *img1, const float *img, int nx, int ny,
                              int nz) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(img1 && img, "pointers must be non-NULL");
    const int64_t n = nvox(nx, ny, nz);
    MC_LAUNCH(ctx, division_kernel, stream_blocks(n), 256, 0, img1, img, n);
    return finish(ctx, "mcsart_division");
}

MC_EXPORT int mcsart_multiple(mcsart_ctx *ctx, float *img1, int nx, int ny, int nz,
                              const float *img0, float weight, int ind) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(img1 && img0, "pointers must be non-NULL");
    MC_REQUIRE(ind >= 1 && ind <= 3, "ind must be 1, 2 or 3 (got %d)", ind);
    MC_LAUNCH(ctx, multiple_kernel, stream_blocks(nvox(nx, ny, nz)), 256, 0, img1, nx, ny, nz,
              img0, weight, ind);
    return finish(ctx, "mcsart_multiple");
}

MC_EXPORT int mcsart_update_udvf(mcsart_ctx *ctx, float *ax, float *ay, float *az, float *bx,
                                 float *by, float *bz, const float *img, const float *img0,
                                 float volume_diff, float flow_diff, int nx, int ny, int nz,
                                 int iter) {
    clear_error();
    (void)iter;  // unused by the reference kernel too (cu_update_udvf.cu:11)
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(ax && ay && az && bx && by && bz && img && img0, "pointers must be non-NULL");
    MC_LAUNCH(ctx, update_udvf_kernel, stream_blocks(nvox(nx, ny, nz)), 256, 0, ax, ay, az, bx, by,
              bz, img, img0, volume_diff, flow_diff, nx, ny, nz);
    return finish(ctx, "mcsart_update_udvf");
}

MC_EXPORT int mcsart_diff(mcsart_ctx *ctx, float *img1, const float *img, int nx, int ny, int nz,
                          int ind) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(img1 && img, "pointers must be non-NULL");
    MC_REQUIRE(ind >= 1 && ind <= 3, "ind must be 1, 2 or 3 (got %d)", ind);
    MC_LAUNCH(ctx, diff_kernel, stream_blocks(nvox(nx, ny, nz)), 256, 0, img1, img, nx, ny, nz,
              ind);
    return finish(ctx, "mcsart_diff");
}

namespace mcsart {
__global__ void sumsq_kernel(const float *x, int64_t n, double *part) {
    double s = 0.0;
    MC_GRID_STRIDE(n) { s += (double)x[id] * (double)x[id]; }
    __shared__ double red[8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        part[blockIdx.x] = t;
    }
}
}  // namespace mcsart

MC_EXPORT int mcsart_snrm2(mcsart_ctx *ctx, int n, const float *d_x, float *h_result) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(n >= 0 && h_result, "n must be >= 0 and h_result non-NULL");
    if (n == 0) {
        *h_result = 0.0f;
        return MCSART_OK;
    }
    MC_REQUIRE(d_x, "d_x must be non-NULL");
    const unsigned blocks = std::min<unsigned>(div_up(n, 256), 1184u);
    void *ws;
    MC_TRY(workspace(ctx, "snrm2", blocks * sizeof(double), &ws));
    MC_LAUNCH(ctx, sumsq_kernel, blocks, 256, 0, d_x, (int64_t)n, (double *)ws);
    double host[1184];
    MC_CHECK_CUDA(cudaMemcpyAsync(host, ws, blocks * sizeof(double), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    MC_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    double s = 0.0;
    for (unsigned i = 0; i < blocks; i++) s += host[i];
    *h_result = (float)sqrt(s);
    return MCSART_OK;
}

// ------------------------------------------------- mixed-precision kernels
namespace {

template <typename VT>
int projection_ex_typed(mcsart_ctx *ctx, float *d_proj, const VT *d_img, int fp_sum, int geom64,
                        float angle, const Geom &g) {
    const int64_t V = nvox(g.nx, g.ny, g.nz);
    void *ws;
    MC_TRY(workspace(ctx, "fp_volT_ex", V * sizeof(VT), &ws));
    VT *imgT = (VT *)ws;
    MC_LAUNCH(ctx, (transpose_kernel<VT, VT>), dim3(div_up(g.nx, 32), div_up(g.ny, 32), g.nz),
              dim3(32, 8), 0, imgT, d_img, g.nx, g.ny);
    FPArgs<VT, 1, VT> a{};
    a.vol.std[0] = d_img;
    a.vol.tr[0] = imgT;
    a.g = g;
    a.angle = angle;
    a.mode = FP_PLAIN;
    a.out = d_proj;
    if (fp_sum == SUM_REF) {
        MC_LAUNCH(ctx, (fp_ref_kernel<1, false, VT, VT>),
                  dim3(div_up(g.na, FPC_COLS), div_up(g.nb, FPC_ROWS), 1), dim3(FPC_THREADS), 0,
                  a);
        return MCSART_OK;
    }
    const int groups = fp_auto_groups((int64_t)div_up(g.na, 32) * g.nb, std::max(g.nx, g.ny));
    const dim3 grid(div_up(g.na, 32), g.nb, 1), block(32, groups);
    const size_t smem = (size_t)groups * 2 * 32 * sizeof(float);
    if (fp_sum == SUM_PLAIN && geom64)
        MC_LAUNCH(ctx, (fp_kernel<1, false, SUM_PLAIN, VT, VT, true>), grid, block, smem, a);
    else if (fp_sum == SUM_PLAIN)
        MC_LAUNCH(ctx, (fp_kernel<1, false, SUM_PLAIN, VT, VT>), grid, block, smem, a);
    else if (geom64)
        MC_LAUNCH(ctx, (fp_kernel<1, false, SUM_KAHAN, VT, VT, true>), grid, block, smem, a);
    else
        MC_LAUNCH(ctx, (fp_kernel<1, false, SUM_KAHAN, VT, VT>), grid, block, smem, a);
    return MCSART_OK;
}

template <typename FT>
int deform_ex_typed(mcsart_ctx *ctx, FT *d_img1, const float *d_img, int nx, int ny, int nz,
                    float volume, float flow, const FT *fields, int interp) {
    const int64_t V = nvox(nx, ny, nz);
    const Fields<FT> f{fields, fields + V, fields + 2 * V, fields + 3 * V, fields + 4 * V,
                       fields + 5 * V};
    const unsigned blocks = stream_blocks(V);
    if (interp == MCSART_INTERP_TEXTURE) {
        if (!ctx->driver) ctx->driver.reset(new DriverState());
        TexVol &tv = ctx->driver->tv_deform;
        MC_TRY(tv.ensure(nx, ny, nz));
        MC_TRY(tv.upload(d_img, ctx->stream));
        MC_LAUNCH(ctx, (deform_typed_kernel<SrcTex, FT>), blocks, 256, 0, d_img1, SrcTex{tv.tex},
                  f, nx, ny, nz, volume, flow);
    } else {
        MC_LAUNCH(ctx, (deform_typed_kernel<SrcLinear<float>, FT>), blocks, 256, 0, d_img1,
                  SrcLinear<float>{d_img}, f, nx, ny, nz, volume, flow);
    }
    return MCSART_OK;
}

}  // namespace

MC_EXPORT int mcsart_projection_ex(mcsart_ctx *ctx, float *d_proj, const void *d_img,
                                   int storage, int fp_sum, int geom64, float angle, float SO,
                                   float SD, float da, int na, float ai, float db, int nb,
                                   float bi, int nx, int ny, int nz) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(d_proj && d_img, "d_proj and d_img must be non-NULL");
    MC_REQUIRE(storage >= MCSART_F32 && storage <= MCSART_F16, "unknown storage type %d", storage);
    MC_REQUIRE(fp_sum >= SUM_REF && fp_sum <= SUM_KAHAN, "fp_sum must be 0, 1 or 2");
    MC_REQUIRE(geom64 == 0 || geom64 == 1, "geom64 must be 0 or 1");
    MC_REQUIRE(geom64 == 0 || fp_sum != SUM_REF,
               "FP64 geometry (geom64) needs a split summation projector (fp_sum 1 or 2)");
    const Geom g = make_geom(SO, SD, da, na, ai, db, nb, bi, nx, ny, nz);
    MC_TRY(validate_geom(g));
    if (storage == MCSART_F32)
        MC_TRY(projection_ex_typed(ctx, d_proj, (const float *)d_img, fp_sum, geom64, angle, g));
    else if (storage == MCSART_BF16)
        MC_TRY(projection_ex_typed(ctx, d_proj, (const __nv_bfloat16 *)d_img, fp_sum, geom64,
                                   angle, g));
    else
        MC_TRY(projection_ex_typed(ctx, d_proj, (const __half *)d_img, fp_sum, geom64, angle, g));
    return finish(ctx, "mcsart_projection_ex");
}

MC_EXPORT int mcsart_backprojection_ex(mcsart_ctx *ctx, float *d_img, const float *d_proj,
                                       int geom64, float angle, float SO, float SD, float da,
                                       int na, float ai, float db, int nb, float bi, int nx,
                                       int ny, int nz) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(d_proj && d_img, "d_proj and d_img must be non-NULL");
    MC_REQUIRE(geom64 == 0 || geom64 == 1, "geom64 must be 0 or 1");
    if (!geom64)
        return mcsart_backprojection(ctx, d_img, d_proj, angle, SO, SD, da, na, ai, db, nb, bi,
                                     nx, ny, nz);
    const Geom g = make_geom(SO, SD, da, na, ai, db, nb, bi, nx, ny, nz);
    MC_TRY(validate_geom(g));
    BPArgs a{};
    a.proj = d_proj;
    a.g = g;
    a.angle = angle;
    a.out = d_img;
    const dim3 grid(div_up(nx, 32), div_up(ny, BP_ROWS), div_up(nz, BP_NZ)), block(32, BP_ROWS);
    MC_LAUNCH(ctx, (bp_kernel<1, BP_PLAIN, false, false, true>), grid, block, 0, a);
    return finish(ctx, "mcsart_backprojection_ex");
}

MC_EXPORT int mcsart_deform_ex(mcsart_ctx *ctx, void *d_img1, const float *d_img, int nx, int ny,
                               int nz, float volume, float flow, const void *d_fields, int storage,
                               int interp) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_TRY(validate_dims(nx, ny, nz));
    MC_REQUIRE(d_img1 && d_img && d_fields, "volume and field pointers must be non-NULL");
    MC_REQUIRE(d_img1 != (const void *)d_img, "d_img1 must not alias d_img");
    MC_REQUIRE(storage >= MCSART_F32 && storage <= MCSART_F16, "unknown storage type %d", storage);
    MC_REQUIRE(interp == MCSART_INTERP_TEXTURE || interp == MCSART_INTERP_EXACT,
               "unknown interpolation model %d", interp);
    if (storage == MCSART_F32)
        MC_TRY(deform_ex_typed(ctx, (float *)d_img1, d_img, nx, ny, nz, volume, flow,
                               (const float *)d_fields, interp));
    else if (storage == MCSART_BF16)
        MC_TRY(deform_ex_typed(ctx, (__nv_bfloat16 *)d_img1, d_img, nx, ny, nz, volume, flow,
                               (const __nv_bfloat16 *)d_fields, interp));
    else
        MC_TRY(deform_ex_typed(ctx, (__half *)d_img1, d_img, nx, ny, nz, volume, flow,
                               (const __half *)d_fields, interp));
    return finish(ctx, "mcsart_deform_ex");
}
