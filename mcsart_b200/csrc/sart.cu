// The SART / motion driver: replacement of host_AUMISART (src/AUMISART.cu:3-313).
//
// Per view the reference launches ~20 kernels, each followed by
// cudaDeviceSynchronize, allocates a cudaArray in every backprojection and
// warp, calls cublasSnrm2 twice in host-pointer mode and copies the measured
// projection H2D and the residual D2H.  Here every pass over the views is a
// fixed sequence of fused kernels on device-resident buffers:
//
//   image pass, static (overload 1, AUMISART.cu:42-63):
//     FP(img) + FP(ones) + residual + norms  ->  BP(residual)/BP(FP(ones)),
//     img += lambda * ratio (and its y-fastest copy)            2 kernels/view
//   image pass, motion-compensated (overload 2, :184-233):
//     warp(img) -> FP + FP(ones) + residual + norms -> BP ratio ->
//     img += lambda * warp^-1(ratio)                            4 kernels/view
//   motion pass (:66-118 / :236-288):
//     img0 and initial2 volumes -> FP of img, img0, ones + residual + norms ->
//     BP ratio -> six field updates                             4 kernels/view
//
// The sequence of a pass is captured once as a CUDA graph and replayed for
// every outer iteration of that kind.
#include <cstring>
#include <vector>

#include "backprojector.cuh"
#include "common.cuh"
#include "elementwise.cuh"
#include "projector.cuh"
#include "sart.cuh"
#include "warp.cuh"

#define MC_EXPORT extern "C" __attribute__((visibility("default")))

namespace mcsart {


int fp_auto_groups(int64_t ray_blocks, int n_slabs);
unsigned stream_blocks(int64_t n);

int DevBuf::ensure(size_t n) {
    if (bytes >= n && ptr) return MCSART_OK;
    release();
    const cudaError_t e = cudaMalloc(&ptr, n ? n : 1);
    if (e != cudaSuccess) {
        ptr = nullptr;
        set_error("device allocation of %zu bytes failed: %s", n, cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? MCSART_ERR_OUT_OF_MEMORY : MCSART_ERR_CUDA;
    }
    bytes = n;
    return MCSART_OK;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

void PassGraph::release() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    key.clear();
    kernels = 0;
}

enum PassKind { PASS_IMAGE_STATIC = 1, PASS_IMAGE_MC = 2, PASS_MOTION = 3 };

template <typename ST, int INTERP, int SUM> struct Runner {
    mcsart_ctx *ctx;
    DriverState &S;
    const Problem &P;
    const mcsart_options &opt;
    int64_t V = 0, NP = 0;
    int fp_bx = 0, fp_by = 0, fp_blocks = 0, groups = 1;
    int subset = 1;  // views per ordered subset in image passes
    int inv_iters = 0;  // fixed-point steps of the true DVF inverse (0: negated amplitudes)
    int cols_view = -1;  // first view whose backprojector column data the last projector wrote
    int cols_views = 0;  // and how many views from it
    std::vector<int> views_img, views_mot;
    std::vector<char> reads_std, reads_tr;  // per view: the copies its projector reads
    Tuning tune;  // launch shapes (variant indices; -1 = built-in choice)

    Runner(mcsart_ctx *c, const Problem &p, const mcsart_options &o)
        : ctx(c), S(*c->driver), P(p), opt(o) {
        tune = c->tuning_override ? *c->tuning_override : tuning_for(c, p.g, o.storage);
        V = nvox(P.g.nx, P.g.ny, P.g.nz);
        NP = (int64_t)P.g.na * P.g.nb;
        fp_bx = SUM == SUM_REF ? (int)div_up(P.g.na, FPC_COLS) : (int)div_up(P.g.na, 32);
        fp_by = SUM == SUM_REF ? (int)div_up(P.g.nb, FPC_ROWS) : P.g.nb;
        fp_blocks = fp_bx * fp_by;
        groups = SUM == SUM_REF ? 1
                 : opt.fp_groups > 0 ? std::min(opt.fp_groups, 8)
                                     : fp_auto_groups(fp_blocks, std::max(P.g.nx, P.g.ny));
        subset = std::min(std::max(opt.subset, 1), BP_MAX_VIEWS);
        inv_iters = P.motion_model ? opt.dvf_inverse : 0;
        for (int v = 0; v < P.n_views; v++) views_img.push_back(v);
        const int step = P.motion_model ? 1 : 10;  // AUMISART.cu:242 vs :72
        for (int v = 1; v < P.n_views; v += step) views_mot.push_back(v);
        reads_std.resize(P.n_views);
        reads_tr.resize(P.n_views);
        for (int v = 0; v < P.n_views; v++) {
            bool ax, ay;
            view_drive_axes(P.angles[v], P.g, &ax, &ay);
            reads_tr[v] = ax;
            reads_std[v] = ay;
        }
    }

    // A per-view copy of a volume the projector of view v reads, else nullptr.
    ST *std_or_null(int v, const DevBuf &b) const { return reads_std[v] ? b.as<ST>() : nullptr; }
    ST *tr_or_null(int v, const DevBuf &b) const { return reads_tr[v] ? b.as<ST>() : nullptr; }

    Fields<ST> fields() const {
        const ST *f = (const ST *)P.fields;
        return Fields<ST>{f, f + V, f + 2 * V, f + 3 * V, f + 4 * V, f + 5 * V};
    }
    const ST *meas(int v) const { return (const ST *)P.proj + (int64_t)v * NP; }

    int alloc() {
        const size_t vs = V * sizeof(ST), vf = V * sizeof(float);
        MC_TRY(S.img1.ensure(vs * subset));
        MC_TRY(S.img1T.ensure(vs * subset));
        MC_TRY(S.imgS.ensure(vs));
        MC_TRY(S.imgST.ensure(vs));
        // img0 and the initial2 volume interleaved for the reference-order
        // projector (PAIR), separate for the split-sum one
        MC_TRY(S.img0.ensure(2 * vs));
        MC_TRY(S.img0T.ensure(2 * vs));
        MC_TRY(S.ones.ensure(vs));
        MC_TRY(S.onesT.ensure(vs));
        MC_TRY(S.ratio.ensure(vf * subset));
        MC_TRY(S.imgT.ensure(vf));
        MC_TRY(S.pairs.ensure(NP * subset * sizeof(float2)));
        MC_TRY(S.bpcolA.ensure((size_t)P.g.nx * P.g.ny * subset * sizeof(float4)));
        MC_TRY(S.bpcolB.ensure((size_t)P.g.nx * P.g.ny * subset * sizeof(float)));
        if (INTERP == MCSART_INTERP_TEXTURE && P.motion_model) {
            MC_TRY(S.tv_img.ensure(P.g.nx, P.g.ny, P.g.nz));
            MC_TRY(S.tv_ratio.ensure(P.g.nx, P.g.ny, P.g.nz));
            for (int j = 1; j < subset; j++)
                MC_TRY(S.tv_ratio_sub[j - 1].ensure(P.g.nx, P.g.ny, P.g.nz));
        }
        if (inv_iters > 0) {
            MC_TRY(S.m3.ensure(3 * vf));
            MC_TRY(S.inv3.ensure(3 * vf));
        }
        MC_TRY(S.angles_dev.ensure((size_t)P.n_views * sizeof(float)));
        MC_CHECK_CUDA(cudaMemcpyAsync(S.angles_dev.ptr, P.angles, P.n_views * sizeof(float),
                                      cudaMemcpyHostToDevice, ctx->stream));
        MC_TRY(S.norm_part.ensure((size_t)P.n_views * fp_blocks * sizeof(double2)));
        MC_TRY(S.norm_tmp.ensure((size_t)P.n_views * sizeof(float)));
        MC_TRY(S.views_image.ensure((size_t)P.n_views * sizeof(int)));
        MC_TRY(S.views_motion.ensure((size_t)P.n_views * sizeof(int)));
        MC_CHECK_CUDA(cudaMemcpyAsync(S.views_image.ptr, views_img.data(),
                                      views_img.size() * sizeof(int), cudaMemcpyHostToDevice,
                                      ctx->stream));
        if (!views_mot.empty())
            MC_CHECK_CUDA(cudaMemcpyAsync(S.views_motion.ptr, views_mot.data(),
                                          views_mot.size() * sizeof(int),
                                          cudaMemcpyHostToDevice, ctx->stream));
        // the host vectors must stay valid until the copies ran
        MC_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
        return MCSART_OK;
    }

    template <int K, bool ONES, typename VT>
    int launch_fp(const FPVolumes<VT, K> &vol, int v, int k, int mode) {
        FPArgs<VT, K, ST> a{};
        a.vol = vol;
        a.g = P.g;
        a.angle = P.angles[v];
        a.angles = nullptr;
        a.mode = mode;
        a.meas = meas(v);
        a.resid = (mode == FP_IMAGE && P.resid) ? P.resid + (int64_t)v * NP : nullptr;
        a.bp_in = S.pairs.as<float2>();
        a.norm_part = S.norm_part.as<double2>() + (int64_t)k * fp_blocks;
        const dim3 grid(fp_bx, fp_by, 1);
        ctx->label = mode == FP_MOTION ? "fp_motion" : "fp_image";
        // the reference-order projector also writes the column data of this
        // view's backprojector, which follows it
        cols_view = SUM == SUM_REF ? v : -1;
        cols_views = 1;
        if (SUM == SUM_REF) {
            a.bpcolA = S.bpcolA.as<float4>();
            a.bpcolB = S.bpcolB.as<float>();
        }
        if constexpr (SUM == SUM_REF && K == 1) {
            // built-in: deeper slab groups when every block is resident at once
            const int var = tune.fp1 >= 0 ? tune.fp1 : fp_one_wave(ctx, fp_bx, fp_by) ? 1 : 0;
            // (slab-group depth, resident blocks per SM)
            switch (var) {
                case 1: MC_LAUNCH(ctx, (fp_ref_kernel<K, ONES, VT, ST, false, 4, 4>), grid,
                                  dim3(FPC_THREADS), 0, a); break;
                case 2: MC_LAUNCH(ctx, (fp_ref_kernel<K, ONES, VT, ST, false, 1, 8>), grid,
                                  dim3(FPC_THREADS), 0, a); break;
                case 3: MC_LAUNCH(ctx, (fp_ref_kernel<K, ONES, VT, ST, false, 2, 7>), grid,
                                  dim3(FPC_THREADS), 0, a); break;
                case 4: MC_LAUNCH(ctx, (fp_ref_kernel<K, ONES, VT, ST, false, 4, 5>), grid,
                                  dim3(FPC_THREADS), 0, a); break;
                default: MC_LAUNCH(ctx, (fp_ref_kernel<K, ONES, VT, ST, false, 2, 6>), grid,
                                   dim3(FPC_THREADS), 0, a);
            }
        } else if constexpr (SUM == SUM_REF) {
            // three volumes, the second and third paired (enqueue_motion)
            switch (tune.fp3) {
                case 1: MC_LAUNCH(ctx, (fp_ref_kernel<K, ONES, VT, ST, false, 2, 4, K == 3>), grid,
                                  dim3(FPC_THREADS), 0, a); break;
                case 2: MC_LAUNCH(ctx, (fp_ref_kernel<K, ONES, VT, ST, false, 2, 5, K == 3>), grid,
                                  dim3(FPC_THREADS), 0, a); break;
                case 3: MC_LAUNCH(ctx, (fp_ref_kernel<K, ONES, VT, ST, false, 4, 5, K == 3>), grid,
                                  dim3(FPC_THREADS), 0, a); break;
                default: MC_LAUNCH(ctx, (fp_ref_kernel<K, ONES, VT, ST, false, 4, 4, K == 3>), grid,
                                   dim3(FPC_THREADS), 0, a);
            }
        } else if (opt.geom64) {
            const size_t smem = (size_t)groups * (K + 1) * 32 * sizeof(float);
            MC_LAUNCH(ctx, (fp_kernel<K, ONES, SUM == SUM_REF ? SUM_PLAIN : SUM, VT, ST, true>),
                      grid, dim3(32, groups), smem, a);
        } else {
            const size_t smem = (size_t)groups * (K + 1) * 32 * sizeof(float);
            MC_LAUNCH(ctx, (fp_kernel<K, ONES, SUM, VT, ST>), grid, dim3(32, groups), smem, a);
        }
        return MCSART_OK;
    }

    // The backprojector's inputs for view v: the projector's (residual,
    // ones-projection) pairs and, when that launch wrote them, its column data.
    BPArgs bp_args(int v) {
        BPArgs b{};
        b.pair = S.pairs.as<float2>();
        b.g = P.g;
        b.angle = P.angles[v];
        b.lambda = P.lambda;
        if (cols_view == v) {
            b.colA = S.bpcolA.as<float4>();
            b.colB = S.bpcolB.as<float>();
        }
        return b;
    }

    // label: the profile label (default bp_div / bp_div_add by mode)
    int launch_bp(int v, int mode, float *out, float *outT, cudaSurfaceObject_t surf = 0,
                  const char *label = nullptr) {
        BPArgs b{};
        b.outSurf = surf;
        b.pair = S.pairs.as<float2>();
        b.g = P.g;
        b.angle = P.angles[v];
        b.lambda = P.lambda;
        b.out = out;
        b.outT = outT;
        if (cols_view == v) {
            b.colA = S.bpcolA.as<float4>();
            b.colB = S.bpcolB.as<float>();
        }
        ctx->label = label ? label : mode == BP_DIV ? "bp_div" : "bp_div_add";
        if (opt.geom64) {  // FP64 geometry and normaliser (no precomputed columns)
            b.colA = nullptr;
            b.colB = nullptr;
            const dim3 grid(div_up(P.g.nx, 32), div_up(P.g.ny, BP_ROWS), div_up(P.g.nz, BP_NZ)),
                block(32, BP_ROWS);
            if (mode == BP_DIV)
                MC_LAUNCH(ctx, (bp_kernel<2, BP_DIV, false, false, true>), grid, block, 0, b);
            else
                MC_LAUNCH(ctx, (bp_kernel<2, BP_DIV_ADD, false, false, true>), grid, block, 0, b);
            return MCSART_OK;
        }
        switch (tune.bp) {  // voxels per thread along z x voxel rows per block
            case 1: return launch_bp_shape<1, 4>(mode, b);
            case 2: return launch_bp_shape<2, 8>(mode, b);
            case 3: return launch_bp_shape<4, 4>(mode, b);
            default: return launch_bp_shape<BP_NZ, BP_ROWS>(mode, b);
        }
    }

    template <int NZ, int ROWS> int launch_bp_shape(int mode, const BPArgs &b) {
        const dim3 grid(div_up(P.g.nx, 32), div_up(P.g.ny, ROWS), div_up(P.g.nz, NZ)),
            block(32, ROWS);
        // the proven form skips the division range checks (bp_geom_proven)
        const bool proven = bp_geom_proven(P.g);
        if (mode == BP_DIV && proven) {
            MC_LAUNCH(ctx, (bp_kernel<2, BP_DIV, false, true, false, NZ, ROWS>), grid, block, 0, b);
        } else if (mode == BP_DIV) {
            MC_LAUNCH(ctx, (bp_kernel<2, BP_DIV, false, false, false, NZ, ROWS>), grid, block, 0, b);
        } else if (proven) {
            MC_LAUNCH(ctx, (bp_kernel<2, BP_DIV_ADD, false, true, false, NZ, ROWS>), grid, block, 0,
                      b);
        } else {
            MC_LAUNCH(ctx, (bp_kernel<2, BP_DIV_ADD, false, false, false, NZ, ROWS>), grid, block, 0,
                      b);
        }
        return MCSART_OK;
    }

    // Ordered subset of kk > 1 views v0 .. v0+kk-1 (list positions k0 ..): one
    // projector launch over the kk views (view = blockIdx.z), the volumes of
    // view j at +j*vol_stride.
    template <int K, bool ONES, typename VT>
    int launch_fp_subset(const FPVolumes<VT, K> &vol, int v0, int k0, int kk, int mode,
                         int64_t vol_stride) {
        FPArgs<VT, K, ST> a{};
        a.vol = vol;
        a.g = P.g;
        a.angle = P.angles[v0];
        a.angles = S.angles_dev.as<float>() + v0;
        a.mode = mode;
        a.meas = meas(v0);
        a.resid = (mode == FP_IMAGE && P.resid) ? P.resid + (int64_t)v0 * NP : nullptr;
        a.bp_in = S.pairs.as<float2>();
        a.norm_part = S.norm_part.as<double2>() + (int64_t)k0 * fp_blocks;
        a.vol_stride = vol_stride;
        // the kk views' backprojector column data for the launch that follows
        a.bpcolA = S.bpcolA.as<float4>();
        a.bpcolB = S.bpcolB.as<float>();
        cols_view = v0;
        cols_views = kk;
        ctx->label = mode == FP_MOTION ? "fp_motion" : "fp_image";
        MC_LAUNCH(ctx, (fp_ref_kernel<K, ONES, VT, ST, true>), dim3(fp_bx, fp_by, kk),
                  dim3(FPC_THREADS), 0, a);
        return MCSART_OK;
    }

    // One backprojector launch over the subset: BP_DIV writes view j's ratio
    // to out + j*V / surfs[j]; BP_DIV_ADD adds lambda/kk times the sum of the
    // views' ratios to out.
    int launch_bp_subset(int v0, int kk, int mode, float *out, float *outT,
                         const cudaSurfaceObject_t *surfs) {
        BPArgs b{};
        b.pair = S.pairs.as<float2>();
        b.g = P.g;
        b.angle = P.angles[v0];
        b.angles = S.angles_dev.as<float>() + v0;
        b.n_views = kk;
        b.lambda = P.lambda / (float)kk;
        b.out = out;
        b.outT = outT;
        for (int j = 0; j < kk && surfs; j++) b.outSurfs[j] = surfs[j];
        if (cols_view == v0 && cols_views == kk) {  // written by the subset's projector launch
            b.colA = S.bpcolA.as<float4>();
            b.colB = S.bpcolB.as<float>();
        }
        const dim3 grid(div_up(P.g.nx, 32), div_up(P.g.ny, BP_ROWS), div_up(P.g.nz, BP_NZ)),
            block(32, BP_ROWS);
        const bool proven = bp_geom_proven(P.g);
        ctx->label = mode == BP_DIV ? "bp_div" : "bp_div_add";
        if (mode == BP_DIV && proven) {
            MC_LAUNCH(ctx, (bp_kernel<2, BP_DIV, true, true>), grid, block, 0, b);
        } else if (mode == BP_DIV) {
            MC_LAUNCH(ctx, (bp_kernel<2, BP_DIV, true>), grid, block, 0, b);
        } else if (proven) {
            MC_LAUNCH(ctx, (bp_kernel<2, BP_DIV_ADD, true, true>), grid, block, 0, b);
        } else {
            MC_LAUNCH(ctx, (bp_kernel<2, BP_DIV_ADD, true>), grid, block, 0, b);
        }
        return MCSART_OK;
    }

    dim3 tile_grid() const { return dim3(div_up(P.g.nx, 32), div_up(P.g.ny, 32), P.g.nz); }
    // warp_fwd_kernel / warp_back_add_kernel: 32 x (8 * WR) tiles
    template <int WR = WARP_ROWS> dim3 warp_grid() const {
        return dim3(div_up(P.g.nx, 32), div_up(P.g.ny, 8 * WR), P.g.nz);
    }

    // The image pass's forward warp of the volume into view v's phase, in
    // the tuned launch shape (voxel rows per thread), writing only the
    // copies view v's projector reads.
    template <int WR> int warp_fwd_shape(int v, bool hw, float volume, float flow) {
        const Geom &g = P.g;
        const Fields<ST> f = fields();
        ST *d = reads_std[v] ? S.img1.as<ST>() : nullptr;
        ST *dT = reads_tr[v] ? S.img1T.as<ST>() : nullptr;
        ctx->label = "warp_fwd";
        if (hw) {
            MC_LAUNCH(ctx, (warp_fwd_kernel<SrcTex, ST, ST, WR>), warp_grid<WR>(), dim3(32, 8), 0,
                      d, dT, SrcTex{S.tv_img.tex}, f, g.nx, g.ny, g.nz, volume, flow);
        } else {
            MC_LAUNCH(ctx, (warp_fwd_kernel<SrcLinear<float>, ST, ST, WR>), warp_grid<WR>(),
                      dim3(32, 8), 0, d, dT, SrcLinear<float>{P.img}, f, g.nx, g.ny, g.nz, volume,
                      flow);
        }
        return MCSART_OK;
    }
    int warp_fwd(int v, bool hw, float volume, float flow) {
        switch (tune.warp) {
            case 1: return warp_fwd_shape<1>(v, hw, volume, flow);
            case 2: return warp_fwd_shape<4>(v, hw, volume, flow);
            default: return warp_fwd_shape<WARP_ROWS>(v, hw, volume, flow);
        }
    }
    // The backward warp of a view's correction and the update, tuned shape.
    template <int WR>
    int warp_back_shape(bool hw, cudaTextureObject_t tex, const float *lin, float ivolume,
                        float iflow, float lam) {
        const Geom &g = P.g;
        const Fields<ST> f = fields();
        ctx->label = "warp_back_add";
        if (hw) {
            MC_LAUNCH(ctx, (warp_back_add_kernel<SrcTex, ST, WR>), warp_grid<WR>(), dim3(32, 8), 0,
                      P.img, S.tv_img.surf, SrcTex{tex}, f, g.nx, g.ny, g.nz, ivolume, iflow, lam);
        } else {
            MC_LAUNCH(ctx, (warp_back_add_kernel<SrcLinear<float>, ST, WR>), warp_grid<WR>(),
                      dim3(32, 8), 0, P.img, (cudaSurfaceObject_t)0, SrcLinear<float>{lin}, f,
                      g.nx, g.ny, g.nz, ivolume, iflow, lam);
        }
        return MCSART_OK;
    }

    int finalize_norms(const int *views_dev, int n) {
        if (n == 0) return MCSART_OK;
        MC_LAUNCH(ctx, norm_finalize_kernel, div_up((int64_t)n * 32, 256), 256, 0,
                  S.norm_tmp.as<float>(), S.norm_part.as<double2>(), fp_blocks, views_dev, n);
        return MCSART_OK;
    }

    // AUMISART.cu:42-63
    int enqueue_image_static() {
        const Geom &g = P.g;
        MC_CHECK_CUDA(cudaMemsetAsync(S.norm_tmp.ptr, 0, P.n_views * sizeof(float), ctx->stream));
        MC_LAUNCH(ctx, (transpose_kernel<float, float>), tile_grid(), dim3(32, 8), 0,
                  S.imgT.as<float>(), P.img, g.nx, g.ny);
        FPVolumes<float, 1> vol{};
        vol.std[0] = P.img;
        vol.tr[0] = S.imgT.as<float>();
        const int n = (int)views_img.size();
        for (int k = 0; k < n; k += subset) {
            const int kk = std::min(subset, n - k), v = views_img[k];
            if (kk == 1) {  // one view at a time: the reference's loop
                MC_TRY((launch_fp<1, true, float>(vol, v, k, FP_IMAGE)));
                MC_TRY(launch_bp(v, BP_DIV_ADD, P.img, S.imgT.as<float>()));
            } else {
                MC_TRY((launch_fp_subset<1, true, float>(vol, v, k, kk, FP_IMAGE, 0)));
                MC_TRY(launch_bp_subset(v, kk, BP_DIV_ADD, P.img, S.imgT.as<float>(), nullptr));
            }
        }
        return finalize_norms(S.views_image.as<int>(), (int)views_img.size());
    }

    // The image pass's correction of view v, sampled from `tex` (texture
    // model) or `lin`, warped back to the reference phase and added with
    // weight lam: with the negated amplitudes (:222) or, with options
    // dvf_inverse, with the true inverse of the view's displacement.
    int back_warp_add(int v, bool hw, cudaTextureObject_t tex, const float *lin, float lam) {
        const Geom &g = P.g;
        const Fields<ST> f = fields();
        if (inv_iters > 0) {  // FP32 fields (validated)
            const float *F = (const float *)P.fields;
            const Fields<float> ff{F, F + V, F + 2 * V, F + 3 * V, F + 4 * V, F + 5 * V};
            const float volume = P.volumes[v] - P.volumes[0];
            const float flow = P.flows[v] - P.flows[0];
            float *m = S.m3.as<float>(), *n = S.inv3.as<float>();
            ctx->label = "dvf_inverse";
            MC_LAUNCH(ctx, forward_dvf_kernel, stream_blocks(V), 256, 0, m, m + V, m + 2 * V, ff,
                      V, volume, flow);
            ctx->label = "dvf_inverse";
            MC_LAUNCH(ctx, invert_dvf_kernel, dim3(div_up(g.nx, 32), div_up(g.ny, 8), g.nz),
                      dim3(32, 8), 0, n, n + V, n + 2 * V, m, m + V, m + 2 * V, g.nx, g.ny, g.nz,
                      inv_iters);
            ctx->label = "warp_back_add";
            if (hw) {
                MC_LAUNCH(ctx, warp_back_add_disp_kernel<SrcTex>, tile_grid(), dim3(32, 8), 0,
                          P.img, S.tv_img.surf, SrcTex{tex}, n, n + V, n + 2 * V, g.nx, g.ny,
                          g.nz, lam);
            } else {
                MC_LAUNCH(ctx, warp_back_add_disp_kernel<SrcLinear<float>>, tile_grid(),
                          dim3(32, 8), 0, P.img, (cudaSurfaceObject_t)0, SrcLinear<float>{lin}, n,
                          n + V, n + 2 * V, g.nx, g.ny, g.nz, lam);
            }
            return MCSART_OK;
        }
        const float ivolume = P.volumes[0] - P.volumes[v];  // :222
        const float iflow = P.flows[0] - P.flows[v];
        switch (tune.warp) {
            case 1: return warp_back_shape<1>(hw, tex, lin, ivolume, iflow, lam);
            case 2: return warp_back_shape<4>(hw, tex, lin, ivolume, iflow, lam);
            default: return warp_back_shape<WARP_ROWS>(hw, tex, lin, ivolume, iflow, lam);
        }
    }

    // Ordered subset of kk > 1 views in the motion-compensated image pass:
    // every view warps the same image to its phase (:193), one projector
    // launch and one backprojector launch serve the kk views, and each view's
    // ratio is warped back from its own phase (:222) and added with weight
    // lambda/kk, in view order.
    int image_mc_subset(int k0, int kk, bool hw) {
        const Geom &g = P.g;
        const Fields<ST> f = fields();
        const int v0 = views_img[k0];
        for (int j = 0; j < kk; j++) {
            const int v = v0 + j;
            const float volume = P.volumes[v] - P.volumes[0];
            const float flow = P.flows[v] - P.flows[0];
            ST *d = S.img1.as<ST>() + j * V, *dT = S.img1T.as<ST>() + j * V;
            ctx->label = "warp_fwd";
            if (hw) {
                MC_LAUNCH(ctx, (warp_fwd_kernel<SrcTex, ST, ST>), warp_grid<>(), dim3(32, 8), 0, d,
                          dT, SrcTex{S.tv_img.tex}, f, g.nx, g.ny, g.nz, volume, flow);
            } else {
                MC_LAUNCH(ctx, (warp_fwd_kernel<SrcLinear<float>, ST, ST>), warp_grid<>(),
                          dim3(32, 8), 0, d, dT, SrcLinear<float>{P.img}, f, g.nx, g.ny, g.nz,
                          volume, flow);
            }
        }
        FPVolumes<ST, 1> vol{};
        vol.std[0] = S.img1.as<ST>();
        vol.tr[0] = S.img1T.as<ST>();
        MC_TRY((launch_fp_subset<1, true, ST>(vol, v0, k0, kk, FP_IMAGE, V)));
        cudaSurfaceObject_t surfs[BP_MAX_VIEWS] = {};
        for (int j = 0; j < kk; j++) surfs[j] = j == 0 ? S.tv_ratio.surf : S.tv_ratio_sub[j - 1].surf;
        if (hw)
            MC_TRY(launch_bp_subset(v0, kk, BP_DIV, nullptr, nullptr, surfs));
        else
            MC_TRY(launch_bp_subset(v0, kk, BP_DIV, S.ratio.as<float>(), nullptr, nullptr));
        const float lam = P.lambda / (float)kk;
        for (int j = 0; j < kk; j++) {
            const cudaTextureObject_t t = j == 0 ? S.tv_ratio.tex : S.tv_ratio_sub[j - 1].tex;
            MC_TRY(back_warp_add(v0 + j, hw, t, S.ratio.as<float>() + j * V, lam));
        }
        return MCSART_OK;
    }

    // AUMISART.cu:184-233 with P = 1.  TEXTURE model: the volume and the
    // normalised correction live in 3D arrays sampled by the texture unit; the
    // backprojector and the update write them through surfaces, so the only
    // copy is the volume's upload at the start of the pass.
    int enqueue_image_mc() {
        const Geom &g = P.g;
        const Fields<ST> f = fields();
        MC_CHECK_CUDA(cudaMemsetAsync(S.norm_tmp.ptr, 0, P.n_views * sizeof(float), ctx->stream));
        const bool hw = INTERP == MCSART_INTERP_TEXTURE;
        if (hw) MC_TRY(S.tv_img.upload(P.img, ctx->stream));
        FPVolumes<ST, 1> vol{};
        vol.std[0] = S.img1.as<ST>();
        vol.tr[0] = S.img1T.as<ST>();
        const int n = (int)views_img.size();
        for (int k = 0; k < n; k += subset) {
            const int kk = std::min(subset, n - k);
            if (kk > 1) {
                MC_TRY(image_mc_subset(k, kk, hw));
                continue;
            }
            const int v = views_img[k];
            const float volume = P.volumes[v] - P.volumes[0];   // :193
            const float flow = P.flows[v] - P.flows[0];
            MC_TRY(warp_fwd(v, hw, volume, flow));
            MC_TRY((launch_fp<1, true, ST>(vol, v, k, FP_IMAGE)));
            if (hw)
                MC_TRY(launch_bp(v, BP_DIV, nullptr, nullptr, S.tv_ratio.surf));
            else
                MC_TRY(launch_bp(v, BP_DIV, S.ratio.as<float>(), nullptr));
            MC_TRY(back_warp_add(v, hw, S.tv_ratio.tex, S.ratio.as<float>(), P.lambda));
        }
        return finalize_norms(S.views_image.as<int>(), (int)views_img.size());
    }

    // AUMISART.cu:66-118 (step 10) / :236-288 (step 1)
    int enqueue_motion() {
        const Geom &g = P.g;
        const Fields<ST> f = fields();
        ST *fw = (ST *)P.fields;
        MC_CHECK_CUDA(cudaMemsetAsync(S.norm_tmp.ptr, 0, P.n_views * sizeof(float), ctx->stream));
        FPVolumes<ST, 3> vol{};
        if (sizeof(ST) == sizeof(float)) {
            vol.std[0] = (const ST *)P.img;
        } else {
            MC_LAUNCH(ctx, (cast_kernel<ST>), stream_blocks(V), 256, 0, S.imgS.as<ST>(),
                      (const float *)P.img, V);
            vol.std[0] = S.imgS.as<ST>();
        }
        MC_LAUNCH(ctx, (transpose_kernel<float, ST>), tile_grid(), dim3(32, 8), 0,
                  S.imgST.as<ST>(), (const float *)P.img, g.nx, g.ny);
        vol.tr[0] = S.imgST.as<ST>();
        // the reference-order projector reads img0 and the initial2 volume
        // as interleaved pairs (one load for both), the split-sum one apart
        constexpr bool pair = SUM == SUM_REF;
        vol.std[1] = S.img0.as<ST>();
        vol.tr[1] = S.img0T.as<ST>();
        vol.std[2] = pair ? nullptr : S.ones.as<ST>();
        vol.tr[2] = pair ? nullptr : S.onesT.as<ST>();
        ST *const ones_std = pair ? nullptr : S.ones.as<ST>();
        ST *const ones_tr = pair ? nullptr : S.onesT.as<ST>();
        // square slices: each view's field update and the next view's prep
        // run as one kernel (one pass over the fields)
        const bool fuse = g.nx == g.ny;
        const int nm = (int)views_mot.size();
        for (int k = 0; k < nm; k++) {
            const int v = views_mot[k];
            const float vd = P.volumes[v] - P.volumes[v - 1];  // :249-250
            const float fd = P.flows[v] - P.flows[v - 1];
            if (!fuse || k == 0) {
                ctx->label = "motion_prep";
                MC_LAUNCH(ctx, (motion_prep_kernel<ST, ST, pair>), tile_grid(), dim3(32, 8), 0,
                          std_or_null(v, S.img0), tr_or_null(v, S.img0T),
                          reads_std[v] ? ones_std : nullptr, reads_tr[v] ? ones_tr : nullptr,
                          (const float *)P.img, f, g.nx, g.ny, g.nz, vd, fd);
            }
            MC_TRY((launch_fp<3, false, ST>(vol, v, k, FP_MOTION)));
            // square slices, FP32 geometry: the backprojection ratio is
            // computed inside the field update (field_update_prep_kernel's
            // BP form) unless the tuning chose a separate field update
            const bool fused_bp = fuse && k + 1 < nm && !opt.geom64 && tune.fup <= 0;
            if (!fused_bp)
                MC_TRY(launch_bp(v, BP_DIV, S.ratio.as<float>(), nullptr, 0, "bp_div_motion"));
            const float nvd = P.volumes[v - 1] - P.volumes[v];  // :272-277
            const float nfd = P.flows[v - 1] - P.flows[v];
            if (fuse && k + 1 < nm) {
                const int vn = views_mot[k + 1];
                const float vdn = P.volumes[vn] - P.volumes[vn - 1];
                const float fdn = P.flows[vn] - P.flows[vn - 1];
                ctx->label = fused_bp ? "bp_field_update_prep" : "field_update_prep";
                ST *const o_std = reads_std[vn] ? ones_std : nullptr;
                ST *const o_tr = reads_tr[vn] ? ones_tr : nullptr;
                const BPArgs b = bp_args(v);
                if (fused_bp && bp_geom_proven(g))
                    MC_LAUNCH(ctx, (field_update_prep_kernel<ST, ST, false, pair, true, true>),
                              tile_grid(), dim3(32, 8), 0, fw, fw + V, fw + 2 * V, fw + 3 * V,
                              fw + 4 * V, fw + 5 * V, (const float *)nullptr, (const float *)P.img,
                              g.nx, g.ny, g.nz, nvd, nfd, std_or_null(vn, S.img0),
                              tr_or_null(vn, S.img0T), o_std, o_tr, vdn, fdn, b);
                else if (fused_bp)
                    MC_LAUNCH(ctx, (field_update_prep_kernel<ST, ST, false, pair, true, false>),
                              tile_grid(), dim3(32, 8), 0, fw, fw + V, fw + 2 * V, fw + 3 * V,
                              fw + 4 * V, fw + 5 * V, (const float *)nullptr, (const float *)P.img,
                              g.nx, g.ny, g.nz, nvd, nfd, std_or_null(vn, S.img0),
                              tr_or_null(vn, S.img0T), o_std, o_tr, vdn, fdn, b);
                else if (tune.fup == 1)
                    MC_LAUNCH(ctx, (field_update_prep_kernel<ST, ST, true, pair>), tile_grid(),
                              dim3(32, 8), 0, fw, fw + V, fw + 2 * V, fw + 3 * V, fw + 4 * V,
                              fw + 5 * V, (const float *)S.ratio.as<float>(), (const float *)P.img,
                              g.nx, g.ny, g.nz, nvd, nfd, std_or_null(vn, S.img0),
                              tr_or_null(vn, S.img0T), o_std, o_tr, vdn, fdn, b);
                else
                    MC_LAUNCH(ctx, (field_update_prep_kernel<ST, ST, false, pair>), tile_grid(),
                              dim3(32, 8), 0, fw, fw + V, fw + 2 * V, fw + 3 * V, fw + 4 * V,
                              fw + 5 * V, (const float *)S.ratio.as<float>(), (const float *)P.img,
                              g.nx, g.ny, g.nz, nvd, nfd, std_or_null(vn, S.img0),
                              tr_or_null(vn, S.img0T), o_std, o_tr, vdn, fdn, b);
            } else {
                ctx->label = "field_update";
                MC_LAUNCH(ctx, (field_update_kernel<ST>), tile_grid(), dim3(32, 8), 0, fw, fw + V,
                          fw + 2 * V, fw + 3 * V, fw + 4 * V, fw + 5 * V,
                          (const float *)S.ratio.as<float>(), (const float *)P.img, g.nx, g.ny,
                          g.nz, nvd, nfd);
            }
        }
        return finalize_norms(S.views_motion.as<int>(), (int)views_mot.size());
    }

    int enqueue(int kind) {
        switch (kind) {
            case PASS_IMAGE_STATIC: return enqueue_image_static();
            case PASS_IMAGE_MC: return enqueue_image_mc();
            default: return enqueue_motion();
        }
    }

    std::vector<uint8_t> graph_key(int kind) const {
        std::vector<uint8_t> k;
        auto put = [&](const void *p, size_t n) {
            const uint8_t *b = (const uint8_t *)p;
            k.insert(k.end(), b, b + n);
        };
        // the storage type itself, not its size: BF16 and F16 are both 2 bytes
        const int hdr[15] = {kind, opt.storage, INTERP, SUM, groups, (int)P.motion_model,
                             (int)views_mot.size(), subset, inv_iters, opt.geom64,
                             tune.fp1, tune.fp3, tune.bp, tune.warp, tune.fup};
        put(hdr, sizeof(hdr));
        put(views_img.data(), views_img.size() * sizeof(int));
        put(views_mot.data(), views_mot.size() * sizeof(int));
        put(&P.g, sizeof(Geom));
        put(&P.n_views, sizeof(int));
        put(&P.lambda, sizeof(float));
        const void *ptrs[4] = {P.img, P.proj, P.fields, P.resid};
        put(ptrs, sizeof(ptrs));
        const void *bufs[16] = {S.img1.ptr, S.img1T.ptr, S.imgS.ptr, S.imgST.ptr, S.img0.ptr,
                                S.img0T.ptr, S.ones.ptr, S.onesT.ptr, S.ratio.ptr, S.imgT.ptr,
                                S.pairs.ptr, S.norm_part.ptr, (const void *)S.tv_img.arr,
                                (const void *)S.tv_ratio.arr, S.bpcolA.ptr, S.bpcolB.ptr};
        put(bufs, sizeof(bufs));
        put(P.angles, P.n_views * sizeof(float));
        put(P.volumes, P.n_views * sizeof(float));
        put(P.flows, P.n_views * sizeof(float));
        return k;
    }

    int run_pass(int kind) {
        if (!opt.use_graph || ctx->profiling) return enqueue(kind);
        PassGraph &pg = S.graphs[kind];
        std::vector<uint8_t> key = graph_key(kind);
        if (pg.exec == nullptr || pg.key != key) {
            pg.release();
            // Capture on the context's own stream: the caller's stream may be the
            // legacy default stream, which cannot be captured.  Capturing runs
            // nothing, so no ordering with the caller's stream is needed here.
            cudaStream_t user = ctx->stream;
            ctx->stream = ctx->own_stream;
            cudaError_t eb = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
            if (eb != cudaSuccess) {
                ctx->stream = user;
                MC_CHECK_CUDA(eb);
            }
            const long long before = ctx->launches;
            const int rc = enqueue(kind);
            cudaGraph_t graph = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &graph);
            ctx->stream = user;
            if (rc != MCSART_OK) {
                if (graph) cudaGraphDestroy(graph);
                return rc;
            }
            MC_CHECK_CUDA(ec);
            const cudaError_t ei = cudaGraphInstantiate(&pg.exec, graph, 0);
            cudaGraphDestroy(graph);
            MC_CHECK_CUDA(ei);
            pg.key = std::move(key);
            pg.kernels = ctx->launches - before;
            ctx->launches = before;
        }
        MC_CHECK_CUDA(cudaGraphLaunch(pg.exec, ctx->stream));
        ctx->launches += pg.kernels;
        return MCSART_OK;
    }

    int run(int n_iter, const int *op_iter, float *norm_out) {
        MC_TRY(alloc());
        for (int it = 0; it < n_iter; it++) {
            int kind;
            if (op_iter[it] == 1)
                kind = P.motion_model ? PASS_IMAGE_MC : PASS_IMAGE_STATIC;
            else
                kind = PASS_MOTION;
            MC_TRY(run_pass(kind));
            if (norm_out)
                MC_CHECK_CUDA(cudaMemcpyAsync(norm_out + (int64_t)it * P.n_views, S.norm_tmp.ptr,
                                              P.n_views * sizeof(float), cudaMemcpyDeviceToDevice,
                                              ctx->stream));
        }
        return MCSART_OK;
    }
};

template <typename ST>
int run_typed(mcsart_ctx *ctx, const Problem &P, int n_iter, const int *op_iter, float *norm_out,
              const mcsart_options &opt) {
#define MC_RUN(I, S) return Runner<ST, I, S>(ctx, P, opt).run(n_iter, op_iter, norm_out)
    if (opt.interp == MCSART_INTERP_TEXTURE) {
        if (opt.fp_sum == SUM_REF) MC_RUN(MCSART_INTERP_TEXTURE, SUM_REF);
        if (opt.fp_sum == SUM_PLAIN) MC_RUN(MCSART_INTERP_TEXTURE, SUM_PLAIN);
        MC_RUN(MCSART_INTERP_TEXTURE, SUM_KAHAN);
    }
    if (opt.fp_sum == SUM_REF) MC_RUN(MCSART_INTERP_EXACT, SUM_REF);
    if (opt.fp_sum == SUM_PLAIN) MC_RUN(MCSART_INTERP_EXACT, SUM_PLAIN);
    MC_RUN(MCSART_INTERP_EXACT, SUM_KAHAN);
#undef MC_RUN
}

int run_driver(mcsart_ctx *ctx, const Problem &P, int n_iter, const int *op_iter, float *norm_out,
               const mcsart_options &opt) {
    if (!ctx->driver) ctx->driver.reset(new DriverState());
    switch (opt.storage) {
        case MCSART_F32: return run_typed<float>(ctx, P, n_iter, op_iter, norm_out, opt);
        case MCSART_BF16: return run_typed<__nv_bfloat16>(ctx, P, n_iter, op_iter, norm_out, opt);
        case MCSART_F16: return run_typed<__half>(ctx, P, n_iter, op_iter, norm_out, opt);
        default: set_error("unknown storage type %d", opt.storage); return MCSART_ERR_INVALID_ARGUMENT;
    }
}

int validate_options(const mcsart_options &o) {
    MC_REQUIRE(o.storage >= MCSART_F32 && o.storage <= MCSART_F16, "unknown storage type %d",
               o.storage);
    MC_REQUIRE(o.interp == MCSART_INTERP_TEXTURE || o.interp == MCSART_INTERP_EXACT,
               "unknown interpolation model %d", o.interp);
    MC_REQUIRE(o.fp_groups >= 0 && o.fp_groups <= 8, "fp_groups must be in [0, 8]");
    MC_REQUIRE(o.fp_sum >= SUM_REF && o.fp_sum <= SUM_KAHAN, "fp_sum must be 0, 1 or 2");
    MC_REQUIRE(o.subset >= 0 && o.subset <= BP_MAX_VIEWS, "subset must be in [0, %d]",
               BP_MAX_VIEWS);
    MC_REQUIRE(o.subset <= 1 || o.fp_sum == SUM_REF,
               "ordered subsets (subset > 1) use the reference-order projector (fp_sum 0)");
    MC_REQUIRE(o.dvf_inverse >= 0 && o.dvf_inverse <= 64, "dvf_inverse must be in [0, 64]");
    MC_REQUIRE(o.dvf_inverse == 0 || o.storage == MCSART_F32,
               "the true DVF inverse (dvf_inverse > 0) needs FP32 storage");
    MC_REQUIRE(o.geom64 == 0 || o.geom64 == 1, "geom64 must be 0 or 1");
    MC_REQUIRE(o.geom64 == 0 || o.fp_sum != SUM_REF,
               "FP64 geometry (geom64) needs a split summation projector (fp_sum 1 or 2)");
    MC_REQUIRE(o.autotune == 0 || o.autotune == 1, "autotune must be 0 or 1");
    return MCSART_OK;
}

int validate_iter(int n_views, int n_iter, const int *op_iter, const float *angles,
                  const float *volumes, const float *flows) {
    MC_REQUIRE(n_views > 0, "n_views must be positive");
    MC_REQUIRE(n_iter >= 0, "n_iter must be >= 0");
    MC_REQUIRE(n_iter == 0 || op_iter, "op_iter must be non-NULL");
    MC_REQUIRE(angles && volumes && flows, "angles, volumes and flows must be non-NULL");
    return MCSART_OK;
}

}  // namespace mcsart

using namespace mcsart;

MC_EXPORT void mcsart_default_options(mcsart_options *opt) {
    if (!opt) return;
    opt->storage = MCSART_F32;
    opt->interp = MCSART_INTERP_TEXTURE;
    opt->use_graph = 1;
    opt->fp_sum = SUM_REF;
    opt->fp_groups = 0;
    opt->subset = 1;
    opt->dvf_inverse = 0;
    opt->geom64 = 0;
    opt->autotune = 0;
}

// The driver's view of a device-resident problem (validated); overload 1
// (no fields) gets the context's zero-initialised fields.
static int prepare_problem(mcsart_ctx *ctx, const mcsart_problem *prob, const mcsart_options &opt,
                           Problem &P) {
    Geom g;
    g.SO = prob->SO; g.SD = prob->SD; g.da = prob->da; g.ai = prob->ai; g.db = prob->db;
    g.bi = prob->bi; g.na = prob->na; g.nb = prob->nb; g.nx = prob->nx; g.ny = prob->ny;
    g.nz = prob->nz;
    MC_TRY(validate_geom(g));
    MC_REQUIRE(prob->n_views > 0, "n_views must be positive");
    MC_REQUIRE(prob->h_angles && prob->h_volumes && prob->h_flows,
               "angles, volumes and flows must be non-NULL");
    MC_REQUIRE(prob->d_img && prob->d_proj, "d_img and d_proj must be non-NULL");
    MC_REQUIRE(opt.dvf_inverse == 0 || prob->d_fields == nullptr || prob->nx == prob->ny,
               "the true DVF inverse (dvf_inverse > 0) needs square slices (nx == ny)");
    if (!ctx->driver) ctx->driver.reset(new DriverState());
    DriverState &S = *ctx->driver;
    const int64_t V = nvox(g.nx, g.ny, g.nz);
    const size_t es = opt.storage == MCSART_F32 ? 4 : 2;
    P = Problem();
    P.g = g;
    P.n_views = prob->n_views;
    P.lambda = prob->lambda;
    P.angles = prob->h_angles;
    P.volumes = prob->h_volumes;
    P.flows = prob->h_flows;
    P.img = prob->d_img;
    P.proj = prob->d_proj;
    P.motion_model = prob->d_fields != nullptr;
    P.resid = prob->d_resid;
    if (P.motion_model) {
        P.fields = prob->d_fields;
    } else {  // overload 1: the DVF starts at zero (AUMISART.cu:25-30)
        MC_TRY(S.zero_fields.ensure(6 * V * es));
        MC_CHECK_CUDA(cudaMemsetAsync(S.zero_fields.ptr, 0, 6 * V * es, ctx->stream));
        P.fields = S.zero_fields.ptr;
    }
    return MCSART_OK;
}

MC_EXPORT int mcsart_aumisart_device(mcsart_ctx *ctx, const mcsart_problem *prob, int n_iter,
                                     const int *h_op_iter, const mcsart_options *opt_in) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(prob, "problem is NULL");
    mcsart_options opt;
    if (opt_in) opt = *opt_in; else mcsart_default_options(&opt);
    MC_TRY(validate_options(opt));
    MC_TRY(validate_iter(prob->n_views, n_iter, h_op_iter, prob->h_angles, prob->h_volumes,
                         prob->h_flows));
    Problem P;
    MC_TRY(prepare_problem(ctx, prob, opt, P));
    if (opt.autotune && !ctx->tuning.count(tuning_key(P.g, opt.storage)))
        MC_TRY(autotune_problem(ctx, P, opt));
    if (prob->d_norm)
        MC_CHECK_CUDA(cudaMemsetAsync(prob->d_norm, 0, (size_t)n_iter * prob->n_views * sizeof(float),
                                      ctx->stream));
    MC_TRY(run_driver(ctx, P, n_iter, h_op_iter, prob->d_norm, opt));
    return finish(ctx, "mcsart_aumisart_device");
}

MC_EXPORT int mcsart_autotune(mcsart_ctx *ctx, const mcsart_problem *prob,
                              const mcsart_options *opt_in) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(prob, "problem is NULL");
    mcsart_options opt;
    if (opt_in) opt = *opt_in; else mcsart_default_options(&opt);
    MC_TRY(validate_options(opt));
    Problem P;
    MC_TRY(prepare_problem(ctx, prob, opt, P));
    MC_TRY(autotune_problem(ctx, P, opt));
    return finish(ctx, "mcsart_autotune");
}

MC_EXPORT int mcsart_batch_run(mcsart_ctx *ctx, const mcsart_problem *problems,
                               int n_problems, int n_iter, const int *h_op_iter,
                               const mcsart_options *opt) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(problems != nullptr, "problems is NULL");
    MC_REQUIRE(n_problems > 0 && n_problems <= MCSART_BATCH_MAX,
               "n_problems must be in [1, %d] (got %d)", MCSART_BATCH_MAX, n_problems);
    // lanes: child contexts on their own non-blocking streams
    while ((int)ctx->lanes.size() < n_problems) {
        std::unique_ptr<mcsart_ctx> lane(new mcsart_ctx());
        lane->device = ctx->device;
        lane->sms = ctx->sms;
        MC_CHECK_CUDA(cudaStreamCreateWithFlags(&lane->own_stream, cudaStreamNonBlocking));
        lane->stream = lane->own_stream;
        cudaEvent_t done;
        MC_CHECK_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        ctx->lane_done.push_back(done);
        ctx->lanes.push_back(std::move(lane));
    }
    if (!ctx->batch_start)
        MC_CHECK_CUDA(cudaEventCreateWithFlags(&ctx->batch_start, cudaEventDisableTiming));
    // the lanes start after the work already queued on the caller's stream
    MC_CHECK_CUDA(cudaEventRecord(ctx->batch_start, ctx->stream));
    int rc = MCSART_OK, started = 0;
    char msg[512] = "";
    for (int i = 0; i < n_problems; i++) {
        mcsart_ctx *lane = ctx->lanes[i].get();
        lane->profiling = ctx->profiling;
        MC_CHECK_CUDA(cudaStreamWaitEvent(lane->stream, ctx->batch_start, 0));
        const long long l0 = lane->launches;
        started = i + 1;
        rc = mcsart_aumisart_device(lane, &problems[i], n_iter, h_op_iter, opt);
        ctx->launches += lane->launches - l0;
        if (rc != MCSART_OK) {
            snprintf(msg, sizeof(msg), "problem %d: %s", i, mcsart_last_error());
            break;
        }
    }
    // the caller's stream waits for every lane that was started, also on error
    for (int i = 0; i < started; i++) {
        MC_CHECK_CUDA(cudaEventRecord(ctx->lane_done[i], ctx->lanes[i]->stream));
        MC_CHECK_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->lane_done[i], 0));
    }
    if (rc != MCSART_OK) {
        set_error("%s", msg);
        return rc;
    }
    return finish(ctx, "mcsart_batch_run");
}

// host_AUMISART with host pointers; h_out_fields[0..5] receive the final
// alpha_x, alpha_y, alpha_z, beta_x, beta_y, beta_z (NULL entries skipped).
static int aumisart_host(mcsart_ctx *ctx, float *h_outimg, float *h_outproj, float *h_outnorm,
                         float *const *h_out_fields, const float *h_img, const float *h_proj,
                         int nx, int ny, int nz, int na, int nb, int outIter, int n_views,
                         int n_iter, const int *op_iter, float da, float db, float ai, float bi,
                         float SO, float SD, float dx, float lambda, const float *volumes,
                         const float *flows, const float *err_weights, const float *angles,
                         const float *ax, const float *ay, const float *az, const float *bx,
                         const float *by, const float *bz) {
    clear_error();
    (void)outIter; (void)dx; (void)err_weights;  // unused by the reference as well
    MC_TRY(validate_ctx(ctx));
    Geom g;
    g.SO = SO; g.SD = SD; g.da = da; g.ai = ai; g.db = db; g.bi = bi;
    g.na = na; g.nb = nb; g.nx = nx; g.ny = ny; g.nz = nz;
    MC_TRY(validate_geom(g));
    MC_TRY(validate_iter(n_views, n_iter, op_iter, angles, volumes, flows));
    MC_REQUIRE(h_outimg && h_outproj && h_outnorm && h_out_fields[0] && h_img && h_proj,
               "image, projection and output pointers must be non-NULL");
    const bool motion = ax != nullptr;
    MC_REQUIRE(!motion || (ay && az && bx && by && bz),
               "alpha_x given: all six DVF fields must be non-NULL");
    if (!ctx->driver) ctx->driver.reset(new DriverState());
    DriverState &S = *ctx->driver;
    const int64_t V = nvox(nx, ny, nz), NP = (int64_t)na * nb;
    const size_t vb = V * sizeof(float), pb = (size_t)n_views * NP * sizeof(float);
    MC_TRY(S.h_img.ensure(vb));
    MC_TRY(S.h_proj.ensure(pb));
    MC_TRY(S.h_fields.ensure(6 * vb));
    MC_TRY(S.h_resid.ensure(pb));
    MC_TRY(S.h_norm.ensure((size_t)std::max(1, n_iter * n_views) * sizeof(float)));
    cudaStream_t st = ctx->stream;
    MC_CHECK_CUDA(cudaMemcpyAsync(S.h_img.ptr, h_img, vb, cudaMemcpyHostToDevice, st));
    MC_CHECK_CUDA(cudaMemcpyAsync(S.h_proj.ptr, h_proj, pb, cudaMemcpyHostToDevice, st));
    float *F = S.h_fields.as<float>();
    if (motion) {
        const float *src[6] = {ax, ay, az, bx, by, bz};
        for (int c = 0; c < 6; c++)
            MC_CHECK_CUDA(cudaMemcpyAsync(F + c * V, src[c], vb, cudaMemcpyHostToDevice, st));
    } else {
        MC_CHECK_CUDA(cudaMemsetAsync(F, 0, 6 * vb, st));
    }
    MC_CHECK_CUDA(cudaMemsetAsync(S.h_resid.ptr, 0, pb, st));
    MC_CHECK_CUDA(cudaMemsetAsync(S.h_norm.ptr, 0, (size_t)n_iter * n_views * sizeof(float), st));
    Problem P;
    P.g = g;
    P.n_views = n_views;
    P.lambda = lambda;
    P.angles = angles;
    P.volumes = volumes;
    P.flows = flows;
    P.img = S.h_img.as<float>();
    P.proj = S.h_proj.ptr;
    P.fields = F;
    P.motion_model = motion;
    P.resid = S.h_resid.as<float>();
    mcsart_options opt;
    mcsart_default_options(&opt);
    opt.interp = ctx->interp;
    MC_TRY(run_driver(ctx, P, n_iter, op_iter, S.h_norm.as<float>(), opt));
    MC_CHECK_CUDA(cudaMemcpyAsync(h_outimg, S.h_img.ptr, vb, cudaMemcpyDeviceToHost, st));
    MC_CHECK_CUDA(cudaMemcpyAsync(h_outproj, S.h_resid.ptr, pb, cudaMemcpyDeviceToHost, st));
    MC_CHECK_CUDA(cudaMemcpyAsync(h_outnorm, S.h_norm.ptr, (size_t)n_iter * n_views * sizeof(float),
                                  cudaMemcpyDeviceToHost, st));
    for (int c = 0; c < 6; c++)
        if (h_out_fields[c])
            MC_CHECK_CUDA(cudaMemcpyAsync(h_out_fields[c], F + c * V, vb, cudaMemcpyDeviceToHost, st));
    MC_CHECK_CUDA(cudaStreamSynchronize(st));
    return MCSART_OK;
}

MC_EXPORT int mcsart_aumisart(mcsart_ctx *ctx, float *h_outimg, float *h_outproj,
                              float *h_outnorm, float *h_outalphax, const float *h_img,
                              const float *h_proj, int nx, int ny, int nz, int na, int nb,
                              int outIter, int n_views, int n_iter, const int *op_iter, float da,
                              float db, float ai, float bi, float SO, float SD, float dx,
                              float lambda, const float *volumes, const float *flows,
                              const float *err_weights, const float *angles, const float *ax,
                              const float *ay, const float *az, const float *bx,
                              const float *by, const float *bz) {
    float *const out[6] = {h_outalphax, nullptr, nullptr, nullptr, nullptr, nullptr};
    return aumisart_host(ctx, h_outimg, h_outproj, h_outnorm, out, h_img, h_proj, nx, ny, nz, na,
                         nb, outIter, n_views, n_iter, op_iter, da, db, ai, bi, SO, SD, dx, lambda,
                         volumes, flows, err_weights, angles, ax, ay, az, bx, by, bz);
}

MC_EXPORT int mcsart_aumisart_fields(mcsart_ctx *ctx, float *h_outimg, float *h_outproj,
                                     float *h_outnorm, float *h_out_ax, float *h_out_ay,
                                     float *h_out_az, float *h_out_bx, float *h_out_by,
                                     float *h_out_bz, const float *h_img, const float *h_proj,
                                     int nx, int ny, int nz, int na, int nb, int outIter,
                                     int n_views, int n_iter, const int *op_iter, float da,
                                     float db, float ai, float bi, float SO, float SD, float dx,
                                     float lambda, const float *volumes, const float *flows,
                                     const float *err_weights, const float *angles,
                                     const float *ax, const float *ay, const float *az,
                                     const float *bx, const float *by, const float *bz) {
    float *const out[6] = {h_out_ax, h_out_ay, h_out_az, h_out_bx, h_out_by, h_out_bz};
    return aumisart_host(ctx, h_outimg, h_outproj, h_outnorm, out, h_img, h_proj, nx, ny, nz, na,
                         nb, outIter, n_views, n_iter, op_iter, da, db, ai, bi, SO, SD, dx, lambda,
                         volumes, flows, err_weights, angles, ax, ay, az, bx, by, bz);
}
