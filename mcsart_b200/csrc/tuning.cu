// Autotuner of the driver's launch shapes, cached per geometry.
//
// The per-view kernels of the SART/motion loop have launch shapes whose best
// choice depends on the problem's size: how many detector rays and voxels one
// view gives against the GPU's 148 SMs, and so how full the last wave is and
// whether a deeper (more register-hungry) slab pipeline costs occupancy.  The
// candidates of each kernel (the variant tables below) compute every ray and
// voxel with the same operations in the same order, so a tuned run is
// bitwise the same as an untuned one; only the time differs.
//
// mcsart_autotune times every candidate on a sample of the problem's own
// views (an image pass and a DVF-update pass over up to 12 views spread over
// the scan, on copies of the volume and fields), twice, and keeps the fastest
// per kernel in the context's cache under the key of the geometry and
// storage type.  The driver then uses the cached shapes for that geometry;
// mcsart_tuning_save / mcsart_tuning_load keep the cache in a text file.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <vector>

#include "common.cuh"
#include "sart.cuh"

#define MC_EXPORT extern "C" __attribute__((visibility("default")))

namespace mcsart {

// Variant counts of each kernel class (the launches are in sart.cu's Runner):
//   fp1  one-volume projector   (slab-group depth, resident blocks per SM)
//                               0: (2, 6)  1: (4, 4)  2: (1, 8)  3: (2, 7)  4: (4, 5)
//   fp3  three-volume projector 0: (4, 4)  1: (2, 4)  2: (2, 5)  3: (4, 5)
//   bp   backprojector          0: 2 voxels/thread, 4 rows      1: 1 voxel, 4 rows
//                               2: 2 voxels, 8 rows             3: 4 voxels, 4 rows
//   warp image-pass warps       0: 2 rows/thread  1: 1 row  2: 4 rows
//   fup  DVF-pass field update  0: with the backprojection ratio computed in it
//                               (square slices, FP32 geometry; else as 2)
//                               1: after a backprojector launch, fields loaded first
//                               2: after a backprojector launch, voxel by voxel
constexpr int N_FP1 = 5, N_FP3 = 4, N_BP = 4, N_WARP = 3, N_FUP = 3;

std::string tuning_key(const Geom &g, int storage) {
    char b[256];
    // floats in hexadecimal: the key is exact
    snprintf(b, sizeof(b), "%dx%dx%d/%dx%d/SO=%a/SD=%a/da=%a/db=%a/ai=%a/bi=%a/s%d", g.nx, g.ny,
             g.nz, g.na, g.nb, (double)g.SO, (double)g.SD, (double)g.da, (double)g.db,
             (double)g.ai, (double)g.bi, storage);
    return b;
}

Tuning tuning_for(const mcsart_ctx *ctx, const Geom &g, int storage) {
    const auto it = ctx->tuning.find(tuning_key(g, storage));
    return it == ctx->tuning.end() ? Tuning{} : it->second;
}

namespace {

// Milliseconds per launch of the profile table's entries labelled with one
// of `labels` (together), or a negative value if none ran.
double per_launch(const mcsart_ctx *ctx, std::initializer_list<const char *> labels) {
    double ms = 0.0;
    long long n = 0;
    for (const auto &e : ctx->prof_table)
        for (const char *l : labels)
            if (e.first == l) {
                ms += e.second.ms;
                n += e.second.launches;
            }
    return n > 0 ? ms / (double)n : -1.0;
}

// Milliseconds per view of the DVF pass's backprojection and field update,
// whether fused or as two launches: the time of both labels' launches over
// the number of field-update launches (the pass's last view, a separate
// backprojector and field update in every variant, counts in the sum).
double per_view_field_update(const mcsart_ctx *ctx) {
    double ms = 0.0;
    long long n = 0;
    for (const auto &e : ctx->prof_table) {
        if (e.first == "bp_field_update_prep" || e.first == "field_update_prep") {
            ms += e.second.ms;
            n += e.second.launches;
        } else if (e.first == "bp_div_motion") {
            ms += e.second.ms;
        }
    }
    return n > 0 ? ms / (double)n : -1.0;
}

}  // namespace

int autotune_problem(mcsart_ctx *ctx, const Problem &P, const mcsart_options &opt_in) {
    MC_REQUIRE(!ctx->profiling, "mcsart_autotune: not while profiling (mcsart_profile_begin)");
    const int64_t V = nvox(P.g.nx, P.g.ny, P.g.nz);
    const size_t es = opt_in.storage == MCSART_F32 ? 4 : 2;
    // a sample of views spread over the scan
    const int ns = std::min(P.n_views, 12);
    std::vector<float> ang(ns), vol(ns), flo(ns);
    for (int j = 0; j < ns; j++) {
        const int v = (int)((int64_t)j * P.n_views / ns);
        ang[j] = P.angles[v];
        vol[j] = P.volumes[v];
        flo[j] = P.flows[v];
    }
    void *img_ws = nullptr, *f_ws = nullptr;
    MC_TRY(workspace(ctx, "tune_img", V * sizeof(float), &img_ws));
    MC_TRY(workspace(ctx, "tune_fields", 6 * V * es, &f_ws));
    Problem Q = P;
    Q.n_views = ns;
    Q.angles = ang.data();
    Q.volumes = vol.data();
    Q.flows = flo.data();
    Q.img = (float *)img_ws;
    Q.fields = f_ws;
    Q.resid = nullptr;
    mcsart_options opt = opt_in;
    opt.use_graph = 0;  // profiling times each launch
    opt.autotune = 0;
    const int op[2] = {1, 0};

    const int n_trials =
        std::max(std::max(std::max(N_FP1, N_FP3), std::max(N_BP, N_WARP)), N_FUP);
    std::vector<double> best_fp1(N_FP1, 1e30), best_fp3(N_FP3, 1e30), best_bp(N_BP, 1e30),
        best_warp(N_WARP, 1e30), best_fup(N_FUP, 1e30);
    int rc = MCSART_OK;
    for (int round = 0; round < 2 && rc == MCSART_OK; round++) {
        for (int t = 0; t < n_trials && rc == MCSART_OK; t++) {
            Tuning trial;
            trial.fp1 = t % N_FP1;
            trial.fp3 = t % N_FP3;
            trial.bp = t % N_BP;
            trial.warp = t % N_WARP;
            trial.fup = t % N_FUP;
            MC_CHECK_CUDA(cudaMemcpyAsync(img_ws, P.img, V * sizeof(float),
                                          cudaMemcpyDeviceToDevice, ctx->stream));
            MC_CHECK_CUDA(cudaMemcpyAsync(f_ws, P.fields, 6 * V * es, cudaMemcpyDeviceToDevice,
                                          ctx->stream));
            ctx->tuning_override = &trial;
            rc = mcsart_profile_begin(ctx);
            if (rc == MCSART_OK) rc = run_driver(ctx, Q, 2, op, nullptr, opt);
            const int re = ctx->profiling ? mcsart_profile_end(ctx) : MCSART_OK;
            ctx->tuning_override = nullptr;
            if (rc == MCSART_OK) rc = re;
            if (rc != MCSART_OK) break;
            const double f1 = per_launch(ctx, {"fp_image"});
            const double f3 = per_launch(ctx, {"fp_motion"});
            const double b = per_launch(ctx, {"bp_div", "bp_div_add"});
            const double w = per_launch(ctx, {"warp_fwd", "warp_back_add"});
            const double u = per_view_field_update(ctx);
            if (f1 >= 0) best_fp1[trial.fp1] = std::min(best_fp1[trial.fp1], f1);
            if (f3 >= 0) best_fp3[trial.fp3] = std::min(best_fp3[trial.fp3], f3);
            if (b >= 0) best_bp[trial.bp] = std::min(best_bp[trial.bp], b);
            if (w >= 0) best_warp[trial.warp] = std::min(best_warp[trial.warp], w);
            if (u >= 0) best_fup[trial.fup] = std::min(best_fup[trial.fup], u);
        }
    }
    ctx->prof_table.clear();
    if (rc != MCSART_OK) return rc;
    auto argmin = [](const std::vector<double> &v) {
        // -1 (the built-in choice) where the kernel did not run
        const auto it = std::min_element(v.begin(), v.end());
        return *it >= 1e30 ? -1 : (int)(it - v.begin());
    };
    Tuning best;
    best.fp1 = argmin(best_fp1);
    best.fp3 = argmin(best_fp3);
    best.bp = argmin(best_bp);
    best.warp = argmin(best_warp);
    best.fup = argmin(best_fup);
    ctx->tuning[tuning_key(P.g, opt_in.storage)] = best;
    MC_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    return MCSART_OK;
}

}  // namespace mcsart

using namespace mcsart;

MC_EXPORT int mcsart_tuning_get(mcsart_ctx *ctx, const mcsart_problem *prob, int storage,
                                int *shapes) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(prob && shapes, "problem and shapes must be non-NULL");
    Geom g;
    g.SO = prob->SO; g.SD = prob->SD; g.da = prob->da; g.ai = prob->ai; g.db = prob->db;
    g.bi = prob->bi; g.na = prob->na; g.nb = prob->nb; g.nx = prob->nx; g.ny = prob->ny;
    g.nz = prob->nz;
    const auto it = ctx->tuning.find(tuning_key(g, storage));
    if (it == ctx->tuning.end()) return 0;
    shapes[0] = it->second.fp1;
    shapes[1] = it->second.fp3;
    shapes[2] = it->second.bp;
    shapes[3] = it->second.warp;
    shapes[4] = it->second.fup;
    return 1;
}

MC_EXPORT int mcsart_tuning_save(mcsart_ctx *ctx, const char *path) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(path, "path is NULL");
    FILE *f = fopen(path, "w");
    MC_REQUIRE(f, "cannot open %s for writing", path);
    fprintf(f, "# mcsart tuning cache v3: key fp1 fp3 bp warp fup\n");
    for (const auto &e : ctx->tuning)
        fprintf(f, "%s %d %d %d %d %d\n", e.first.c_str(), e.second.fp1, e.second.fp3,
                e.second.bp, e.second.warp, e.second.fup);
    const bool ok = fclose(f) == 0;
    MC_REQUIRE(ok, "writing %s failed", path);
    return MCSART_OK;
}

MC_EXPORT int mcsart_tuning_load(mcsart_ctx *ctx, const char *path) {
    clear_error();
    MC_TRY(validate_ctx(ctx));
    MC_REQUIRE(path, "path is NULL");
    FILE *f = fopen(path, "r");
    MC_REQUIRE(f, "cannot open %s", path);
    char line[512];
    int n = 0, bad = 0;
    while (fgets(line, sizeof(line), f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        char key[400];
        Tuning t;
        if (sscanf(line, "%399s %d %d %d %d %d", key, &t.fp1, &t.fp3, &t.bp, &t.warp, &t.fup) !=
                6 ||
            t.fp1 < -1 || t.fp1 >= N_FP1 || t.fp3 < -1 || t.fp3 >= N_FP3 || t.bp < -1 ||
            t.bp >= N_BP || t.warp < -1 || t.warp >= N_WARP || t.fup < -1 || t.fup >= N_FUP) {
            bad++;
            continue;
        }
        ctx->tuning[key] = t;
        n++;
    }
    fclose(f);
    MC_REQUIRE(bad == 0, "%s: %d malformed tuning entries", path, bad);
    return n;
}
