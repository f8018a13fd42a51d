// Device-resident SART / motion driver state (the replacement of
// host_AUMISART, src/AUMISART.cu:3-313).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace mcsart {

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    int ensure(size_t n);  // grow (contents undefined)
    void release();
    ~DevBuf() { release(); }
    template <typename T> T *as() const { return (T *)ptr; }
};

struct PassGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<uint8_t> key;
    long long kernels = 0;  // kernel nodes per replay
    void release();
    ~PassGraph() { release(); }
};

// One reconstruction problem as the driver sees it.
struct Problem {
    Geom g;
    int n_views;
    float lambda;
    const float *angles, *volumes, *flows;  // host, n_views each
    float *img;                             // device, FP32
    const void *proj;                       // device, storage type, n_views*na*nb
    void *fields;                           // device, storage type, 6 volumes
    bool motion_model;                      // overload 2
    float *resid;                           // device FP32 or nullptr
};

// Which volume copies the projector reads for a view (abi_kernels.cu):
// any_x: some rays are x-driven (the y-fastest copy), any_y: some are
// y-driven (the x-fastest volume).
void view_drive_axes(float angle, const Geom &g, bool *any_x, bool *any_y);

// Runs n_iter passes of host_AUMISART's loop (sart.cu).
int run_driver(mcsart_ctx *ctx, const Problem &P, int n_iter, const int *op_iter, float *norm_out,
               const mcsart_options &opt);

// Tuning cache key of a geometry and storage type, and the tuned launch
// shapes for it (the built-in choices where none are cached) (tuning.cu).
std::string tuning_key(const Geom &g, int storage);
Tuning tuning_for(const mcsart_ctx *ctx, const Geom &g, int storage);
// Times the variants of the driver's kernels on a sample of P's views and
// caches the fastest for P's geometry (tuning.cu).
int autotune_problem(mcsart_ctx *ctx, const Problem &P, const mcsart_options &opt);

struct DriverState {
    // working volumes of the passes
    DevBuf img1, img1T, imgS, imgST, img0, img0T, ones, onesT, ratio, imgT;
    DevBuf pairs, norm_part, norm_tmp, views_image, views_motion, zero_fields;
    DevBuf bpcolA, bpcolB;  // one view's backprojector column data (projector output)
    // staging for the host-pointer entry point
    DevBuf h_img, h_proj, h_fields, h_resid, h_norm;
    // 3D arrays sampled by the texture unit (INTERP_TEXTURE): the volume and
    // the normalised correction of the image pass, and mcsart_deform's source
    TexVol tv_img, tv_ratio, tv_deform;
    // ordered subsets (options.subset > 1): the corrections of views 2.. of a
    // subset, and the views' angles on the device
    TexVol tv_ratio_sub[15];
    DevBuf angles_dev;
    // options.dvf_inverse > 0: a view's forward displacement and its inverse
    DevBuf m3, inv3;
    std::map<int, PassGraph> graphs;  // keyed by pass kind
    void invalidate_graphs() { graphs.clear(); }
};

}  // namespace mcsart
