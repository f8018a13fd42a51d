// Test infrastructure, not product code.
//
// C-ABI harness around the UNMODIFIED reference CUDA sources of
// bill52547/McSART (src/cu_*.cu, src/AUMISART.cu, src/mex_diff.cu), which the
// recipe in oracle/Makefile compiles from the reference tree together with this
// file into oracle/_ref/libmcsart_ref.so.  Tests load that library to obtain
// outputs of the reference itself on the same GPU and inputs ("the rebuilt
// reference"), which pins both the CPU oracle and the sm_100a kernels.
//
// Every ref_* wrapper forwards to exactly one reference function with the
// reference's own argument order; nothing here changes the reference's
// arithmetic.  The MATLAB API functions the reference links against are
// provided as inert stubs (the reference only prints through them).
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

#include "AUMISART.h"
#include "cu_multiple.h"

// src/mex_diff.cu declares these at file scope (mex_diff.cu:5-6).
__host__ void host_diff(float *img1, float *img, int nx, int ny, int nz, int ind);

// ---------------------------------------------------------------- MATLAB stubs
extern "C" {
int mexPrintf(const char *fmt, ...) {
    if (!getenv("MCSART_REF_VERBOSE")) return 0;
    va_list ap;
    va_start(ap, fmt);
    int n = vfprintf(stderr, fmt, ap);
    va_end(ap);
    return n;
}
int mexEvalString(const char *) { return 0; }
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    fprintf(stderr, "[ref shim] %s: ", id);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
}
mxArray *mxGetField(const mxArray *, size_t, const char *) { return nullptr; }
double mxGetScalar(const mxArray *) { return 0.0; }
void *mxGetData(const mxArray *) { return nullptr; }
mxArray *mxCreateNumericMatrix(size_t, size_t, mxClassID, mxComplexity) { return nullptr; }
void mxSetDimensions(mxArray *, const mwSize *, size_t) {}
void mxSetData(mxArray *, void *) {}
void *mxMalloc(size_t n) { return malloc(n); }
}  // extern "C"

// ------------------------------------------------------------- device memory
extern "C" {
void *ref_malloc(size_t bytes) {
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    return p;
}
int ref_free(void *p) { return (int)cudaFree(p); }
int ref_h2d(void *d, const void *h, size_t bytes) {
    return (int)cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice);
}
int ref_d2h(void *h, const void *d, size_t bytes) {
    return (int)cudaMemcpy(h, d, bytes, cudaMemcpyDeviceToHost);
}
int ref_sync(void) { return (int)cudaDeviceSynchronize(); }
int ref_last_error(void) { return (int)cudaGetLastError(); }

// ------------------------------------------------------- reference launchers
// src/cu_projection.cu:7
void ref_projection(float *d_proj, float *d_img, float angle, float SO, float SD,
                    float da, int na, float ai, float db, int nb, float bi,
                    int nx, int ny, int nz) {
    host_projection(d_proj, d_img, angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz);
}
// src/cu_backprojection.cu:8
void ref_backprojection(float *d_img, float *d_proj, float angle, float SO, float SD,
                        float da, int na, float ai, float db, int nb, float bi,
                        int nx, int ny, int nz) {
    host_backprojection(d_img, d_proj, angle, SO, SD, da, na, ai, db, nb, bi, nx, ny, nz);
}
// src/cu_deform.cu:3
void ref_deform(float *d_img1, float *d_img, int nx, int ny, int nz, float volume,
                float flow, float *ax, float *ay, float *az, float *bx, float *by,
                float *bz) {
    host_deform(d_img1, d_img, nx, ny, nz, volume, flow, ax, ay, az, bx, by, bz);
}
// src/cu_deform.cu:49
void ref_deform2(float *d_img1, float *d_img, int nx, int ny, int nz, float volume,
                 float flow, float *ax, float *ay, float *az, float *bx, float *by,
                 float *bz) {
    host_deform2(d_img1, d_img, nx, ny, nz, volume, flow, ax, ay, az, bx, by, bz);
}
// src/cu_deform.cu:66, launched with the grid host_deform uses (cu_deform.cu:5-6,11)
void ref_forward_dvf(float *mx, float *my, float *mz, float *ax, float *ay, float *az,
                     float *bx, float *by, float *bz, float volume, float flow, int nx,
                     int ny, int nz) {
    const dim3 grid((nx + BLOCKSIZE_X - 1) / BLOCKSIZE_X, (ny + BLOCKSIZE_Y - 1) / BLOCKSIZE_Y,
                    (nz + BLOCKSIZE_Z - 1) / BLOCKSIZE_Z);
    const dim3 block(BLOCKSIZE_X, BLOCKSIZE_Y, BLOCKSIZE_Z);
    kernel_forwardDVF<<<grid, block>>>(mx, my, mz, ax, ay, az, bx, by, bz, volume, flow, nx,
                                       ny, nz);
    cudaDeviceSynchronize();
}
// src/cu_add.cu:2, :20
void ref_add(float *img1, float *img, int nx, int ny, int nz, float weight) {
    host_add(img1, img, nx, ny, nz, weight);
}
void ref_add2(float *img1, float *img, int nx, int ny, int nz, float *img0, float weight,
              int ind) {
    host_add2(img1, img, nx, ny, nz, img0, weight, ind);
}
// src/cu_initial.cu:2, :20
void ref_initial(float *img, int nx, int ny, int nz, float value) {
    host_initial(img, nx, ny, nz, value);
}
void ref_initial2(float *img, int nx, int ny, int nz, float *img0, float volume, float flow) {
    host_initial2(img, nx, ny, nz, img0, volume, flow);
}
// src/cu_division.cu:2
void ref_division(float *img1, float *img, int nx, int ny, int nz) {
    host_division(img1, img, nx, ny, nz);
}
// src/cu_multiple.cu:2
void ref_multiple(float *img1, int nx, int ny, int nz, float *img0, float weight, int ind) {
    host_multiple(img1, nx, ny, nz, img0, weight, ind);
}
// src/cu_update_udvf.cu:3
void ref_update_udvf(float *ax, float *ay, float *az, float *bx, float *by, float *bz,
                     float *img, float *img0, float volume_diff, float flow_diff, int nx,
                     int ny, int nz, int iter) {
    host_update_udvf(ax, ay, az, bx, by, bz, img, img0, volume_diff, flow_diff, nx, ny, nz,
                     iter);
}
// src/mex_diff.cu:67
void ref_diff(float *img1, float *img, int nx, int ny, int nz, int ind) {
    host_diff(img1, img, nx, ny, nz, ind);
}
// src/AUMISART.cu:3 (overload 1: DVF zero-initialised).  Host pointers.
// Ends in cudaDeviceReset(), so callers must not share the process's CUDA
// context with anything else.
void ref_aumisart1(float *h_outimg, float *h_outproj, float *h_outnorm, float *h_outalphax,
                   float *h_img, float *h_proj, int nx, int ny, int nz, int na, int nb,
                   int outIter, int n_views, int n_iter, int *op_iter, float da, float db,
                   float ai, float bi, float SO, float SD, float dx, float lambda,
                   float *volumes, float *flows, float *err_weights, float *angles) {
    host_AUMISART(h_outimg, h_outproj, h_outnorm, h_outalphax, h_img, h_proj, nx, ny, nz, na,
                  nb, outIter, n_views, n_iter, op_iter, da, db, ai, bi, SO, SD, dx, lambda,
                  volumes, flows, err_weights, angles);
}
// src/AUMISART.cu:143 (overload 2: DVF supplied).  Same caveat as above.
void ref_aumisart2(float *h_outimg, float *h_outproj, float *h_outnorm, float *h_outalphax,
                   float *h_img, float *h_proj, int nx, int ny, int nz, int na, int nb,
                   int outIter, int n_views, int n_iter, int *op_iter, float da, float db,
                   float ai, float bi, float SO, float SD, float dx, float lambda,
                   float *volumes, float *flows, float *err_weights, float *angles, float *ax,
                   float *ay, float *az, float *bx, float *by, float *bz) {
    host_AUMISART(h_outimg, h_outproj, h_outnorm, h_outalphax, h_img, h_proj, nx, ny, nz, na,
                  nb, outIter, n_views, n_iter, op_iter, da, db, ai, bi, SO, SD, dx, lambda,
                  volumes, flows, err_weights, angles, ax, ay, az, bx, by, bz);
}
}  // extern "C"
