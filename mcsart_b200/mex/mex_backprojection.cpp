/* img = mex_backprojection(proj, geo_para)  (geo_para.angle in radians)
 *
 * The reference gateway (src/mex_backprojection.cu) on the engine. */
#include <cuda_runtime.h>

#include "mcsart_mex_common.h"

static void cuda_ok(cudaError_t e) {
    if (e != cudaSuccess) mexErrMsgIdAndTxt("McSART:cuda", "%s", cudaGetErrorString(e));
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    (void)nlhs;
    if (nrhs < 2) mexErrMsgIdAndTxt("MATLAB:badInput", "mex_backprojection needs 2 inputs.\n");
    const mcsart_mex_geo g = mcsart_parse_geo(prhs[1]);
    const float angle = mcsart_req_float(prhs[1], "angle", NULL,
                                         "Can't found valid projection angle, which is denoted with para.angle.\n");
    mcsart_ctx *ctx = mcsart_mex_ctx();
    const size_t nimg = (size_t)g.nx * g.ny * g.nz, nproj = (size_t)g.na * g.nb;
    float *d_img = NULL, *d_proj = NULL;
    cuda_ok(cudaMalloc((void **)&d_img, nimg * sizeof(float)));
    cuda_ok(cudaMalloc((void **)&d_proj, nproj * sizeof(float)));
    cuda_ok(cudaMemcpy(d_proj, mxGetData(prhs[0]), nproj * sizeof(float), cudaMemcpyHostToDevice));
    const int rc = mcsart_backprojection(ctx, d_img, d_proj, angle, g.SO, g.SD, g.da, g.na, g.ai,
                                         g.db, g.nb, g.bi, g.nx, g.ny, g.nz);
    plhs[0] = mcsart_new_single(g.nx, g.ny, g.nz);
    if (rc == MCSART_OK)
        cuda_ok(cudaMemcpy(mxGetData(plhs[0]), d_img, nimg * sizeof(float), cudaMemcpyDeviceToHost));
    cudaFree(d_img);
    cudaFree(d_proj);
    mcsart_mex_check(rc);
}
