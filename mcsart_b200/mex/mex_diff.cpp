/* img1 = mex_diff(img, struct('nx',.., 'ny',.., 'nz',.., 'ind',..))
 *
 * The reference gateway (src/mex_diff.cu) on the engine: backward difference
 * along ind (1, 2 or 3), zero on both faces. */
#include <cuda_runtime.h>

#include "mcsart_mex_common.h"

static void cuda_ok(cudaError_t e) {
    if (e != cudaSuccess) mexErrMsgIdAndTxt("McSART:cuda", "%s", cudaGetErrorString(e));
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    (void)nlhs;
    if (nrhs < 2) mexErrMsgIdAndTxt("MATLAB:badInput", "mex_diff needs 2 inputs.\n");
    const mxArray *p = prhs[1];
    const int nx = mcsart_req_int(p, "nx", NULL, "Can't found valid volume resolution nx.\n");
    const int ny = mcsart_req_int(p, "ny", NULL, "Can't found valid volume resolution ny.\n");
    const int nz = mcsart_req_int(p, "nz", NULL, "Can't found valid volume resolution nz.\n");
    const int ind = mcsart_req_int(p, "ind", NULL, "Can't found ind.\n");
    mcsart_ctx *ctx = mcsart_mex_ctx();
    const size_t n = (size_t)nx * ny * nz;
    float *d_in = NULL, *d_out = NULL;
    cuda_ok(cudaMalloc((void **)&d_in, n * sizeof(float)));
    cuda_ok(cudaMalloc((void **)&d_out, n * sizeof(float)));
    cuda_ok(cudaMemcpy(d_in, mxGetData(prhs[0]), n * sizeof(float), cudaMemcpyHostToDevice));
    cuda_ok(cudaMemset(d_out, 0, n * sizeof(float)));
    const int rc = mcsart_diff(ctx, d_out, d_in, nx, ny, nz, ind);
    plhs[0] = mcsart_new_single(nx, ny, nz);
    if (rc == MCSART_OK)
        cuda_ok(cudaMemcpy(mxGetData(plhs[0]), d_out, n * sizeof(float), cudaMemcpyDeviceToHost));
    cudaFree(d_in);
    cudaFree(d_out);
    mcsart_mex_check(rc);
}
