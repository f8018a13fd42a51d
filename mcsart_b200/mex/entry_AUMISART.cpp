/* [img, norm, alpha_x, resid] = entry_AUMISART(img0, proj, geo_para, iter_para)
 *
 * The reference gateway (src/entry_AUMISART.cu) on the engine: same inputs,
 * struct fields, aliases, defaults and outputs; the SART/motion loop runs in
 * libmcsart (mcsart_aumisart), overload 2 when iter_para.alpha_x is present. */
#include <string.h>

#include "mcsart_mex_common.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    (void)nlhs;
    if (nrhs < 4) mexErrMsgIdAndTxt("MATLAB:badInput", "entry_AUMISART needs 4 inputs.\n");
    const mxArray *img_in = prhs[0], *proj_in = prhs[1], *geo = prhs[2], *it = prhs[3];
    const mcsart_mex_geo g = mcsart_parse_geo(geo);

    int n_iter = 1;
    if (mxGetField(it, 0, "n_iter"))
        n_iter = (int)mxGetScalar(mxGetField(it, 0, "n_iter"));
    else
        mexPrintf("Automatically set number of iterations to 1. \n");
    const mxArray *f_op = mxGetField(it, 0, "op_iter");
    if (!f_op) mexErrMsgIdAndTxt("MATLAB:badInput", "Can't found valid iteration distribution as iter_para.op_iter.\n");
    const int *op_iter = (const int *)mxGetData(f_op);
    const int n_views = mcsart_req_int(it, "n_views", NULL,
                                       "Can't found valid number bins, which is denoted as iter_para.n_views.\n");
    const float lambda = mcsart_req_float(it, "lambda", NULL, "Can't found valid coefficience iter_para.lambda.\n");
    const int outIter = mcsart_req_int(it, "outIter", NULL, "Can't found valid coefficience iter_para.outIter.\n");
    const char *arr_names[4] = {"volumes", "flows", "err_weights", "angles"};
    const char *arr_msgs[4] = {"Can't found valid volume in iter_para.volumes.\n",
                               "Can't found valid flow in iter_para.flows.\n",
                               "Can't found valid flow in iter_para.err_weights.\n",
                               "Can't found valid angles iter_para.angles.\n"};
    const float *arrs[4];
    for (int i = 0; i < 4; i++) {
        const mxArray *f = mxGetField(it, 0, arr_names[i]);
        if (!f) mexErrMsgIdAndTxt("MATLAB:badInput", "%s", arr_msgs[i]);
        arrs[i] = (const float *)mxGetData(f);
    }

    plhs[0] = mcsart_new_single(g.nx, g.ny, g.nz);
    plhs[1] = mxCreateNumericMatrix((size_t)n_iter * n_views, 1, mxSINGLE_CLASS, mxREAL);
    plhs[2] = mcsart_new_single(g.nx, g.ny, g.nz);
    plhs[3] = mcsart_new_single(g.na, g.nb, n_views);

    const float *fld[6] = {NULL, NULL, NULL, NULL, NULL, NULL};
    if (mxGetField(it, 0, "alpha_x")) {
        const char *names[6] = {"alpha_x", "alpha_y", "alpha_z", "beta_x", "beta_y", "beta_z"};
        for (int i = 0; i < 6; i++) {
            const mxArray *f = mxGetField(it, 0, names[i]);
            if (!f) mexErrMsgIdAndTxt("MATLAB:badInput", "Can't found iter_para.%s.\n", names[i]);
            fld[i] = (const float *)mxGetData(f);
        }
    }
    mcsart_mex_check(mcsart_aumisart(
        mcsart_mex_ctx(), (float *)mxGetData(plhs[0]), (float *)mxGetData(plhs[3]),
        (float *)mxGetData(plhs[1]), (float *)mxGetData(plhs[2]),
        (const float *)mxGetData(img_in), (const float *)mxGetData(proj_in), g.nx, g.ny, g.nz,
        g.na, g.nb, outIter, n_views, n_iter, op_iter, g.da, g.db, g.ai, g.bi, g.SO, g.SD, g.dx,
        lambda, arrs[0], arrs[1], arrs[2], arrs[3], fld[0], fld[1], fld[2], fld[3], fld[4],
        fld[5]));
}
