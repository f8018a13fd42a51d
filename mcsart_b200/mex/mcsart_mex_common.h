/* Shared helpers of the MATLAB gateways built on libmcsart.
 *
 * Field lookup with the reference's aliases, defaults and error messages
 * (src/entry_AUMISART.cu:18-160, src/mex_backprojection.cu:14-108,
 * src/mex_diff.cu:17-37), written as small table-free helpers so that every
 * gateway parses its structs the same way.  One engine context is kept for
 * the life of the MEX file (the reference resets the device after every call,
 * src/AUMISART.cu:140,312). */
#ifndef MCSART_MEX_COMMON_H
#define MCSART_MEX_COMMON_H

#include "mex.h"
#include "mcsart.h"

static mcsart_ctx *g_mcsart_ctx = NULL;

static void mcsart_mex_release(void) {
    if (g_mcsart_ctx) mcsart_destroy(g_mcsart_ctx);
    g_mcsart_ctx = NULL;
}

static mcsart_ctx *mcsart_mex_ctx(void) {
    if (!g_mcsart_ctx) {
        if (mcsart_create(&g_mcsart_ctx, 0) != MCSART_OK)
            mexErrMsgIdAndTxt("McSART:engine", "%s", mcsart_last_error());
        mcsart_set_synchronous(g_mcsart_ctx, 1);
        mexAtExit(mcsart_mex_release);
    }
    return g_mcsart_ctx;
}

static void mcsart_mex_check(int rc) {
    if (rc != MCSART_OK) mexErrMsgIdAndTxt("McSART:engine", "%s", mcsart_last_error());
}

/* First present field among up to two names, or NULL. */
static const mxArray *mcsart_field(const mxArray *s, const char *a, const char *b) {
    const mxArray *f = mxGetField(s, 0, a);
    if (!f && b) f = mxGetField(s, 0, b);
    return f;
}

static int mcsart_req_int(const mxArray *s, const char *a, const char *b, const char *msg) {
    const mxArray *f = mcsart_field(s, a, b);
    if (!f) mexErrMsgIdAndTxt("MATLAB:badInput", "%s", msg);
    return (int)mxGetScalar(f);
}

static float mcsart_req_float(const mxArray *s, const char *a, const char *b, const char *msg) {
    const mxArray *f = mcsart_field(s, a, b);
    if (!f) mexErrMsgIdAndTxt("MATLAB:badInput", "%s", msg);
    return (float)mxGetScalar(f);
}

static float mcsart_opt_float(const mxArray *s, const char *a, float dflt) {
    const mxArray *f = mxGetField(s, 0, a);
    if (!f) {
        mexPrintf("Automatically set %s to %g.\n", a, (double)dflt);
        return dflt;
    }
    return (float)mxGetScalar(f);
}

/* Geometry in voxel units with the detector offsets shifted to the first
 * cell's centre (src/entry_AUMISART.cu:76-94). */
typedef struct {
    int nx, ny, nz, na, nb;
    float dx, da, db, ai, bi, SO, SD;
} mcsart_mex_geo;

static mcsart_mex_geo mcsart_parse_geo(const mxArray *g) {
    mcsart_mex_geo o;
    o.nx = mcsart_req_int(g, "nx", NULL, "Can't found valid volume resolution nx.\n");
    o.ny = mcsart_req_int(g, "ny", NULL, "Can't found valid volume resolution ny.\n");
    o.nz = mcsart_req_int(g, "nz", NULL, "Can't found valid volume resolution nz.\n");
    o.na = mcsart_req_int(g, "na", "nv",
                          "Can't found valid number of detector in plane, which is denoted as na or nu.\n");
    o.nb = mcsart_req_int(g, "nb", "nu",
                          "Can't found valid number of detector across plane, which is denoted as nb or nv.\n");
    o.dx = mcsart_opt_float(g, "dx", 1.0f);
    o.da = mcsart_opt_float(g, "da", 1.0f);
    o.db = mcsart_opt_float(g, "db", 1.0f);
    o.ai = mcsart_opt_float(g, "ai", 0.0f) - ((float)o.na / 2 - 0.5f);
    o.bi = mcsart_opt_float(g, "bi", 0.0f) - ((float)o.nb / 2 - 0.5f);
    o.SO = mcsart_req_float(g, "SO", "SI",
                            "Can't found valid distance between source and isocenter, which is denoted with para.SO or para.DI.\n");
    if (mxGetField(g, 0, "SD"))
        o.SD = (float)mxGetScalar(mxGetField(g, 0, "SD"));
    else if (mxGetField(g, 0, "DI"))
        o.SD = (float)mxGetScalar(mxGetField(g, 0, "DI")) + o.SO;
    else
        mexErrMsgIdAndTxt("MATLAB:badInput",
                          "Can't found valid distance between source and detector plane, which is denoted with para.SD or para.SI + para.DI.\n");
    return o;
}

static mxArray *mcsart_new_single(int a, int b, int c) {
    const mwSize dims[3] = {(mwSize)a, (mwSize)b, (mwSize)c};
    mxArray *m = mxCreateNumericMatrix(0, 0, mxSINGLE_CLASS, mxREAL);
    mxSetDimensions(m, dims, 3);
    mxSetData(m, mxMalloc((size_t)a * b * c * sizeof(float)));
    return m;
}

#endif
