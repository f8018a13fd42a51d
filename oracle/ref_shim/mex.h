/* Minimal stand-in for MATLAB's mex.h so that the reference CUDA sources
 * (which include it through include/universal.h) compile outside MATLAB.
 * Test infrastructure only: used to rebuild the reference as oracle/_ref. */
#ifndef MCSART_REF_SHIM_MEX_H
#define MCSART_REF_SHIM_MEX_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct mcsart_shim_mxArray mxArray;
typedef size_t mwSize;
typedef enum { mxSINGLE_CLASS = 7 } mxClassID;
typedef enum { mxREAL = 0 } mxComplexity;
int mexPrintf(const char *fmt, ...);
int mexEvalString(const char *cmd);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
mxArray *mxGetField(const mxArray *a, size_t index, const char *name);
double mxGetScalar(const mxArray *a);
void *mxGetData(const mxArray *a);
mxArray *mxCreateNumericMatrix(size_t m, size_t n, mxClassID c, mxComplexity x);
void mxSetDimensions(mxArray *a, const mwSize *dims, size_t ndim);
void mxSetData(mxArray *a, void *data);
void *mxMalloc(size_t n);
#ifdef __cplusplus
}
#endif
#endif
