/* Test infrastructure: declarations of the MATLAB MEX API used by the
 * gateways in mcsart_b200/mex, so that they can be compile-checked where
 * MATLAB is not installed.  Nothing here is linked or run. */
#ifndef MCSART_TEST_MEX_SHIM_H
#define MCSART_TEST_MEX_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct mcsart_test_mxArray mxArray;
typedef size_t mwSize;
typedef enum { mxSINGLE_CLASS = 7 } mxClassID;
typedef enum { mxREAL = 0 } mxComplexity;
int mexPrintf(const char *fmt, ...);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
int mexAtExit(void (*fn)(void));
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
