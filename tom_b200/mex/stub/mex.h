/* Declarations of the MATLAB MEX API used by the gateways in this folder, for
 * compile checks where MATLAB is not installed.  A real build uses MATLAB's
 * own mex.h via the `mex` command (see the build line in each gateway). */
#ifndef TOMGPU_STUB_MEX_H
#define TOMGPU_STUB_MEX_H
#include <stddef.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxUNKNOWN_CLASS = 0, mxDOUBLE_CLASS = 6, mxSINGLE_CLASS = 7, mxINT32_CLASS = 12 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;
void *mxGetData(const mxArray *a);
const mwSize *mxGetDimensions(const mxArray *a);
mwSize mxGetNumberOfDimensions(const mxArray *a);
mwSize mxGetNumberOfElements(const mxArray *a);
mwSize mxGetM(const mxArray *a);
mwSize mxGetN(const mxArray *a);
int mxIsSingle(const mxArray *a);
int mxIsDouble(const mxArray *a);
int mxIsInt32(const mxArray *a);
int mxIsEmpty(const mxArray *a);
char *mxArrayToString(const mxArray *a);
void mxFree(void *p);
mxArray *mxCreateNumericArray(mwSize n, const mwSize *d, mxClassID c, mxComplexity x);
void mexErrMsgTxt(const char *m);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
#endif
