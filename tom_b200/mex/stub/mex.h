/* Declarations of the MATLAB MEX API used by the gateways in this folder, for
 * compile checks where MATLAB is not installed.  A real build uses MATLAB's
 * own mex.h via the `mex` command (see the build line in each gateway). */
#ifndef TOMGPU_STUB_MEX_H
#define TOMGPU_STUB_MEX_H
#include <stddef.h>
#include <stdint.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxUNKNOWN_CLASS = 0, mxDOUBLE_CLASS = 6, mxSINGLE_CLASS = 7, mxINT32_CLASS = 12, mxUINT32_CLASS = 13 } mxClassID;
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
int mxIsChar(const mxArray *a);
int mxIsCell(const mxArray *a);
int mxIsNumeric(const mxArray *a);
int mxIsComplex(const mxArray *a);
mxArray *mxGetCell(const mxArray *a, mwSize i);
double mxGetScalar(const mxArray *a);
double *mxGetPr(const mxArray *a);
double mxGetNaN(void);
void *mxMalloc(size_t n);
void *mxCalloc(size_t n, size_t size);
void *mxRealloc(void *p, size_t n);
mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID c, mxComplexity x);
mxArray *mxCreateStructArray(mwSize ndim, const mwSize *dims, int nfields, const char **fieldnames);
void mxSetField(mxArray *a, mwSize i, const char *field, mxArray *value);
mxArray *mxCreateString(const char *s);
void mexErrMsgTxt(const char *m);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
#endif
