/* Minimal stand-in for MATLAB's matrix.h (see mex.h in this folder).
 * Test infrastructure only; no function here is ever reached. */
#ifndef ORACLE_STUB_MATRIX_H
#define ORACLE_STUB_MATRIX_H
#include <stdlib.h>

typedef struct mxArray_tag mxArray;
typedef enum { mxUNKNOWN_CLASS = 0, mxSINGLE_CLASS = 7 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;

static void *mxGetData(const mxArray *a) { (void)a; abort(); return 0; }
static const int *mxGetDimensions(const mxArray *a) { (void)a; abort(); return 0; }
static int mxGetNumberOfDimensions(const mxArray *a) { (void)a; abort(); return 0; }
static int mxIsSingle(const mxArray *a) { (void)a; abort(); return 0; }
static char *mxArrayToString(const mxArray *a) { (void)a; abort(); return 0; }
static mxArray *mxCreateNumericArray(int n, const int *d, mxClassID c, mxComplexity x)
{ (void)n; (void)d; (void)c; (void)x; abort(); return 0; }
#endif
