/* Shared helpers of the tomgpu MEX gateways: one lazily created context per
 * MATLAB session, and the conversion of tomgpu status codes into MATLAB
 * errors (mexErrMsgTxt), the reference gateways' error behaviour. */
#ifndef TOMGPU_MEX_COMMON_H
#define TOMGPU_MEX_COMMON_H
#include "mex.h"
#include "tomgpu.h"

static inline tomgpu_ctx *tomgpu_mex_ctx(void)
{
    static tomgpu_ctx *ctx = 0;
    if (!ctx && tomgpu_ctx_create(0, &ctx) != TOMGPU_OK)
        mexErrMsgTxt(tomgpu_last_error(0));
    return ctx;
}

static inline void tomgpu_mex_check(int status)
{
    if (status != TOMGPU_OK) mexErrMsgTxt(tomgpu_last_error(tomgpu_mex_ctx()));
}

static inline void tomgpu_mex_dims3(const mxArray *a, int d[3])
{
    const mwSize *s = mxGetDimensions(a);
    mwSize n = mxGetNumberOfDimensions(a);
    d[0] = (int)s[0];
    d[1] = n > 1 ? (int)s[1] : 1;
    d[2] = n > 2 ? (int)s[2] : 1;
}
#endif
