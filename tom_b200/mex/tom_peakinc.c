/* MEX gateway tom_peakinc(stream, dims_int32, max_single, pos_int32) on the GPU.
 *
 * Same in-place outputs as the reference gateway (Analysis/tom_peakinc.c:60-77,
 * called by Analysis/tom_peakc.m:70): the first strict maximum of the single
 * volume, its value written into MAX and its 1-based position into POS_MAX.
 *
 *   mex -I<repo>/include -L<repo>/tom_b200 -ltomgpu tom_peakinc.c
 */
#include "tomgpu_mex_common.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    const int *dims;
    float *val;
    int *pos;
    (void)nlhs;
    (void)plhs;
    if (nrhs != 4) mexErrMsgTxt("4 input arguments required: stream, dims, max, pos");
    dims = (const int *)mxGetData(prhs[1]);
    val = (float *)mxGetData(prhs[2]);
    pos = (int *)mxGetData(prhs[3]);
    tomgpu_mex_check(tomgpu_peak(tomgpu_mex_ctx(), (const float *)mxGetData(prhs[0]), dims, val, pos));
}
