/* MEX gateway w = tom_calc_weight_functioninc(dims, angles', thickness) on the GPU.
 *
 * Same inputs and single output as the reference's 3-D branch
 * (Filtrans/tom_calc_weight_functioninc.c:259-289): dims as doubles, angles
 * 2 x n_tilt degrees (phi; theta), thickness double.
 *
 *   mex -I<repo>/include -L<repo>/tom_b200 -ltomgpu tom_calc_weight_functioninc.c
 */
#include "tomgpu_mex_common.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    const double *h;
    int dims[3];
    mwSize md[3];
    (void)nlhs;
    if (nrhs < 3) mexErrMsgTxt("3 input arguments required: dims, angles, thickness");
    h = (const double *)mxGetData(prhs[0]);
    if (mxGetNumberOfElements(prhs[0]) != 3) mexErrMsgTxt("only the 3-D weighting runs on the GPU");
    dims[0] = (int)h[0];
    dims[1] = (int)h[1];
    dims[2] = (int)h[2];
    md[0] = dims[0];
    md[1] = dims[1];
    md[2] = dims[2];
    plhs[0] = mxCreateNumericArray(3, md, mxSINGLE_CLASS, mxREAL);
    tomgpu_mex_check(tomgpu_weight3d(tomgpu_mex_ctx(), dims, (const double *)mxGetData(prhs[1]),
                                     (int)mxGetN(prhs[1]), *(const double *)mxGetData(prhs[2]),
                                     (float *)mxGetData(plhs[0])));
}
