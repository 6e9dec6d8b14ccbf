/* MEX gateway tom_rotatec(in, out, euler, 'linear', center) on the GPU.
 *
 * Same name, inputs and in-place output as the reference gateway
 * (Sptrans/tom_rotatec.c:407-480), so Sptrans/tom_rotate.m calls it unchanged:
 * 5 inputs, 0 outputs, single volumes of equal size, euler 1x3 degrees or a
 * 3x3 matrix (chosen by its row count), centre 0-based.
 *
 *   mex -I<repo>/include -L<repo>/tom_b200 -ltomgpu tom_rotatec.c
 */
#include <string.h>
#include "tomgpu_mex_common.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    int d_in[3], d_out[3];
    char *ip;
    const mwSize *de;
    float center[3] = {0, 0, 0};
    const float *c;
    (void)plhs;
    if (nrhs != 5)
        mexErrMsgTxt("5 input arguments required.\n Syntax: rot3d(input_image,output_image,[Angle(s)],Interpolation_type,[center])");
    if (nlhs > 1) mexErrMsgTxt("Too many output arguments.");
    if (!mxIsSingle(prhs[0]) || !mxIsSingle(prhs[1])) mexErrMsgTxt("Input volumes must be single.\n");
    if (mxGetNumberOfDimensions(prhs[0]) != mxGetNumberOfDimensions(prhs[1]))
        mexErrMsgTxt("Image volumes must have same dimensions.\n");
    ip = mxArrayToString(prhs[3]);
    if (!ip || strcmp(ip, "linear") != 0)
        mexErrMsgTxt("Unknown interpolation type ... only linear interpolation implemented\n");
    mxFree(ip);
    tomgpu_mex_dims3(prhs[0], d_in);
    tomgpu_mex_dims3(prhs[1], d_out);
    if (d_in[0] != d_out[0] || d_in[1] != d_out[1] || d_in[2] != d_out[2])
        mexErrMsgTxt("Volumes must have same size.\n");
    c = (const float *)mxGetData(prhs[4]);
    center[0] = c[0];
    center[1] = c[1];
    if (mxGetNumberOfElements(prhs[4]) > 2) center[2] = c[2];
    de = mxGetDimensions(prhs[2]);
    tomgpu_mex_check(tomgpu_rotate3d(tomgpu_mex_ctx(), (const float *)mxGetData(prhs[0]),
                                     (float *)mxGetData(prhs[1]), d_in, (const float *)mxGetData(prhs[2]),
                                     de[0] == 3 ? TOMGPU_MATRIX : TOMGPU_EULER_DEG, center));
}
