/* MEX gateway [ccc, angles] = tom_os3_match(volume, template, mask, psf, angleList)
 * on the GPU: the whole angle loop of tom_os3_findTemplate
 * (Oscar3/matlabPicker/search/tom_os3_findTemplate.m:255-307) in one call.
 *
 * volume, template, mask: single; psf: single template-sized weight or [] for
 * none; angleList: R x 3 single [phi psi theta] in degrees.  The template is
 * preprocessed like findTemplate (:157, :233-234).  Outputs follow the
 * reference: ccc single (-1000 where never updated) and angles single holding
 * the 1-based angle-list index (-1000 where never updated).
 *
 *   mex -I<repo>/include -L<repo>/tom_b200 -ltomgpu tom_os3_match.c
 */
#include <stdlib.h>
#include "tomgpu_mex_common.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    int dv[3], dt[3];
    mwSize md[3];
    const float *ang;
    float *eul, *ccc, *angles;
    int32_t *idx;
    mwSize R, i, n;
    int rc;
    if (nrhs != 5) mexErrMsgTxt("5 inputs: volume, template, mask, psf, angleList");
    if (!mxIsSingle(prhs[0]) || !mxIsSingle(prhs[1]) || !mxIsSingle(prhs[2]) || !mxIsSingle(prhs[4]))
        mexErrMsgTxt("volume, template, mask and angleList must be single");
    tomgpu_mex_dims3(prhs[0], dv);
    tomgpu_mex_dims3(prhs[1], dt);
    R = mxGetM(prhs[4]);
    if (mxGetN(prhs[4]) != 3) mexErrMsgTxt("angleList must be R x 3");
    ang = (const float *)mxGetData(prhs[4]);
    eul = (float *)malloc(sizeof(float) * 3 * (R ? R : 1));
    for (i = 0; i < R; ++i) { /* column-major R x 3 -> row triplets */
        eul[3 * i] = ang[i];
        eul[3 * i + 1] = ang[i + R];
        eul[3 * i + 2] = ang[i + 2 * R];
    }
    md[0] = dv[0];
    md[1] = dv[1];
    md[2] = dv[2];
    n = md[0] * md[1] * md[2];
    plhs[0] = mxCreateNumericArray(3, md, mxSINGLE_CLASS, mxREAL);
    plhs[1] = mxCreateNumericArray(3, md, mxSINGLE_CLASS, mxREAL);
    ccc = (float *)mxGetData(plhs[0]);
    angles = (float *)mxGetData(plhs[1]);
    idx = (int32_t *)malloc(sizeof(int32_t) * n);
    rc = tomgpu_match(tomgpu_mex_ctx(), (const float *)mxGetData(prhs[0]), dv, (const float *)mxGetData(prhs[1]),
                      dt, (const float *)mxGetData(prhs[2]),
                      mxIsEmpty(prhs[3]) ? 0 : (const float *)mxGetData(prhs[3]), eul, (int)R, 0, ccc, idx);
    free(eul);
    if (rc == TOMGPU_OK)
        for (i = 0; i < n; ++i) angles[i] = idx[i] >= 0 ? (float)(idx[i] + 1) : -1000.0f;
    free(idx);
    (void)nlhs;
    tomgpu_mex_check(rc);
}
