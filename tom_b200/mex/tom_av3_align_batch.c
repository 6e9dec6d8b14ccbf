/* MEX gateway of subtomogram alignment on the GPU, one particle or many:
 *
 *   [angles, shifts, ccf_peak] = tom_av3_align_batch(ref, part, phi, psi, theta,
 *                                                    mask, mask_ccf, wedge_ref, wedge_part)
 *
 * The first three outputs of tom_av3_align (av3_new/tom_av3_align.m:97-189)
 * with filter.Apply = 0, for every particle: the scan, the angle of the first
 * maximum of ccf_max .* mask_ccf, and the spline peak of one more tom_corr at
 * that angle.  The computation runs in tomgpu_av3_align (the particles of a
 * box edge batched together).
 *
 *   ref        a volume (single or double), shared by all particles, or a
 *              cell array with one per particle
 *   part       a volume or a cell array of volumes (one per particle)
 *   phi, psi, theta
 *              [start increment end] in degrees: 1 x 3 for all particles, or
 *              n x 3 with a row per particle
 *   mask       a volume (shared) or a cell array, or [] for
 *              tom_spheremask(ones(size(part)))
 *   mask_ccf   a volume, a cell array or [] (ones)
 *   wedge_ref  a volume, a cell array or [] (the form without wedges)
 *   wedge_part a volume, a cell array or [] (wedge_ref)
 *
 * angles and shifts are 3 x n, ccf_peak 1 x n (double).  Errors end in
 * mexErrMsgTxt.  A loop of tom_av3_align calls over the particles of an
 * iteration (as in av3_tomomatch) becomes one call of this gateway.
 *
 *   mex -I<repo>/include -L<repo>/tom_b200 -ltomgpu tom_av3_align_batch.c
 */
#include <math.h>
#include <string.h>

#include "tomgpu_mex_common.h"

/* Converted inputs: one float copy per distinct mxArray (kept in a small
 * table so that an array shared by the particles is converted once). */
typedef struct {
    const mxArray *src;
    float *data;
} Conv;

static Conv *g_conv;
static int g_nconv, g_cap;

static void fail(const char *msg)
{
    g_conv = 0;
    g_nconv = g_cap = 0;
    mexErrMsgTxt(msg);
}

/* the float data of a real single or double volume (single: MATLAB's own
 * buffer; double: a converted copy, made once per array) */
static const float *as_float(const mxArray *a)
{
    int i;
    mwSize n, k;
    float *f;
    if (mxIsSingle(a)) return (const float *)mxGetData(a);
    if (!mxIsDouble(a) || mxIsComplex(a)) fail("tom_av3_align_batch: volumes must be real single or double");
    for (i = 0; i < g_nconv; ++i)
        if (g_conv[i].src == a) return g_conv[i].data;
    if (g_nconv == g_cap) {
        int cap = g_cap ? 2 * g_cap : 16;
        g_conv = (Conv *)(g_conv ? mxRealloc(g_conv, sizeof(Conv) * cap) : mxMalloc(sizeof(Conv) * cap));
        g_cap = cap;
    }
    n = mxGetNumberOfElements(a);
    f = (float *)mxMalloc(sizeof(float) * (n ? n : 1));
    for (k = 0; k < n; ++k) f[k] = (float)mxGetPr(a)[k];
    g_conv[g_nconv].src = a;
    g_conv[g_nconv].data = f;
    ++g_nconv;
    return f;
}

/* entry i of an argument that is either one array for all or a cell array */
static const mxArray *nth(const mxArray *a, mwSize i)
{
    if (!a || mxIsEmpty(a)) return 0;
    if (mxIsCell(a)) return mxGetCell(a, i);
    return a;
}

static mwSize count_of(const mxArray *a)
{
    return a && mxIsCell(a) ? mxGetNumberOfElements(a) : 0;
}

/* tom_spheremask(ones(n)): 1 where the distance from floor(n/2) + 1 (1-based)
 * is below floor((min(n) - 1) / 2) (Geom/tom_spheremask.m:41-67) */
static float *default_mask(const int d[3])
{
    const double r = floor(((d[0] < d[1] ? (d[0] < d[2] ? d[0] : d[2]) : (d[1] < d[2] ? d[1] : d[2])) - 1) / 2.0);
    float *m = (float *)mxMalloc(sizeof(float) * (size_t)d[0] * d[1] * d[2]);
    int x, y, z;
    for (z = 0; z < d[2]; ++z)
        for (y = 0; y < d[1]; ++y)
            for (x = 0; x < d[0]; ++x) {
                const double dx = x + 1 - (floor(d[0] / 2.0) + 1), dy = y + 1 - (floor(d[1] / 2.0) + 1),
                             dz = z + 1 - (floor(d[2] / 2.0) + 1);
                m[x + (size_t)d[0] * (y + (size_t)d[1] * z)] = sqrt(dx * dx + dy * dy + dz * dz) < r ? 1.f : 0.f;
            }
    return m;
}

static void angle_range(const mxArray *a, mwSize i, mwSize n, float out[3], const char *name)
{
    const mwSize m = mxGetM(a);
    int k;
    if (!mxIsDouble(a) && !mxIsSingle(a)) fail("tom_av3_align_batch: angle ranges must be double or single");
    if (mxGetNumberOfElements(a) == 3) {
        for (k = 0; k < 3; ++k) out[k] = mxIsDouble(a) ? (float)mxGetPr(a)[k] : ((const float *)mxGetData(a))[k];
        return;
    }
    if (m != n || mxGetN(a) != 3) {
        (void)name;
        fail("tom_av3_align_batch: an angle range is 1 x 3 or n x 3");
    }
    for (k = 0; k < 3; ++k)
        out[k] = mxIsDouble(a) ? (float)mxGetPr(a)[i + m * k] : ((const float *)mxGetData(a))[i + m * k];
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    mwSize n = 1, i;
    tomgpu_align_job *jobs;
    float *ang, *shf, *pk;
    double *oa, *os, *op;
    int k;
    /* default masks, one per box size met */
    int md[8][3];
    float *mv[8];
    int nmd = 0;
    g_conv = 0;
    g_nconv = g_cap = 0;
    if (nrhs < 5 || nrhs > 9) fail("tom_av3_align_batch: (ref, part, phi, psi, theta [, mask, mask_ccf, wedge_ref, wedge_part])");
    if (nlhs > 3) fail("tom_av3_align_batch: at most three outputs (angles, shifts, ccf_peak)");
    {
        const mwSize c[6] = {count_of(prhs[0]), count_of(prhs[1]), nrhs > 5 ? count_of(prhs[5]) : 0,
                             nrhs > 6 ? count_of(prhs[6]) : 0, nrhs > 7 ? count_of(prhs[7]) : 0,
                             nrhs > 8 ? count_of(prhs[8]) : 0};
        n = 0;
        for (k = 0; k < 6; ++k) {
            if (!c[k]) continue;
            if (n && c[k] != n) fail("tom_av3_align_batch: the cell arrays must have one entry per particle");
            n = c[k];
        }
        if (!n) n = 1;
    }
    jobs = (tomgpu_align_job *)mxCalloc(n, sizeof(tomgpu_align_job));
    for (i = 0; i < n; ++i) {
        const mxArray *r = nth(prhs[0], i), *p = nth(prhs[1], i);
        const mxArray *m = nrhs > 5 ? nth(prhs[5], i) : 0, *mc = nrhs > 6 ? nth(prhs[6], i) : 0;
        const mxArray *wr = nrhs > 7 ? nth(prhs[7], i) : 0, *wp = nrhs > 8 ? nth(prhs[8], i) : 0;
        int d[3], e[3];
        if (!r || !p) fail("tom_av3_align_batch: every particle needs a reference and a particle volume");
        tomgpu_mex_dims3(p, d);
        tomgpu_mex_dims3(r, e);
        if (d[0] != e[0] || d[1] != e[1] || d[2] != e[2]) fail("tom_av3_align_batch: reference and particle sizes differ");
        for (k = 0; k < 3; ++k) jobs[i].n[k] = d[k];
        jobs[i].ref = as_float(r);
        jobs[i].part = as_float(p);
        if (m) {
            jobs[i].mask = as_float(m);
        } else {
            int q;
            for (q = 0; q < nmd; ++q)
                if (md[q][0] == d[0] && md[q][1] == d[1] && md[q][2] == d[2]) break;
            if (q == nmd) {
                if (nmd == 8) fail("tom_av3_align_batch: pass the masks for more than eight box sizes");
                md[q][0] = d[0];
                md[q][1] = d[1];
                md[q][2] = d[2];
                mv[q] = default_mask(d);
                ++nmd;
            }
            jobs[i].mask = mv[q];
        }
        jobs[i].mask_ccf = mc ? as_float(mc) : 0;
        jobs[i].wedge_ref = wr ? as_float(wr) : 0;
        jobs[i].wedge_part = wp ? as_float(wp) : 0;
        if (!wr && wp) fail("tom_av3_align_batch: a particle wedge needs a reference wedge");
        angle_range(prhs[2], i, n, jobs[i].phi, "phi");
        angle_range(prhs[3], i, n, jobs[i].psi, "psi");
        angle_range(prhs[4], i, n, jobs[i].theta, "theta");
    }
    ang = (float *)mxMalloc(sizeof(float) * 3 * n);
    shf = (float *)mxMalloc(sizeof(float) * 3 * n);
    pk = (float *)mxMalloc(sizeof(float) * n);
    tomgpu_mex_check(tomgpu_av3_align(tomgpu_mex_ctx(), jobs, (int)n, 0, ang, shf, pk));
    plhs[0] = mxCreateNumericMatrix(3, n, mxDOUBLE_CLASS, mxREAL);
    oa = mxGetPr(plhs[0]);
    for (i = 0; i < 3 * n; ++i) oa[i] = ang[i];
    if (nlhs > 1) {
        plhs[1] = mxCreateNumericMatrix(3, n, mxDOUBLE_CLASS, mxREAL);
        os = mxGetPr(plhs[1]);
        for (i = 0; i < 3 * n; ++i) os[i] = shf[i];
    }
    if (nlhs > 2) {
        plhs[2] = mxCreateNumericMatrix(1, n, mxDOUBLE_CLASS, mxREAL);
        op = mxGetPr(plhs[2]);
        for (i = 0; i < n; ++i) op[i] = pk[i];
    }
    g_conv = 0;
    g_nconv = g_cap = 0;
}
