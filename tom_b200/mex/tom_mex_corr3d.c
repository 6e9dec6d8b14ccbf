/* MEX gateway of the C++ picker's batched aligner on the GPU:
 *
 *   out = tom_mex_corr3d([datatype], size, templates, particles, angles, mask,
 *                        wedge_ref, wedge_part, [type], [mask_cc])
 *
 * with the argument list of Oscar3/c++Picker/src/mex/tom_mex_corr3d.cpp:53-806
 * (the reference's 'peak' type, tom::corr3d_batch with
 * CorrelationHandlerPeaks).  The computation runs in tomgpu_corr3d_peaks.
 *
 *   datatype   optional 'single' or 'double'; the GPU computes in single
 *              precision with double-precision sums either way
 *   size       3-vector of positive integers: the box size of every volume
 *   templates, particles
 *              a real volume of that size (single or double), an EM file
 *              name, or a cell array of these
 *   angles     3 x N [phi; psi; theta] in degrees
 *   mask       [] (none), a radius (tom::init_spheremask) or a volume
 *   wedge_ref, wedge_part
 *              [] (none), or one entry for all volumes, or one per volume;
 *              an entry is [] (no wedge), a scalar half-angle in degrees
 *              (SimpleWedge), an fftshifted weight volume or an EM file name
 *   type       'peak' (the default); the reference's 'cc' and 'cc2em' types
 *              are not built and end in an error
 *   mask_cc    [] or a radius or an fftshifted volume: where the peak may lie
 *
 * out is an ntemplates x nparticles struct array with the reference's
 * fields: peak (1 x 3 double, 0-based x y z), ncc_val, angle (1 x 3 degrees),
 * angle_idx (uint32, 1-based; 0 and NaN values when no angle gave a peak),
 * template and particle (the EM file name, or "template i" / "particle j").
 * Errors end in mexErrMsgTxt, as in the reference.
 *
 *   mex -I<repo>/include -L<repo>/tom_b200 -ltomgpu tom_mex_corr3d.c
 */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "tomgpu_mex_common.h"

#define MAXVOL_NAME 512

/* One input volume as float on the host. */
typedef struct {
    float *data;
    char name[MAXVOL_NAME];
} HostVol;

/* Host memory comes from mxMalloc / mxCalloc / mxRealloc: MATLAB frees it
 * when mexErrMsgTxt leaves the gateway, so an error path leaks nothing. */
static size_t g_nv;        /* voxels per volume */
static int g_dims[3];      /* box size */
static HostVol *g_vols;    /* every volume read in this call */
static int g_nvols, g_cap;

static void fail(const char *msg)
{
    g_vols = 0;
    g_nvols = g_cap = 0;
    mexErrMsgTxt(msg);
}

/* element i of a real single, double or int32 array as double */
static double num_at(const mxArray *a, mwSize i)
{
    if (mxIsDouble(a)) return mxGetPr(a)[i];
    if (mxIsSingle(a)) return (double)((const float *)mxGetData(a))[i];
    if (mxIsInt32(a)) return (double)((const int32_t *)mxGetData(a))[i];
    fail("tom_mex_corr3d: numeric parameters must be double, single or int32");
    return 0;
}

static HostVol *new_vol(void)
{
    if (g_nvols == g_cap) {
        int cap = g_cap ? 2 * g_cap : 16;
        HostVol *v = (HostVol *)(g_vols ? mxRealloc(g_vols, sizeof(HostVol) * cap) : mxMalloc(sizeof(HostVol) * cap));
        g_vols = v;
        g_cap = cap;
    }
    g_vols[g_nvols].data = (float *)mxMalloc(sizeof(float) * g_nv);
    g_vols[g_nvols].name[0] = 0;
    return &g_vols[g_nvols++];
}

static int same_size(const mxArray *a)
{
    const mwSize *d = mxGetDimensions(a);
    return mxGetNumberOfDimensions(a) == 3 && (int)d[0] == g_dims[0] && (int)d[1] == g_dims[1] &&
           (int)d[2] == g_dims[2];
}

/* A real single or double volume of the box size, or an EM file name, as
 * float; NULL when the element is neither. */
static const float *read_volume(const mxArray *el, const char *what, int index)
{
    HostVol *v;
    size_t i;
    if (mxIsChar(el)) {
        char *fn = mxArrayToString(el);
        int d[3];
        int rc;
        if (!fn) return 0;
        v = new_vol();
        rc = tomgpu_em_read(fn, d, v->data, g_nv);
        if (rc == TOMGPU_OK && (d[0] != g_dims[0] || d[1] != g_dims[1] || d[2] != g_dims[2])) rc = -1;
        snprintf(v->name, MAXVOL_NAME, "%s", fn);
        mxFree(fn);
        return rc == TOMGPU_OK ? v->data : 0;
    }
    if (!mxIsNumeric(el) || mxIsComplex(el) || !same_size(el)) return 0;
    if (!mxIsSingle(el) && !mxIsDouble(el)) return 0;
    v = new_vol();
    if (mxIsSingle(el)) {
        memcpy(v->data, mxGetData(el), sizeof(float) * g_nv);
    } else {
        const double *p = mxGetPr(el);
        for (i = 0; i < g_nv; ++i) v->data[i] = (float)p[i];
    }
    snprintf(v->name, MAXVOL_NAME, "%s %d", what, index);
    return v->data;
}

/* The elements of a volume-list argument: a cell array's cells, else the argument itself. */
static mwSize list_count(const mxArray *a) { return mxIsCell(a) ? mxGetNumberOfElements(a) : 1; }
static const mxArray *list_item(const mxArray *a, mwSize i) { return mxIsCell(a) ? mxGetCell(a, i) : a; }

/* tom::init_spheremask(mask, radius, 0, 0): 1 where the squared distance
 * from the integer centre n/2 is <= radius^2, float arithmetic
 * (Oscar3/c++Picker/src/tom/core/volume_fcn.cpp:979-1028). */
static const float *sphere_mask(double radius)
{
    HostVol *v = new_vol();
    const float r = (float)(radius > 0 ? radius : 0);
    int x, y, z;
    for (z = 0; z < g_dims[2]; ++z)
        for (y = 0; y < g_dims[1]; ++y)
            for (x = 0; x < g_dims[0]; ++x) {
                const float dx = (float)(x - g_dims[0] / 2), dy = (float)(y - g_dims[1] / 2),
                            dz = (float)(z - g_dims[2] / 2);
                const float d2 = dx * dx + (dy * dy + dz * dz);
                v->data[x + (size_t)g_dims[0] * (y + (size_t)g_dims[1] * z)] = r > 0 && d2 <= r * r ? 1.f : 0.f;
            }
    return v->data;
}

/* [] (none), a radius or a volume of the box size (MASK and MASK_CC). */
static const float *mask_arg(const mxArray *a, const char *msg)
{
    const float *m;
    if (!mxIsNumeric(a) || mxIsComplex(a)) fail(msg);
    if (mxGetNumberOfElements(a) == 0) return 0;
    if (mxGetNumberOfElements(a) == 1) return sphere_mask(mxGetScalar(a));
    m = read_volume(a, "mask", 0);
    if (!m) fail(msg);
    return m;
}

/* WEDGE_REF / WEDGE_PART: NULL for [], else count specs (one entry for all,
 * or one per volume). */
static tomgpu_wedge_spec *wedge_arg(const mxArray *a, int count, const char *which)
{
    char msg[256];
    tomgpu_wedge_spec *w;
    mwSize ne, i;
    if (mxIsNumeric(a) && mxGetNumberOfElements(a) == 0) return 0;
    if (!mxIsChar(a) && !mxIsNumeric(a) && !mxIsCell(a)) {
        snprintf(msg, sizeof msg,
                 "tom_mex_corr3d: %s must be either [] (no wedge), a scalar (angle of the wedge), a volume (the hole "
                 "weighting in fourier space, fftshifted) or a cell array of these.", which);
        fail(msg);
    }
    ne = list_count(a);
    if (ne != 1 && (int)ne != count) {
        snprintf(msg, sizeof msg,
                 "tom_mex_corr3d: The number of %s must be either 0 (none), 1 (the same wedge for all) or %d "
                 "(individual wedge)", which, count);
        fail(msg);
    }
    w = (tomgpu_wedge_spec *)mxCalloc((size_t)count, sizeof(tomgpu_wedge_spec));
    for (i = 0; i < ne; ++i) {
        const mxArray *el = list_item(a, i);
        tomgpu_wedge_spec s;
        s.kind = TOMGPU_WEDGE_NONE;
        s.angle_deg = 0.f;
        s.volume = 0;
        if (mxIsNumeric(el) && !mxIsComplex(el) && mxGetNumberOfElements(el) == 0) {
            s.kind = TOMGPU_WEDGE_NONE;
        } else if (mxIsNumeric(el) && !mxIsComplex(el) && mxGetNumberOfElements(el) == 1) {
            s.kind = TOMGPU_WEDGE_SIMPLE;
            s.angle_deg = (float)mxGetScalar(el);
        } else {
            s.kind = TOMGPU_WEDGE_VOLUME;
            s.volume = read_volume(el, "wedge", (int)i);
            if (!s.volume) {
                snprintf(msg, sizeof msg,
                         "tom_mex_corr3d: %s must be either [], angle(s) in degree, em-filename(s) or real floating "
                         "point volume(s) of size %dx%dx%d.", which, g_dims[0], g_dims[1], g_dims[2]);
                fail(msg);
            }
        }
        if (ne == 1) {
            int k;
            for (k = 0; k < count; ++k) w[k] = s;
        } else {
            w[i] = s;
        }
    }
    return w;
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    static const char *fields[6] = {"peak", "ncc_val", "angle_idx", "angle", "template", "particle"};
    char msg[256];
    const mxArray **a = prhs;
    const float **tp, **pp, *mask, *mask_cc = 0;
    tomgpu_wedge_spec *wt, *wp;
    double *ang, *peak, *val;
    int32_t *idx;
    int nt, np, nang, i, j, k, rc, first_template, first_particle;
    int narg = nrhs;
    mwSize odims[2];
    (void)nlhs;
    if (narg > 0 && mxIsChar(a[0])) {  /* the optional precision string */
        char *p = mxArrayToString(a[0]);
        const int ok = p && (!strcmp(p, "single") || !strcmp(p, "double"));
        if (p) mxFree(p);
        if (!ok)
            mexErrMsgTxt("tom_mex_corr3d: The first parameter can be (optionally) a string specifying the precision "
                         "of the computation (either 'single' or 'double').");
        ++a;
        --narg;
    }
    if (narg < 7)
        mexErrMsgTxt("tom_mex_corr3d requires arguments: [out] = tom_mex_corr3d([datatype], size, templates, "
                     "particles, angles, mask, wedge_ref, wedge_part, type, [...])");
    /* size */
    if (!mxIsNumeric(a[0]) || mxIsComplex(a[0]) || mxGetNumberOfElements(a[0]) != 3)
        mexErrMsgTxt("tom_mex_corr3d: The first parameter must be the size of the volumes (i.e. a 3-vector).");
    for (i = 0; i < 3; ++i) {
        const double d = num_at(a[0], (mwSize)i);
        if (d < 1 || d != floor(d) || d > 2147483647.0)
            mexErrMsgTxt("tom_mex_corr3d: The parameter SIZE must be the dimension of the volumes (i.e. a 3-vector "
                         "of positive integers).");
        g_dims[i] = (int)d;
    }
    g_nv = (size_t)g_dims[0] * g_dims[1] * g_dims[2];
    /* templates and particles */
    nt = (int)list_count(a[1]);
    np = (int)list_count(a[2]);
    tp = (const float **)mxCalloc((size_t)(nt > 0 ? nt : 1), sizeof(float *));
    pp = (const float **)mxCalloc((size_t)(np > 0 ? np : 1), sizeof(float *));
    first_template = g_nvols;
    for (i = 0; i < nt; ++i)
        if (!(tp[i] = read_volume(list_item(a[1], i), "template", i))) nt = -1;
    if (nt < 1) {
        snprintf(msg, sizeof msg,
                 "tom_mex_corr3d: The content of the parameter TEMPLATES must be either em-filename(s) or real "
                 "floating point volume(s) of size %dx%dx%d.", g_dims[0], g_dims[1], g_dims[2]);
        fail(msg);
    }
    first_particle = g_nvols;
    for (i = 0; i < np; ++i)
        if (!(pp[i] = read_volume(list_item(a[2], i), "particle", i))) np = -1;
    if (np < 1) {
        snprintf(msg, sizeof msg,
                 "tom_mex_corr3d: The content of the parameter PARTICLES must be either em-filename(s) or real "
                 "floating point volume(s) of size %dx%dx%d.", g_dims[0], g_dims[1], g_dims[2]);
        fail(msg);
    }
    /* angles: 3 x N degrees -> N triplets */
    if (!mxIsNumeric(a[3]) || mxIsComplex(a[3]) || mxGetNumberOfDimensions(a[3]) > 2 ||
        mxGetNumberOfElements(a[3]) < 1 || mxGetM(a[3]) != 3)
        fail("tom_mex_corr3d: The parameter ANGLES must be a Nx3 matrix of euler-angles [phi, psi, theta] in "
             "degrees.");
    nang = (int)mxGetN(a[3]);
    ang = (double *)mxMalloc(sizeof(double) * 3 * (size_t)nang);
    for (i = 0; i < 3 * nang; ++i)
        ang[i] = num_at(a[3], (mwSize)i);
    snprintf(msg, sizeof msg, "tom_mex_corr3d: The parameter MASK must be a numeric mask of size %dx%dx%d", g_dims[0],
             g_dims[1], g_dims[2]);
    mask = mask_arg(a[4], msg);
    wt = wedge_arg(a[5], nt, "WEDGE_REF");
    wp = wedge_arg(a[6], np, "WEDGE_PART");
    if (narg >= 8) {
        char *ty = mxArrayToString(a[7]);
        const int peak_type = ty && !strcmp(ty, "peak");
        if (ty) mxFree(ty);
        if (!peak_type) {
            fail("tom_mex_corr3d: TYPE 'peak' is built on the GPU; the types 'cc' and 'cc2em' are not.");
        }
    }
    if (narg >= 9)
        mask_cc = mask_arg(a[8], "tom_mex_corr3d: TYPE 'peak' needs a correlation mask as parameter: either [], the "
                                 "radius of a sphere in voxels, or the full floating volume.");
    peak = (double *)mxMalloc(sizeof(double) * 3 * (size_t)nt * np);
    val = (double *)mxMalloc(sizeof(double) * (size_t)nt * np);
    idx = (int32_t *)mxMalloc(sizeof(int32_t) * (size_t)nt * np);
    rc = tomgpu_corr3d_peaks(tomgpu_mex_ctx(), g_dims, tp, nt, pp, np, ang, nang, mask, wt, wp, mask_cc, peak, val,
                             idx);
    if (rc == TOMGPU_OK) {
        odims[0] = (mwSize)nt;
        odims[1] = (mwSize)np;
        plhs[0] = mxCreateStructArray(2, odims, 6, fields);
        for (j = 0, k = 0; j < np; ++j)
            for (i = 0; i < nt; ++i, ++k) {
                mxArray *mp = mxCreateNumericMatrix(1, 3, mxDOUBLE_CLASS, mxREAL);
                mxArray *mv = mxCreateNumericMatrix(1, 1, mxDOUBLE_CLASS, mxREAL);
                mxArray *ma = mxCreateNumericMatrix(1, 3, mxDOUBLE_CLASS, mxREAL);
                mxArray *mi = mxCreateNumericMatrix(1, 1, mxUINT32_CLASS, mxREAL);
                const int ai = idx[k];
                int c;
                for (c = 0; c < 3; ++c) {
                    mxGetPr(mp)[c] = ai > 0 ? peak[3 * k + c] : 0.0;
                    mxGetPr(ma)[c] = ai > 0 ? ang[3 * (ai - 1) + c] : mxGetNaN();
                }
                mxGetPr(mv)[0] = ai > 0 ? val[k] : mxGetNaN();
                ((uint32_t *)mxGetData(mi))[0] = (uint32_t)(ai > 0 ? ai : 0);
                mxSetField(plhs[0], (mwSize)k, "peak", mp);
                mxSetField(plhs[0], (mwSize)k, "ncc_val", mv);
                mxSetField(plhs[0], (mwSize)k, "angle_idx", mi);
                mxSetField(plhs[0], (mwSize)k, "angle", ma);
                mxSetField(plhs[0], (mwSize)k, "template", mxCreateString(g_vols[first_template + i].name));
                mxSetField(plhs[0], (mwSize)k, "particle", mxCreateString(g_vols[first_particle + j].name));
            }
    }
    for (i = 0; i < g_nvols; ++i) mxFree(g_vols[i].data);
    if (g_vols) mxFree(g_vols);
    g_vols = 0;
    g_nvols = g_cap = 0;
    mxFree(ang);
    if (wt) mxFree(wt);
    if (wp) mxFree(wp);
    mxFree(tp);
    mxFree(pp);
    mxFree(peak);
    mxFree(val);
    mxFree(idx);
    tomgpu_mex_check(rc);
}
