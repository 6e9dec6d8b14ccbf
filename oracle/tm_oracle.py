"""CPU oracle for TOM's template-matching hot path.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module, and only as the checker
(or, for the baseline, as the timed CPU restatement).  The CUDA library in
``tom_b200`` never imports, links or calls anything here.

Two layers:

* ``liboracle.so`` (``oracle/flcf_oracle.c``): C restatements of the
  reference's C routines with the same float arithmetic, bit-exact with the
  compiled reference (``oracle/_ref/libref_*.so``, built from the reference's
  own sources by ``oracle/Makefile``).
* this file: numpy restatement of the MATLAB-level FLCF search (Oscar3
  MATLAB picker) in FP64, following

  - ``Oscar3/matlabPicker/search/tom_os3_findTemplate.m:157-307``
  - ``Oscar3/matlabPicker/search/tom_os3_corr.m:77-192``
  - ``Oscar3/matlabPicker/statistics/tom_os3_mean.m:44-62``
  - ``Oscar3/matlabPicker/statistics/tom_os3_std.m:43-67``
  - ``Oscar3/matlabPicker/statistics/tom_os3_normUnderMask.m:3-8``
  - ``Oscar3/matlabPicker/search/tom_os3_sphereMask.m:4-37``
  - ``Oscar3/matlabPicker/tools/tom_os3_pasteCenter.m:17-39``
  - ``Oscar3/matlabPicker/search/tom_os3_bestPeak.m:42-47,94-96``
  - ``Filtrans/tom_apply_weight_function.m:56-62``, ``Filtrans/tom_wedge.m:62-77``
  - ``Analysis/tom_peak.m:80-108,203-279,437-525``
  - ``Analysis/tom_corr.m:51-121``, ``av3_new/tom_av3_align.m:97-189``

The FFT itself is third-party arithmetic in the reference (MATLAB ``fftn``,
FFTW inside); the DFT is mathematically defined, so numpy's pocketfft in FP64
is the reference value here.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int)


def _p(a, t):
    return a.ctypes.data_as(t)


_LIBS: dict = {}


def _load(name):
    if name not in _LIBS:
        path = os.path.join(REF_DIR, name)
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} missing: run `make -C oracle oracle` (reference libraries: `make -C oracle ref REF=<TOM source tree>`)")
        _LIBS[name] = ctypes.CDLL(path)
    return _LIBS[name]


def oracle_lib():
    lib = _load("liboracle.so")
    lib.oracle_euler_matrix.argtypes = [_f32p, _f32p]
    lib.oracle_rot3d.argtypes = [_f32p, _f32p, ctypes.c_long, ctypes.c_long, ctypes.c_long,
                                 _f32p, ctypes.c_float, ctypes.c_float, ctypes.c_float]
    lib.oracle_rot3d_batch.argtypes = [_f32p, _f32p, ctypes.c_long, ctypes.c_long, ctypes.c_long,
                                       _f32p, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_float]
    lib.oracle_find_max.argtypes = [_f32p, _i32p, _f32p, _i32p]
    lib.oracle_weight3d.argtypes = [_f32p, _i32p, _f64p, ctypes.c_int, ctypes.c_double]
    return lib


def ref_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, n))
               for n in ("libref_rotate.so", "libref_peak.so", "libref_weight.so"))


def ref_rotate_lib():
    lib = _load("libref_rotate.so")
    # rot3d(float*, float*, long, long, long, float*, char, float, float, float, int)
    lib.rot3d.argtypes = [_f32p, _f32p, ctypes.c_long, ctypes.c_long, ctypes.c_long, _f32p,
                          ctypes.c_char, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                          ctypes.c_int]
    return lib


def ref_peak_lib():
    lib = _load("libref_peak.so")
    lib.find_max.argtypes = [_f32p, _i32p, _f32p, _i32p]
    return lib


def ref_weight_lib():
    lib = _load("libref_weight.so")
    lib.weight3d.argtypes = [_f32p, _i32p, _f64p, ctypes.c_int, _f64p]
    return lib


# ---------------------------------------------------------------------------
# Arrays: volumes are numpy arrays indexed [x, y, z] (MATLAB order) stored in
# Fortran order, so the flat memory is x-fastest like MATLAB and the C code.
# ---------------------------------------------------------------------------

def _f32_fortran(a):
    return np.asfortranarray(a, dtype=np.float32)


def default_center(shape):
    """tom_rotate default centre ceil(size/2) passed 0-based (Sptrans/tom_rotate.m:105)."""
    return tuple(float(np.ceil(s / 2)) for s in shape)


def euler_matrix(euler_deg):
    """9 floats rm00, rm10, rm20, rm01, rm11, rm21, rm02, rm12, rm22."""
    e = np.asarray(euler_deg, dtype=np.float32).reshape(3).copy()
    m = np.zeros(9, np.float32)
    oracle_lib().oracle_euler_matrix(_p(e, _f32p), _p(m, _f32p))
    return m


def rotate(vol, euler_deg, center=None):
    """tom_rotate(vol, [phi psi theta], 'linear', center) in FP32 (C restatement of rot3d)."""
    v = _f32_fortran(vol)
    c = default_center(v.shape) if center is None else tuple(float(x) for x in center)
    out = np.zeros(v.shape, np.float32, order="F")
    m = euler_matrix(euler_deg)
    sx, sy, sz = v.shape
    oracle_lib().oracle_rot3d(_p(v, _f32p), _p(out, _f32p), sx, sy, sz, _p(m, _f32p), *c)
    return out


def rotate_matrix(vol, m9, center=None):
    """tom_rotate with a 3x3 matrix argument (matrix mode of rot3d): m9 in rm00, rm10, ... order."""
    v = _f32_fortran(vol)
    c = default_center(v.shape) if center is None else tuple(float(x) for x in center)
    out = np.zeros(v.shape, np.float32, order="F")
    m = np.asarray(m9, np.float32).reshape(9).copy()
    sx, sy, sz = v.shape
    oracle_lib().oracle_rot3d(_p(v, _f32p), _p(out, _f32p), sx, sy, sz, _p(m, _f32p), *c)
    return out


def rotate_batch(vol, eulers, center=None):
    v = _f32_fortran(vol)
    c = default_center(v.shape) if center is None else tuple(float(x) for x in center)
    e = np.ascontiguousarray(eulers, dtype=np.float32).reshape(-1, 3)
    R = e.shape[0]
    out = np.zeros((R,) + v.shape[::-1], np.float32)  # C order [r][z][y][x]
    sx, sy, sz = v.shape
    oracle_lib().oracle_rot3d_batch(_p(v, _f32p), _p(out, _f32p), sx, sy, sz, _p(e, _f32p), R, *c)
    return [np.asfortranarray(out[r].transpose(2, 1, 0)) for r in range(R)]


def ref_rotate(vol, euler_or_matrix, center=None):
    """The reference's own compiled rot3d (oracle/_ref)."""
    v = _f32_fortran(vol)
    c = default_center(v.shape) if center is None else tuple(float(x) for x in center)
    out = np.zeros(v.shape, np.float32, order="F")
    e = np.asarray(euler_or_matrix, np.float32).reshape(-1).copy()
    euler_dim = 1 if e.size == 3 else 3
    sx, sy, sz = v.shape
    ref_rotate_lib().rot3d(_p(v, _f32p), _p(out, _f32p), sx, sy, sz, _p(e, _f32p), b"l",
                           c[0], c[1], c[2], euler_dim)
    return out


def find_max(v):
    a = _f32_fortran(v)
    dims = np.array(a.shape + (1,) * (3 - a.ndim), np.int32)
    val = np.zeros(1, np.float32)
    pos = np.zeros(3, np.int32)
    oracle_lib().oracle_find_max(_p(a, _f32p), _p(dims, _i32p), _p(val, _f32p), _p(pos, _i32p))
    return float(val[0]), tuple(int(x) for x in pos)


def ref_find_max(v):
    a = _f32_fortran(v)
    dims = np.array(a.shape + (1,) * (3 - a.ndim), np.int32)
    val = np.zeros(1, np.float32)
    pos = np.zeros(3, np.int32)
    ref_peak_lib().find_max(_p(a, _f32p), _p(dims, _i32p), _p(val, _f32p), _p(pos, _i32p))
    return float(val[0]), tuple(int(x) for x in pos)


def weight3d(dims, angles_2xn, thickness):
    d = np.array(dims, np.int32)
    ang = np.ascontiguousarray(np.asarray(angles_2xn, np.float64).T)  # n x 2 -> (phi, theta) pairs
    out = np.zeros(tuple(dims), np.float32, order="F")
    oracle_lib().oracle_weight3d(_p(out, _f32p), _p(d, _i32p), _p(ang, _f64p), ang.shape[0],
                                 float(thickness))
    return out


def ref_weight3d(dims, angles_2xn, thickness):
    d = np.array(dims, np.int32)
    ang = np.ascontiguousarray(np.asarray(angles_2xn, np.float64).T)
    out = np.zeros(tuple(dims), np.float32, order="F")
    th = np.array([float(thickness)], np.float64)
    ref_weight_lib().weight3d(_p(out, _f32p), _p(d, _i32p), _p(ang, _f64p), ang.shape[0],
                              _p(th, _f64p))
    return out


# ---------------------------------------------------------------------------
# MATLAB-level restatement (FP64)
# ---------------------------------------------------------------------------

def tom_norm_mean0_1std(a):
    """tom_norm(a,'mean0+1std') (Sptrans/tom_norm.m:83-119 with tom_dev's population std)."""
    a = np.asarray(a, np.float64) * 2 + 100
    m = a.mean()
    s = a.std()
    return (a - m) / s if s != 0 else a - m


def tom_dev(a, mask=None):
    """(mean, max, min, std) of Analysis/tom_dev.m:57-60: in double, over the
    voxels where mask > 0 (all without a mask), std with the 1/n normalisation."""
    a = np.asarray(a, np.float64)
    v = a[np.asarray(mask) > 0] if mask is not None else a.ravel()
    return v.mean(), v.max(), v.min(), v.std()


def tom_norm(a, scf="mean0+1std", mask=None):
    """Sptrans/tom_norm.m:79-153, every branch: 'mean0+1std' (after a -> 2a + 100,
    :83-85), 'phase', '1std' / '2std' / '3std' (tom_limit about the mean),
    'oscar' (3std limit + 100, then phase-normalised) and a number scf (the
    range [min, max] mapped to [0, scf]; a / scf for a constant input; a when
    the mean already equals scf).  Statistics from tom_dev, inside the mask
    when one is given."""
    a = np.asarray(a, np.float64)
    if isinstance(scf, str) and scf == "mean0+1std":
        a = a * 2 + 100
    mea, ma, mi, st = tom_dev(a, mask)
    if isinstance(scf, str):
        if scf == "phase":
            return (a - mea) / (mea + 1e-12)
        if scf in ("1std", "2std", "3std"):
            k = float(scf[0])
            return tom_limit(a, mea - k * st, mea + k * st) - mea
        if scf == "mean0+1std":
            return (a - mea) / st if st != 0 else a - mea
        if scf == "oscar":
            m2, _, _, s2 = tom_dev(a)
            c = tom_limit(a, m2 - 3 * s2, m2 + 3 * s2) - m2 + 100
            mc = tom_dev(c, mask)[0]
            return (c - mc) / (mc + 1e-12)
        raise ValueError("Only numbers and keyword 'phase', '2std' , '3std' or 'mean0+1std' allowed.")
    if st != 0 and mea != scf:
        s = a - mi
        return scf * s / s.max()
    if st == 0 and mea != scf:
        return a / scf
    return a


def os3_sphere_mask(shape):
    """tom_os3_sphereMask(template): radius floor(min/2)-1, centre floor(n/2)+1 (1-based),
    zero where distance >= radius; non-cubic input -> all ones."""
    shape = tuple(shape)
    if len(set(shape)) != 1:
        return np.ones(shape), int(np.prod(shape))
    radius = np.floor(min(shape) / 2) - 1
    return sphere_mask(shape, radius, strict=False), None


def sphere_mask(shape, radius, center=None, strict=False):
    """Binary sphere: 1 where distance < radius (os3 sphMask, strict=False) or
    distance <= radius (tom_sphere, strict=True).  centre is 1-based like MATLAB."""
    if center is None:
        center = [np.floor(s / 2) + 1 for s in shape]
    g = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij")
    d = np.sqrt(sum((gi + 1 - c) ** 2 for gi, c in zip(g, center)))
    m = np.ones(shape)
    if strict:
        m[d > radius] = 0
    else:
        m[d >= radius] = 0
    return m


def centered_grid(shape):
    return np.meshgrid(*[np.arange(-(s // 2), -(s // 2) + s, dtype=np.float64) for s in shape],
                       indexing="ij")


def tom_wedge(shape, angle_deg):
    """Filtrans/tom_wedge.m:62-77: zero where tan(angle) > |x|/|z| on a centred grid."""
    x, _, z = centered_grid(shape)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.abs(x) / np.abs(z)
    w = np.ones(shape)
    w[np.tan(np.deg2rad(angle_deg)) > r] = 0
    return w


def av3_wedge(shape, minangle, maxangle):
    """av3_new/tom_av3_wedge.m / av3/utils/av3_wedge.m:23-26."""
    x, _, z = centered_grid(shape)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = x / z
    a = np.tan(np.pi / 2 - np.deg2rad(maxangle)) > r
    b = np.tan(-np.pi / 2 - np.deg2rad(minangle)) < r
    w = np.ones(shape)
    w[a & b] = 0
    return w


def apply_weight_function(vol, w):
    """Filtrans/tom_apply_weight_function.m:56-62: real(ifftn(ifftshift(fftshift(fftn(in)).*w)))."""
    f = np.fft.fftshift(np.fft.fftn(np.asarray(vol, np.float64)))
    return np.real(np.fft.ifftn(np.fft.ifftshift(f * w)))


def norm_under_mask(vol, mask):
    """statistics/tom_os3_normUnderMask.m:3-8: mean and population std under the mask."""
    m = mask != 0
    n = m.sum()
    v = np.asarray(vol, np.float64)
    # a NaN or Inf anywhere in vol (the unguarded same-size division of
    # tom_os3_corr.m:172-176) makes both statistics NaN, as in MATLAB (NaN * 0 = NaN)
    with np.errstate(invalid="ignore"):
        mea = ((v * m) * (v != 0)).sum() / n
        st = np.sqrt(((((~m) * mea) + (v * m) - mea) ** 2).sum() / n)
        return ((v - mea) / st) * m, mea, st


def paste_center(shape, small):
    """tools/tom_os3_pasteCenter.m:36-39 (3-D case)."""
    out = np.zeros(shape)
    o = [s // 2 - t // 2 for s, t in zip(shape, small.shape)]
    out[o[0]:o[0] + small.shape[0], o[1]:o[1] + small.shape[1], o[2]:o[2] + small.shape[2]] = small
    return out


def local_stats(volume, mask):
    """tom_os3_mean / tom_os3_std: local mean and std under the mask, FP64.

    mean = real(ifftshift(ifftn(F_I . F_M)))/M ;
    std  = sqrt(max(real(ifftshift(ifftn(F_{I^2} . F_M)))/M - mean^2, 0)).
    """
    vol = np.asarray(volume, np.float64)
    N = vol.shape
    mp = paste_center(N, np.asarray(mask, np.float64))
    M = float((mask != 0).sum())
    fm = np.fft.rfftn(mp)
    mean = np.fft.ifftshift(np.fft.irfftn(np.fft.rfftn(vol) * fm, s=N, axes=(0, 1, 2))) / M
    e2 = np.fft.ifftshift(np.fft.irfftn(np.fft.rfftn(vol * vol) * fm, s=N, axes=(0, 1, 2))) / M
    var = np.maximum(e2 - mean * mean, 0)
    return mean, np.sqrt(var), M


class FLCF:
    """Per-volume state of tom_os3_corr's FLCF branch (statistics cached once)."""

    def __init__(self, volume, mask):
        self.N = tuple(volume.shape)
        self.mask = np.asarray(mask, np.float64)
        self.mean, self.std, self.M = local_stats(volume, self.mask)
        self.fimage = np.fft.rfftn(np.asarray(volume, np.float64))

    def corr(self, t, tmean, tstd):
        """search/tom_os3_corr.m:151-176 for one (already rotated/modified) template.
        A template holding NaN (an autocorrelation map from the same-size
        branch) gives NaN numerators and denominators, and the denominator
        rule then leaves 0 at every voxel, as the reference's res(nonzero)."""
        with np.errstate(invalid="ignore"):
            p = paste_center(self.N, np.asarray(t, np.float64) * self.mask)
        ft = np.fft.rfftn(p)
        num = np.fft.ifftshift(np.fft.irfftn(self.fimage * np.conj(ft), s=self.N, axes=(0, 1, 2))) / self.M
        num = num - self.mean * tmean
        den = tstd * self.std
        res = np.zeros(self.N)
        eps = np.finfo(np.float64).eps
        nz = np.abs(den - eps) > eps
        res[nz] = num[nz] / den[nz]
        return res


def prepare_template(template, mask, psf=None):
    """findTemplate preprocessing (tom_os3_findTemplate.m:157,233-234):
    tom_norm(1e5*(t+1),'mean0+1std'); statistics of the unrotated, modified template."""
    t = tom_norm_mean0_1std(1e5 * (np.asarray(template, np.float64) + 1))
    tmp = t if psf is None else apply_weight_function(t, psf)
    _, tmean, tstd = norm_under_mask(tmp, mask)
    return t, tmean, tstd


def find_template(volume, template, mask, angles, psf=None, keep_second=False):
    """Exhaustive FLCF search, tom_os3_findTemplate.m:255-307 + tom_os3_bestPeak (ccc mode).

    Returns (ccc, idx) with idx the 0-based angle index (reference: 1-based
    iterator) and -1 where never updated (reference init -1000).  With
    keep_second, also returns the second-best CC per voxel (for tie analysis).
    """
    t, tmean, tstd = prepare_template(template, mask, psf)
    st = FLCF(volume, mask)
    ccc = np.full(st.N, -1000.0)
    idx = np.full(st.N, -1, np.int64)
    second = np.full(st.N, -1000.0)
    for it, ang in enumerate(np.asarray(angles, np.float64).reshape(-1, 3)):
        tr = rotate(t.astype(np.float32), ang).astype(np.float64) * mask
        if psf is not None:
            tr = apply_weight_function(tr, psf)
        cc = st.corr(tr.astype(np.float32).astype(np.float64), tmean, tstd)
        upd = ccc < cc
        if keep_second:
            second = np.where(upd, ccc, np.maximum(second, cc))
        ccc[upd] = cc[upd]
        idx[upd] = it
    return (ccc, idx, second) if keep_second else (ccc, idx)


def flcf_direct_at(volume, t, mask, tmean, tstd, voxels):
    """FLCF of one rotated/masked/filtered template at given voxels (0-based, [x,y,z])
    by direct FP64 sums: the correlation sum of tom_os3_corr.m:151-153 and the
    convolution sums of tom_os3_mean/std, without any FFT."""
    vol = np.asarray(volume, np.float64)
    N = np.array(vol.shape)
    T = np.array(mask.shape)
    c = T // 2
    jj = np.argwhere(np.ones(tuple(T), bool))
    tw = (np.asarray(t, np.float64) * mask)[tuple(jj.T)]
    mw = np.asarray(mask, np.float64)[tuple(jj.T)]
    M = float((mask != 0).sum())
    out = []
    for x in np.asarray(voxels).reshape(-1, 3):
        q = (x[None, :] + jj - c[None, :]) % N            # correlation: I(x + j - c)
        s = float((tw * vol[tuple(q.T)]).sum())
        qc = (x[None, :] + c[None, :] - jj) % N           # convolution: I(x + c - j)
        iv = vol[tuple(qc.T)]
        mu = float((mw * iv).sum()) / M
        e2 = float((mw * iv * iv).sum()) / M
        sig = np.sqrt(max(e2 - mu * mu, 0.0))
        den = tstd * sig
        out.append((s / M - mu * tmean) / den if den != 0 else 0.0)
    return np.array(out)


def find_template_direct_at(volume, template, mask, angles, voxels, psf=None):
    """Per-voxel max over angles and its first index (bestPeak rule) at given voxels, direct sums."""
    t, tmean, tstd = prepare_template(template, mask, psf)
    best = np.full(len(voxels), -1000.0)
    second = np.full(len(voxels), -1000.0)
    idx = np.full(len(voxels), -1, np.int64)
    for it, ang in enumerate(np.asarray(angles, np.float64).reshape(-1, 3)):
        tr = rotate(t.astype(np.float32), ang).astype(np.float64) * mask
        if psf is not None:
            tr = apply_weight_function(tr, psf)
        cc = flcf_direct_at(volume, tr.astype(np.float32), mask, tmean, tstd, voxels)
        upd = best < cc
        second = np.where(upd, best, np.maximum(second, cc))
        best = np.where(upd, cc, best)
        idx = np.where(upd, it, idx)
    return best, idx, second


# ---------------------------------------------------------------------------
# Peak analysis: PSR and autocorrelation (SOC) maps
# ---------------------------------------------------------------------------

def psr_mask_box(tshape):
    """The PSR mask of tom_os3_analyzePeak.m:68,90 inside its template-sized box:
    tom_os3_sphereMask(template) with a centred box of floor(T/4) voxels per
    axis zeroed (pasteCenter(mask, 0*sphereMask(zeros(T/4)))).  The N-sized
    mask is this box pasted at the centre."""
    box, _ = os3_sphere_mask(tshape)
    box = np.array(box, np.float64)
    q = [t // 4 for t in tshape]
    if min(q) > 0:
        o = [t // 2 - s // 2 for t, s in zip(tshape, q)]
        box[o[0]:o[0] + q[0], o[1]:o[1] + q[1], o[2]:o[2] + q[2]] = 0
    return box


def _single_eps(x):
    """MATLAB eps(single(x)) for x >= 0."""
    return float(np.spacing(np.float32(x)))


def analyze_psr(peak, tshape):
    """tom_os3_analyzePeak(img, peakMap, template, 'PSR') (analyze/tom_os3_analyzePeak.m:61-101):
    (peakMap - mean)/std under the PSR mask, 0 where std <= 1000 eps(max std)."""
    p = np.asarray(peak, np.float64)
    mean, std, _ = local_stats(p, psr_mask_box(tuple(tshape)))
    s32 = std.astype(np.float32)
    tol = 1000 * _single_eps(np.abs(s32).max())
    res = np.zeros(p.shape)
    nz = s32 > tol
    res[nz] = (p - mean)[nz] / s32[nz].astype(np.float64)
    return res


def _hot_threshold(img, std):
    """The two 'numeric artefact' branches of tom_os3_corr.m:108-127.  The first
    (tom_norm of the image and template when mean(std) < 0.01) is an affine map
    of both inputs and leaves the FLCF unchanged; the second marks voxels whose
    renormalised local std is below 0.05 when the renormalised mean std is
    still below 0.01.  Returns the threshold on the original std (or None)."""
    if std.mean() >= 0.01:
        return None
    a = np.asarray(img, np.float64)
    s = a.std()                       # tom_norm's tom_dev std
    scale = 1.0 / s if s != 0 else 2.0
    if (std * scale).mean() >= 0.01:
        return None
    return 0.05 / scale


def os3_corr_same(img, t):
    """tom_os3_corr(img, template) with no options for same-size inputs
    (search/tom_os3_corr.m:77-176): default sphere mask, statistics of both
    inputs under it, res = numerator./denominator at every voxel."""
    a = np.asarray(img, np.float64)
    t = np.asarray(t, np.float64)
    mask, _ = os3_sphere_mask(t.shape)
    mask = np.asarray(mask, np.float64)
    mean, std, M = local_stats(a, mask)
    _, tmean, tstd = norm_under_mask(t, mask)
    ft = np.fft.rfftn(t * mask)
    num = np.fft.ifftshift(np.fft.irfftn(np.fft.rfftn(a) * np.conj(ft), s=a.shape, axes=(0, 1, 2))) / M
    with np.errstate(divide="ignore", invalid="ignore"):
        res = (num - mean * tmean) / (tstd * std)
    thr = _hot_threshold(a, std)
    if thr is not None:
        res[std < thr] = 0
    return res


def analyze_autocorr(peak, t, mask):
    """tom_os3_analyzePeak(0, peakMap, template, 'Autocorrelation')
    (analyze/tom_os3_analyzePeak.m:174-190): the template's autocorrelation
    A = tom_os3_corr(t, t), then the FLCF of the peak map with A under the
    correlation mask, with A's own statistics (tom_os3_corr.m, sizes differ)."""
    A = os3_corr_same(t, t).astype(np.float32).astype(np.float64)
    p = np.asarray(peak, np.float64)
    st = FLCF(p, mask)
    _, am, asd = norm_under_mask(A, mask)
    res = st.corr(A, am, asd)
    thr = _hot_threshold(p, st.std)
    if thr is not None:
        res[st.std < thr] = 0
    return res


def find_template_analysis(volume, template, mask, angles, psf=None, ccc=True, psr=False, autocorr=False,
                           margins=False):
    """tom_os3_findTemplate.m:255-307 with the PSR and autocorrelation maps of
    every rotation and tom_os3_bestPeak's update (search/tom_os3_bestPeak.m:12-47):
    a voxel takes the rotation's (cc, psr, soc, index) where every selected
    criterion strictly improves.  Returns (ccc, idx, psr, soc); idx 0-based,
    -1 where never updated; ccc/psr/soc -1000 there.  With margins, also the
    per-voxel smallest |old - new| / (1 + |new|) over all decisions taken on
    the selected criteria (voxels whose decisions were all clear-cut)."""
    t, tmean, tstd = prepare_template(template, mask, psf)
    st = FLCF(volume, mask)
    out_c = np.full(st.N, -1000.0)
    out_p = np.full(st.N, -1000.0)
    out_a = np.full(st.N, -1000.0)
    idx = np.full(st.N, -1, np.int64)
    margin = np.full(st.N, np.inf)
    T = mask.shape
    for it, ang in enumerate(np.asarray(angles, np.float64).reshape(-1, 3)):
        tr = rotate(t.astype(np.float32), ang).astype(np.float64) * mask
        if psf is not None:
            tr = apply_weight_function(tr, psf)
        tr = tr.astype(np.float32).astype(np.float64)
        cc = st.corr(tr, tmean, tstd).astype(np.float32).astype(np.float64)
        pm = analyze_psr(cc, T)
        am = analyze_autocorr(cc, tr, mask)
        upd = np.ones(st.N, bool)
        for sel, old, new in ((ccc, out_c, cc), (psr, out_p, pm), (autocorr, out_a, am)):
            if sel:
                upd &= old < new
                with np.errstate(invalid="ignore"):
                    margin = np.minimum(margin, np.abs(old - new) / (1 + np.abs(new)))
        out_c[upd], out_p[upd], out_a[upd], idx[upd] = cc[upd], pm[upd], am[upd], it
    res = (out_c, idx, out_p, out_a)
    return res + (margin,) if margins else res


# ---------------------------------------------------------------------------
# Averaging after alignment
# ---------------------------------------------------------------------------

def tom_shift(im, delta):
    """Filtrans/tom_shift.m: Fourier shift by delta (FP64), real part."""
    im = np.asarray(im, np.float64)
    dims = im.shape
    g = np.meshgrid(*[np.arange(-(n // 2), -(n // 2) + n, dtype=np.float64) for n in dims], indexing="ij")
    d = np.array(delta, np.float64).reshape(3).copy()
    d[[i for i, n in enumerate(dims) if n == 1]] = 0
    d = d / np.array(dims, np.float64)
    x = d[0] * g[0] + d[1] * g[1] + d[2] * g[2]
    return np.real(np.fft.ifftn(np.fft.fftn(im) * np.exp(-2j * np.pi * np.fft.ifftshift(x))))


def tom_limit(a, low, up, mode=None):
    """Sptrans/tom_limit.m: clamp; 'z': below low -> 0, above up -> up."""
    a = np.array(a, np.float64, copy=True)
    if mode == "z":
        a[a < low] = 0
        a[a > up] = up
    else:
        a[a < low] = low
        a[a > up] = up
    return a


def av3_average_add(items, shape):
    """av3/alignment/av3_tomomatch.m:239-249 for (particle, wedge, tshift, [phi psi theta]) items, in order."""
    avg = np.zeros(shape)
    wei = np.zeros(shape)
    for part, wedge, tshift, ang in items:
        phi, psi, the = ang
        inv = (-psi, -phi, -the)
        sh = tom_shift(part, -np.asarray(tshift, np.float64))
        avg += rotate(sh.astype(np.float32), inv).astype(np.float64)
        rw = rotate(np.asarray(wedge, np.float32), inv).astype(np.float64)
        wei += 2 * tom_limit(tom_limit(rw, 0.5, 1, "z"), 0, 0.5)
    return avg, wei


def av3_average_final(avg, wei):
    """av3_tomomatch.m:263-265: w = 1./wei (above 1e5 -> 0), sphere-masked
    (radius floor(n/2)-3) spectral weighting of the sum."""
    with np.errstate(divide="ignore"):
        w = 1.0 / wei
    w[w > 100000] = 0
    lowp = avg.shape[0] // 2 - 3
    f = np.fft.fftshift(np.fft.fftn(avg)) * w
    f = f * sphere_mask(avg.shape, lowp, strict=False)
    return np.real(np.fft.ifftn(np.fft.ifftshift(f)))


# ---------------------------------------------------------------------------
# The C++ picker's batched aligner (Oscar3/c++Picker): tom_mex_corr3d 'peak'
# ---------------------------------------------------------------------------
# Volumes are [x, y, z] arrays (x fastest in memory, Fortran order) like the
# C++ tom::Volume.  Reduced spectra halve the z axis (the last one), which is
# what numpy's rfftn/irfftn do on these arrays, and irfftn ignores the
# imaginary parts of the kz = 0 and kz = nz/2 planes like FFTW's c2r.

CPP_PI = 3.141592653589793238512808959406186204433


def cpp_rotmat(phi, theta, psi):
    """tom_transf_init_rotmat_3d(P, 3, 3, {z, x, z}, {phi, theta, psi})
    (src/tom/core/transform.c:99-176): P = Rz(phi) Rx(theta) Rz(psi), radians;
    an angle with angle - floor(angle/(pi/2))*2*pi == 0 is skipped."""
    P = np.eye(3)
    for axis, a in ((2, phi), (0, theta), (2, psi)):
        if a - np.floor(a / (np.pi / 2.0)) * (2.0 * np.pi) == 0.0:
            continue
        s, c = np.sin(a), np.cos(a)
        i, j = (1, 2) if axis == 0 else (0, 1)
        p0, p1 = P[:, i].copy(), P[:, j].copy()
        P[:, i] = p0 * c - p1 * s
        P[:, j] = p0 * s + p1 * c
    return P


def cpp_rotate_coords(shape, phi, psi, theta):
    """Source coordinates of tom::rotate(src, dst, phi, psi, theta)
    (include/tom/core/volume_fcn.hpp:206, src/tom/core/volume_fcn.cpp:740-800):
    src = c + R (dst - c), c = ceil((n-1)/2), as p00*x + (p01*y + (p02*z + p03))."""
    R = cpp_rotmat(phi, theta, psi)
    c = np.array([np.ceil((n - 1) / 2.0) for n in shape])
    t = c - R @ c
    X, Y, Z = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")
    out = []
    for r in range(3):
        out.append(R[r, 0] * X + (R[r, 1] * Y + (R[r, 2] * Z + t[r])))
    return out, R, t


def cpp_interp_trilinear(vol, x, y, z):
    """tom_transf_interpol3d_trilinear_float (src/tom/core/_transform.c:119-262,
    the active branch): 0 outside [0, n-1]; float weights x - floor(x); the
    neighbours of an axis are read only where its weight is > 0."""
    v = np.asarray(vol, np.float32)
    sx, sy, sz = v.shape
    out = np.zeros(x.shape, np.float32)
    ins = (x >= 0) & (y >= 0) & (z >= 0) & (x <= sx - 1) & (y <= sy - 1) & (z <= sz - 1)
    fx = np.where(ins, x, 0).astype(np.int64)
    fy = np.where(ins, y, 0).astype(np.int64)
    fz = np.where(ins, z, 0).astype(np.int64)
    xo = (np.where(ins, x, 0) - fx).astype(np.float32)
    yo = (np.where(ins, y, 0) - fy).astype(np.float32)
    zo = (np.where(ins, z, 0) - fz).astype(np.float32)

    def at(dx, dy, dz):
        return v[np.minimum(fx + dx, sx - 1), np.minimum(fy + dy, sy - 1), np.minimum(fz + dz, sz - 1)]

    s000 = at(0, 0, 0)
    s100, s010, s001 = at(1, 0, 0), at(0, 1, 0), at(0, 0, 1)
    s110, s101, s011, s111 = at(1, 1, 0), at(1, 0, 1), at(0, 1, 1), at(1, 1, 1)
    f32 = np.float32
    lx = lambda a, b: (a + (b - a) * xo).astype(f32)
    ly = lambda a, b: (a + (b - a) * yo).astype(f32)
    lz = lambda a, b: (a + (b - a) * zo).astype(f32)
    case = (xo > 0).astype(int) | ((yo > 0).astype(int) << 1) | ((zo > 0).astype(int) << 2)
    x0yx = (lx(s000, s100) + (lx(s010, s110) - lx(s000, s100)) * yo).astype(f32)
    r7 = (x0yx + (((lx(s001, s101) + (lx(s011, s111) - lx(s001, s101)) * yo).astype(f32)) - x0yx) * zo).astype(f32)
    x0y0 = ly(s000, s010)
    r6 = (x0y0 + ((s001 + (s011 - s001) * yo).astype(f32) - x0y0) * zo).astype(f32)
    x00x = lx(s000, s100)
    r5 = (x00x + ((s001 + (s101 - s001) * xo).astype(f32) - x00x) * zo).astype(f32)
    r3 = (x00x + ((s010 + (s110 - s010) * xo).astype(f32) - x00x) * yo).astype(f32)
    res = np.select([case == 7, case == 6, case == 5, case == 3, case == 4, case == 2, case == 1],
                    [r7, r6, r5, r3, lz(s000, s001), ly(s000, s010), lx(s000, s100)], s000)
    out[ins] = res[ins]
    return out


def cpp_rotate(vol, phi, psi, theta):
    """tom::rotate(src, dst, phi, psi, theta) with the trilinear interpolation, radians."""
    (x, y, z), _, _ = cpp_rotate_coords(np.shape(vol), phi, psi, theta)
    return np.asfortranarray(cpp_interp_trilinear(vol, x, y, z))


def ref_transform_lib():
    lib = _load("libref_transform.so")
    lib.tom_transf_init_rotmat_3d.argtypes = [_f64p, ctypes.c_size_t, ctypes.c_size_t, _i32p, _f64p]
    lib.tom_transf_invert.argtypes = [_f64p, _f64p, ctypes.c_int]
    lib.tom_transf_transf3d_float.argtypes = [
        _f32p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t,
        _f32p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t,
        _f64p, ctypes.c_int, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]
    return lib


def ref_cpp_rotate(vol, phi, psi, theta):
    """tom::rotate through the reference's own compiled transform.c: the
    matrix assembly of volume_fcn.cpp:740-780 written out here, the rotation
    matrix, the inversion and the transform called from the reference."""
    lib = ref_transform_lib()
    v = np.asfortranarray(vol, dtype=np.float32)
    sx, sy, sz = v.shape
    P = np.zeros(16)
    P[15] = 1.0
    axes = np.array([2, 0, 2], np.int32)
    ang = np.array([phi, theta, psi], np.float64)
    lib.tom_transf_init_rotmat_3d(_p(P, _f64p), 4, 3, _p(axes, _i32p), _p(ang, _f64p))
    lib.tom_transf_invert(_p(P, _f64p), _p(P, _f64p), 4)
    c = [np.ceil((n - 1) / 2.0) for n in (sx, sy, sz)]
    for r in range(3):
        P[4 * r + 3] = c[r] + P[4 * r] * (-c[0]) + P[4 * r + 1] * (-c[1]) + P[4 * r + 2] * (-c[2])
    out = np.zeros(v.shape, np.float32, order="F")
    opt = np.zeros(1, np.float64)
    fn = ctypes.cast(lib.tom_transf_interpol3d_trilinear_float, ctypes.c_void_p)
    rc = lib.tom_transf_transf3d_float(_p(v, _f32p), sx, sy, sz, sx, sx * sy, _p(out, _f32p), sx, sy, sz, sx,
                                       sx * sy, _p(P, _f64p), 1, 0.0, fn, opt.ctypes.data_as(ctypes.c_void_p))
    assert rc == 0
    return out


def cpp_norm_mask(v, mask):
    """tom::norm_mask(v, mask, NORM_NO_NORM, &variance, false)
    (src/tom/core/volume_fcn.cpp:172-258): shift to mean 0 under mask != 0,
    multiply by the mask, shift the masked voxels to mean 0 again; variance =
    (sum2 - n mean^2) / numel of the masked values."""
    v = np.asarray(v, np.float64)
    m = np.asarray(mask, np.float64)
    inside = m != 0
    n = inside.sum()
    mean0 = v[inside].sum() / n
    w = np.where(inside, (v - mean0) * m, 0.0).astype(np.float32).astype(np.float64)
    s1, s2 = w[inside].sum(), (w[inside] ** 2).sum()
    mean1 = s1 / n
    var = (s2 - n * mean1 * mean1) / v.size
    if mean1 != 0:
        w = np.where(inside, w - mean1, w)
    return w.astype(np.float32), var


def cpp_stat(v):
    """tom::Volume::stat(mean, variance, false): population variance, one pass."""
    v = np.asarray(v, np.float64)
    mean = v.sum() / v.size
    var = ((v * v).sum() - v.size * mean * mean) / v.size
    return mean, var


def cpp_simple_wedge(shape, angle, cutoff, phi=0.0, psi=0.0, theta=0.0, reduced=True):
    """tom::SimpleWedge::init_wedge_volume (src/tom/core/wedge.cpp:107-180) in
    float: the frequency k = ((i + ceil(n/2)) mod n) - ceil((n-1)/2) rotated by
    R(phi, theta, psi) is kept where |R k| <= cutoff and (|z'| < 1e-4 or
    tan(angle) <= |x'|/|z'|) (cutoff > 0 branch)."""
    sx, sy, sz = shape
    f32 = np.float32
    c = [f32(np.ceil((n - 1) / 2.0)) for n in shape]
    R = cpp_rotmat(phi, theta, psi)
    Pd = np.zeros(12)
    Pd[0:3], Pd[4:7], Pd[8:11] = R[0], R[1], R[2]
    for r in range(3):
        Pd[4 * r + 3] = -(Pd[4 * r] * c[0] + Pd[4 * r + 1] * c[1] + Pd[4 * r + 2] * c[2])
    P = Pd.astype(f32)
    off = [n // 2 + n % 2 for n in shape]
    nz = sz // 2 + 1 if reduced else sz
    xs = ((np.arange(sx) + off[0]) % sx).astype(f32)
    ys = ((np.arange(sy) + off[1]) % sy).astype(f32)
    zs = ((np.arange(nz) + off[2]) % sz).astype(f32)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    maxdist = f32(np.sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]))
    tan_a = f32(np.tan(angle))
    cut = f32(cutoff) if (cutoff > 0 and cutoff < maxdist) else f32(0)

    def row(r, Xv, Yv, Zv):
        zt = (P[4 * r + 2] * Zv + P[4 * r + 3]).astype(f32)
        yt = (P[4 * r + 1] * Yv + zt).astype(f32)
        return (P[4 * r] * Xv + yt).astype(f32)

    x_ = row(0, X, Y, Z)
    if cut:
        y_ = row(1, X, Y, Z)
        z_ = np.abs(row(2, X, Y, Z))
        with np.errstate(divide="ignore", invalid="ignore"):
            keep = (np.sqrt((x_ * x_ + y_ * y_ + z_ * z_).astype(f32)) <= cut) & \
                   ((z_ < f32(1e-4)) | (tan_a <= np.abs(x_) / z_))
    else:
        z_ = row(2, X, Y, Z)
        with np.errstate(divide="ignore", invalid="ignore"):
            keep = (z_ < f32(1e-4)) | (tan_a <= np.abs(x_) / np.abs(z_))
    return keep.astype(f32)


def cpp_volume_wedge(w, phi=0.0, psi=0.0, theta=0.0):
    """tom::VolumeWedge::init_wedge_volume (wedge.cpp:330-350): the rotated
    weight volume, ifftshifted (full grid; the reduced form is its first
    nz/2+1 z-planes)."""
    r = cpp_rotate(w, phi, psi, theta)
    return np.fft.ifftshift(r)


def cpp_first_max(v, mask=None):
    """tom::peak (volume_fcn.cpp:505-540, 890-922): the first voxel of the
    maximum in x-fastest order, optionally only where mask != 0."""
    flat = np.asarray(v).ravel(order="F")
    if mask is not None:
        mflat = np.asarray(mask).ravel(order="F") != 0
        cand = np.where(mflat, flat, -np.inf)
        i = int(np.argmax(cand))
    else:
        i = int(np.argmax(flat))
    return np.unravel_index(i, np.shape(v), order="F"), flat[i]


def corr3d_peaks(templates, particles, angles_deg, mask=None, wedge_t=None, wedge_p=None, mask_cc=None):
    """tom_mex_corr3d(size, templates, particles, angles, mask, wedge_ref,
    wedge_part, 'peak', mask_cc) -> tom::corr3d_batch
    (src/mex/tom_mex_corr3d.cpp:700-720, src/tom/corr/corr.cpp:1217-1470) with
    CorrelationHandlerPeaks (src/tom/corr/correlation_handler.cpp:96-120).
    wedge_t / wedge_p: per volume None, ('simple', angle_deg) or
    ('volume', fftshifted weight).  mask_cc is fftshifted.  Returns a dict of
    arrays indexed [template, particle]: peak (0-based x, y, z), val,
    angle_idx (0-based, -1 if none) and second (the best value of the other
    angles, for tie analysis)."""
    shape = np.shape(particles[0])
    numel = int(np.prod(shape))
    nt, npart = len(templates), len(particles)
    ang = np.asarray(angles_deg, np.float64).reshape(-1, 3) * (CPP_PI / 180.0)
    cutoff = (min(shape) - 1) // 2
    lmask = None if mask_cc is None else np.fft.ifftshift(np.asarray(mask_cc))

    def wedge_weight(spec, phi, psi, theta):
        if spec is None:
            return None
        kind, arg = spec
        if kind == "simple":
            a = arg * CPP_PI / 180.0
            if not (a > 0 or cutoff > 0):
                return None
            return cpp_simple_wedge(shape, a, cutoff, phi, psi, theta, reduced=True).astype(np.float64)
        w = np.asarray(arg, np.float64)
        if np.all(w == 1):
            return None
        return cpp_volume_wedge(w.astype(np.float32), phi, psi, theta)[:, :, :shape[2] // 2 + 1].astype(np.float64)

    def var_after(F):
        r = np.fft.irfftn(F, s=shape, axes=(0, 1, 2)) * numel
        return (r * r).sum() / numel / (float(numel) * numel)

    # templates: mean 0, std 1 (population), skipped when the variance is 0
    tn = []
    for t in templates:
        m, vv = cpp_stat(t)
        tn.append(None if not vv else ((np.asarray(t, np.float64) - m) * (1.0 / np.sqrt(vv))).astype(np.float32))
    # particles: norm_mask or mean removal, spectrum with DC 0
    pf, pvar = [], []
    for p in particles:
        if mask is not None:
            q, vv = cpp_norm_mask(p, mask)
        else:
            m, vv = cpp_stat(p)
            q = (np.asarray(p, np.float64) - m).astype(np.float32)
        if not vv:
            pf.append(None)
            pvar.append(0.0)
            continue
        F = np.fft.rfftn(q.astype(np.float64))
        F[0, 0, 0] = 0
        pf.append(F)
        pvar.append(vv)
    res = {"peak": np.zeros((nt, npart, 3), np.int64), "val": np.full((nt, npart), np.nan),
           "angle_idx": np.full((nt, npart), -1, np.int64), "second": np.full((nt, npart), -np.inf)}
    for ia, (phi, psi, theta) in enumerate(ang):
        for it in range(nt):
            if tn[it] is None:
                continue
            r = cpp_rotate(tn[it], phi, psi, theta)
            if mask is not None:
                r, vt0 = cpp_norm_mask(r, mask)
            else:
                m, vt0 = cpp_stat(r)
                r = (r.astype(np.float32) + np.float32(-m)).astype(np.float32)
            TF = np.fft.rfftn(r.astype(np.float64))
            TF[0, 0, 0] = 0
            wt = wedge_weight(None if wedge_t is None else wedge_t[it], phi, psi, theta)
            for ip in range(npart):
                if pf[ip] is None:
                    continue
                vp = pvar[ip]
                PF = pf[ip]
                if wt is not None:
                    PF = PF * wt
                    PF[0, 0, 0] = 0
                    vp = var_after(PF)
                TW = TF
                vt = vt0
                wp = wedge_weight(None if wedge_p is None else wedge_p[ip], 0.0, 0.0, 0.0)
                if wp is not None:
                    TW = TF * wp
                    TW[0, 0, 0] = 0
                    vt = var_after(TW)
                C = TW * np.conj(PF)
                C[0, 0, 0] = 0
                cc = np.fft.irfftn(C, s=shape, axes=(0, 1, 2)) * numel / (np.sqrt(vp * vt) * numel * numel)
                pos, val = cpp_first_max(cc, lmask)
                if val > res["val"][it, ip] or res["angle_idx"][it, ip] < 0:
                    if res["angle_idx"][it, ip] >= 0:
                        res["second"][it, ip] = res["val"][it, ip]
                    res["val"][it, ip] = val
                    res["peak"][it, ip] = pos
                    res["angle_idx"][it, ip] = ia
                else:
                    res["second"][it, ip] = max(res["second"][it, ip], val)
    return res


# ---------------------------------------------------------------------------
# The learned proposer's layers (no reference counterpart): FP64 restatement
# of the convolution, dense layer and losses, for the gradient checks.
# ---------------------------------------------------------------------------
# Volumes [C][Z][Y][X]; weights [Cout][Cin][27], tap t = tx + 3 ty + 9 tz,
# offset (tx-1, ty-1, tz-1) * dilation, zero padding, "same" size.

def cnn_conv3d(x, w, b, dil):
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    ci, Z, Y, X = x.shape
    xp = np.pad(x, ((0, 0), (dil, dil), (dil, dil), (dil, dil)))
    out = np.zeros((w.shape[0], Z, Y, X))
    for t in range(27):
        ox, oy, oz = t % 3, (t // 3) % 3, t // 9
        patch = xp[:, oz * dil:oz * dil + Z, oy * dil:oy * dil + Y, ox * dil:ox * dil + X]
        out += np.einsum("oc,czyx->ozyx", w[:, :, t], patch)
    if b is not None:
        out += np.asarray(b, np.float64)[:, None, None, None]
    return out


def cnn_conv3d_grads(x, w, dil, gout):
    """(d/dx, d/dw, d/db) of sum(gout * conv3d(x, w, b, dil))."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    g = np.asarray(gout, np.float64)
    ci, Z, Y, X = x.shape
    xp = np.pad(x, ((0, 0), (dil, dil), (dil, dil), (dil, dil)))
    gxp = np.zeros_like(xp)
    gw = np.zeros(w.shape)
    for t in range(27):
        ox, oy, oz = t % 3, (t // 3) % 3, t // 9
        sl = (slice(None), slice(oz * dil, oz * dil + Z), slice(oy * dil, oy * dil + Y), slice(ox * dil, ox * dil + X))
        gw[:, :, t] = np.einsum("ozyx,czyx->oc", g, xp[sl])
        gxp[sl] += np.einsum("oc,ozyx->czyx", w[:, :, t], g)
    gx = gxp[:, dil:dil + Z, dil:dil + Y, dil:dil + X]
    return gx, gw, g.sum(axis=(1, 2, 3))


def cnn_bce(logit, target, pos_weight):
    z = np.asarray(logit, np.float64)
    y = np.asarray(target, np.float64)
    sp_neg = np.log1p(np.exp(-np.abs(z))) + np.maximum(-z, 0)
    w = np.where(y > 0, pos_weight, 1.0)
    loss = (w * (y * sp_neg + (1 - y) * (sp_neg + z))).mean()
    grad = w * (1 / (1 + np.exp(-z)) - y) / z.size
    return loss, grad


def cnn_softmax_ce(logits, labels):
    """logits [K][P] -> (mean CE, grad)."""
    l = np.asarray(logits, np.float64)
    m = l.max(axis=0)
    e = np.exp(l - m)
    sm = e / e.sum(axis=0)
    P = l.shape[1]
    lab = np.asarray(labels)
    loss = -np.mean(np.log(sm[lab, np.arange(P)]))
    g = sm.copy()
    g[lab, np.arange(P)] -= 1
    return loss, g / P


# ---------------------------------------------------------------------------
# Angles
# ---------------------------------------------------------------------------

def av3_angle_grid(start, incr, end):
    """Euler triplets in tom_av3_angle2index order (phi fastest, theta slowest),
    inclusive ranges (av3_new/tom_av3_angle2index.m:45-51)."""
    rng = [np.arange(s, e + incr_i * 0.5, incr_i) for s, incr_i, e in zip(start, incr, end)]
    out = [(ph, ps, th) for th in rng[2] for ps in rng[1] for ph in rng[0]]
    return np.array(out, np.float64)


def av3_angle2index(angle, start, incr, end):
    n = [int(round((e - s) / i)) + 1 for s, i, e in zip(start, incr, end)]
    k = [int(round((a - s) / i)) for a, s, i in zip(angle, start, incr)]
    return k[2] * n[0] * n[1] + k[1] * n[0] + k[0]


def av3_index2angle(index, start, incr, end):
    """av3_new/tom_av3_index2angle.m:47-54."""
    n = [(e - s) / i + 1 for s, i, e in zip(start, incr, end)]
    a3 = np.floor(index / (n[0] * n[1]))
    rest = index - a3 * n[0] * n[1]
    a2 = np.floor(rest / n[0])
    a1 = rest - a2 * n[0]
    return np.array([a1, a2, a3]) * np.array(incr) + np.array(start)


# ---------------------------------------------------------------------------
# Peaks
# ---------------------------------------------------------------------------

def tom_peak(a):
    """[c val] = tom_peak(A): first maximum in column-major order, 1-based coordinates."""
    a = np.asarray(a)
    v = a.max()
    flat = np.flatnonzero(np.ravel(a, order="F") == v)[0]
    c = np.unravel_index(flat, a.shape, order="F")
    return tuple(int(x) + 1 for x in c), float(v)


def tom_peak_radius(a, radius):
    """[c val M] = tom_peak(A,R) (Analysis/tom_peak.m:203-279): also zero a ball
    (tom_sphere / tom_circle: distance <= R) around the first maximum."""
    a = np.array(a, dtype=np.float64, copy=True)
    c, v = tom_peak(a)
    g = np.meshgrid(*[np.arange(s) for s in a.shape], indexing="ij")
    d2 = sum((gi - (ci - 1)) ** 2 for gi, ci in zip(g, c))
    a[d2 <= radius * radius] = 0
    return c, v, a


def tom_peak_spline(a):
    """[c val] = tom_peak(A,'spline') via tom_intpeak (Analysis/tom_peak.m:437-525).

    A 3-point not-a-knot spline is the parabola through the points; its
    maximum is searched on the grid 1:0.001:3 like interp1 + max."""
    a = np.asarray(a, np.float64)
    c1, v = tom_peak(a)
    x1 = np.arange(2001) * 0.001 + 1.0
    cs, vals = [], []
    for d in range(a.ndim):
        s = c1[d]
        if s == 1 or s == a.shape[d]:
            cs.append(float(s))
            vals.append(v)
            continue
        idx = [ci - 1 for ci in c1]
        pk = []
        for o in (-1, 0, 1):
            ii = list(idx)
            ii[d] += o
            pk.append(a[tuple(ii)])
        y0, y1, y2 = pk
        # parabola through (1,y0),(2,y1),(3,y2)
        A = (y0 - 2 * y1 + y2) / 2
        B = (y1 - y0) - A * 3
        C = y0 - A - B
        yy = A * x1 * x1 + B * x1 + C
        j = int(np.argmax(yy))
        vals.append(float(yy[j]))
        cs.append(s - 1 + j * 0.001)
    return tuple(cs), max(vals)


def topk_peaks(a, k, radius):
    """Repeated tom_peak(A,R): K peaks, each followed by zeroing a ball of radius R."""
    a = np.array(a, np.float64, copy=True)
    out = []
    for _ in range(k):
        c, v, a = tom_peak_radius(a, radius)
        out.append((c, v))
    return out


# ---------------------------------------------------------------------------
# tom_corr 'norm' and tom_av3_align
# ---------------------------------------------------------------------------

def norm_inside_mask(vol, mask):
    """Analysis/tom_corr.m:98-121 (sample std, n-1)."""
    m = mask != 0
    n = m.sum()
    v = np.asarray(vol, np.float64)
    mea = ((v * m) * (v != 0)).sum() / n
    st = np.sqrt(((((~m) * mea) + (v * m) - mea) ** 2).sum() / (n - 1))
    return ((v - mea) / st) * m, mea, st, n


def tom_corr_norm(a, b, mask, psf1=None, psf2=None):
    """ccf = tom_corr(a,b,'norm',mask[,psf1,psf2]) (Analysis/tom_corr.m:75-95)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if psf1 is not None:
        a = np.fft.ifftn(np.fft.fftn(a) * np.fft.fftn(psf2))
        b = np.fft.ifftn(np.fft.fftn(b) * np.fft.fftn(psf1))
        a = np.real(a)
        b = np.real(b)
    a, _, _, n = norm_inside_mask(a, mask)
    b, _, _, _ = norm_inside_mask(b, mask)
    return np.real(np.fft.fftshift(np.fft.ifftn(np.fft.fftn(b) * np.conj(np.fft.fftn(a))))) / n


def rotmatrix_double(euler_deg):
    """tom_angles2rotmatrix (Sptrans/tom_sum_rotation.m): Rz(psi) Rx(theta) Rz(phi) in double."""
    ph, ps, th = np.deg2rad(np.asarray(euler_deg, np.float64))
    rz = lambda a: np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1.0]])
    rx = np.array([[1, 0, 0], [0, np.cos(th), -np.sin(th)], [0, np.sin(th), np.cos(th)]])
    return rz(ps) @ rx @ rz(ph)


def av3_axis(rng3):
    """MATLAB start:incr:end of one angle axis."""
    s, i, e = [float(x) for x in rng3]
    n = int(np.floor((e - s) / i + 1e-9)) + 1
    return s + i * np.arange(n)


def av3_align(ref, part, phi, psi, theta, mask, mask_ccf, wedge_ref, wedge_part):
    """[angles shifts ccf_peak] = tom_av3_align(ref,part,phi,psi,theta,mask,filter,mask_ccf,wedge_ref,wedge_part)
    with filter.Apply = 0 (av3_new/tom_av3_align.m:97-189), FP64 except rot3d (FP32)."""
    ref = np.asarray(ref, np.float64)
    part = np.asarray(part, np.float64)
    n = ref.shape
    psf_part = np.real(np.fft.ifftn(np.fft.ifftshift(wedge_part)))
    ccf_max = np.full(n, -2.0)
    angle_max = np.full(n, -2.0)
    start = (phi[0], psi[0], theta[0])
    incr = (phi[1], psi[1], theta[1])
    end = (phi[2], psi[2], theta[2])
    for i_phi in av3_axis(phi):
        for i_psi in av3_axis(psi):
            for i_theta in av3_axis(theta):
                R = rotmatrix_double((i_phi, i_psi, i_theta))
                ref_rot = rotate_matrix(ref, R.astype(np.float32).flatten(order="F")).astype(np.float64)
                wrot = rotate(wedge_ref, (i_phi, i_psi, i_theta)).astype(np.float64)
                psf_ref = np.real(np.fft.ifftn(np.fft.ifftshift(wrot)))
                ref_rot = ref_rot * mask
                part = part * mask
                ccf = tom_corr_norm(ref_rot, part, mask, psf_ref, psf_part)
                new_max = np.where(ccf > ccf_max, ccf, ccf_max)
                aidx = av3_angle2index((i_phi, i_psi, i_theta), start, incr, end)
                angle_max = np.where(ccf >= new_max, aidx, angle_max)
                ccf_max = new_max
    pos, _ = tom_peak(ccf_max * mask_ccf)
    ai = angle_max[tuple(p - 1 for p in pos)]
    angles = av3_index2angle(ai, start, incr, end)
    rot_ref = rotate(ref, angles).astype(np.float64)
    ccf_s = tom_corr_norm(rot_ref, part, mask)
    pos, peak = tom_peak_spline(ccf_s * mask_ccf)
    shifts = np.array(pos) - (np.floor(np.array(n) / 2) + 1)
    return angles, shifts, peak, dict(ccf_max=ccf_max, angle_max=angle_max, ccf_s=ccf_s)
