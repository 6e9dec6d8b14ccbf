"""TOM-compatible host API over libtomgpu.

Functions keep the names, argument meaning and return conventions of the
TOM toolbox's MATLAB functions on the template-matching path, so calling code
reads like the reference:

  tom_rotate            Sptrans/tom_rotate.m:89-165 (-> tom_rotatec MEX)
  tom_peak              Analysis/tom_peak.m:80-525 (-> tom_peakinc MEX)
  tom_calc_weight_functioninc  Filtrans/tom_calc_weight_functioninc.c:259-289
  tom_wedge / av3_wedge Filtrans/tom_wedge.m:62-77, av3/utils/av3_wedge.m:23-26
  tom_fourier / tom_ifourier   Filtrans/tom_fourier.m, Filtrans/tom_ifourier.m
  tom_os3_sphereMask    Oscar3/matlabPicker/search/tom_os3_sphereMask.m:4-37
  tom_os3_corr          Oscar3/matlabPicker/search/tom_os3_corr.m:56-192 (FLCF)
  tom_os3_findTemplate  Oscar3/matlabPicker/search/tom_os3_findTemplate.m:157-307
  tom_os3_angleList     Oscar3/matlabPicker/tools/tom_os3_angleList.m:44-97
  tom_av3_angle2index / tom_av3_index2angle  av3_new/tom_av3_angle2index.m, tom_av3_index2angle.m

Volumes are numpy arrays indexed [x, y, z] (MATLAB order).  Every compute
step runs on the GPU through the C ABI; nothing here falls back to the CPU.
Device-resident work (the fast path) goes through :class:`MatchPlan` with
torch CUDA tensors shaped (z, y, x).
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _lib
from ._lib import MatchParams, check, lib

# ---------------------------------------------------------------- context


class Context:
    """A libtomgpu context on one CUDA device (own stream unless set)."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        st = lib().tomgpu_ctx_create(int(device), ctypes.byref(h))
        check(st, None)
        self.handle = h
        self.device = device
        self.use_torch_stream()

    def close(self):
        if self.handle:
            lib().tomgpu_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None):
        check(lib().tomgpu_ctx_set_stream(self.handle, ctypes.c_void_p(stream_ptr or 0)), self.handle)

    def use_torch_stream(self):
        """Issue this context's work on torch's current stream of its device."""
        import torch
        self.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def synchronize(self):
        check(lib().tomgpu_ctx_synchronize(self.handle), self.handle)

    @property
    def launches(self) -> int:
        return int(lib().tomgpu_ctx_launch_count(self.handle))

    def check(self, status):
        check(status, self.handle)

    def profile(self, enable: bool):
        """Start (and reset) or stop the per-kernel-class event timers."""
        self.check(lib().tomgpu_ctx_profile(self.handle, 1 if enable else 0))

    def kernel_times(self):
        """{class name: (total ms, launches)} of the matching loop's kernels."""
        out = {}
        for k, name in enumerate(_lib.KERNEL_CLASSES):
            ms = ctypes.c_double()
            n = ctypes.c_int64()
            self.check(lib().tomgpu_ctx_profile_read(self.handle, k, ctypes.byref(ms), ctypes.byref(n)))
            out[name] = (ms.value, n.value)
        return out


_ctx_lock = threading.Lock()
_default: dict = {}


def default_context(device: int = 0) -> Context:
    with _ctx_lock:
        if device not in _default:
            _default[device] = Context(device)
        return _default[device]


# ---------------------------------------------------------------- helpers

def _dims(a):
    a = np.asarray(a)
    if a.ndim == 2:
        return (a.shape[0], a.shape[1], 1)
    if a.ndim != 3:
        raise ValueError("volume must be 2-D or 3-D")
    return tuple(int(s) for s in a.shape)


def _cdims(d):
    return (ctypes.c_int * 3)(*[int(x) for x in d])


def _f32_xfast(a):
    """Host buffer with x fastest (MATLAB column-major) as float32."""
    return np.asfortranarray(np.asarray(a, dtype=np.float32))


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def to_device(a, device=0):
    """numpy [x, y, z] -> torch CUDA tensor (z, y, x), float32 contiguous."""
    import torch
    a = np.asarray(a, np.float32)
    if a.ndim == 2:
        a = a[:, :, None]
    return torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).to(f"cuda:{device}")


def from_device(t):
    """torch (z, y, x) -> numpy [x, y, z] (a Fortran-ordered view)."""
    return t.detach().cpu().numpy().transpose(2, 1, 0)


def _tptr(t):
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return ctypes.c_void_p(t.data_ptr())


# --------------------------------------------------------------- rotation

def euler_matrix(euler):
    """The 9 floats rm00, rm10, rm20, rm01, rm11, rm21, rm02, rm12, rm22 of tom_rotatec."""
    e = (ctypes.c_float * 3)(*[float(x) for x in np.asarray(euler).reshape(3)])
    m = (ctypes.c_float * 9)()
    check(lib().tomgpu_euler_matrix(e, m))
    return np.array(m[:], np.float32)


def tom_rotatec(in_, out, euler, interp, center, ctx: Context | None = None):
    """MEX form: writes the rotation of in_ into the pre-allocated float32 array out
    (Sptrans/tom_rotatec.c:407-480; 5 inputs, 0 outputs)."""
    if interp != "linear":
        raise ValueError("Unknown interpolation type ... only linear interpolation implemented")
    a = np.asarray(in_)
    if a.dtype != np.float32 or out.dtype != np.float32:
        raise TypeError("Input volumes must be single.")
    if a.shape != out.shape:
        raise ValueError("Volumes must have same size.")
    res = _rotate(a, euler, center, ctx)
    out[...] = res


def _rotate(a, euler, center, ctx):
    ctx = ctx or default_context()
    d = _dims(a)
    src = _f32_xfast(a.reshape(d, order="F") if a.ndim == 2 else a)
    dst = np.zeros(d, np.float32, order="F")
    e = np.asarray(euler, np.float32)
    if e.size == 3:
        mode, buf = _lib.TOMGPU_EULER_DEG, e.reshape(3)
    elif e.size == 9:
        mode, buf = _lib.TOMGPU_MATRIX, np.asarray(e.reshape(3, 3).flatten(order="F"), np.float32)
    else:
        raise ValueError("euler must be [phi psi theta] or a 3x3 matrix")
    buf = np.ascontiguousarray(buf, np.float32)
    c = np.asarray(center, np.float32).reshape(-1)
    if c.size == 2:
        c = np.array([c[0], c[1], 0], np.float32)
    ctx.check(lib().tomgpu_rotate3d(ctx.handle, _ptr(src), _ptr(dst), _cdims(d),
                                    buf.ctypes.data_as(_lib.c_float_p), mode,
                                    np.ascontiguousarray(c, np.float32).ctypes.data_as(_lib.c_float_p)))
    return dst.reshape(a.shape, order="F")


def tom_rotate(in_, euler_angles, interp="linear", center=None, ctx: Context | None = None):
    """out = tom_rotate(in, [phi psi theta] | 3x3, 'linear', [center]) (Sptrans/tom_rotate.m:89-165).
    Default centre ceil(size/2), 0-based.  Returns double like the reference."""
    if interp != "linear":
        raise ValueError("only linear interpolation implemented")
    a = np.asarray(in_)
    if a.ndim != 3:
        raise ValueError("tom_rotate: only 3-D volumes are supported on the GPU path")
    if center is None:
        center = [np.ceil(s / 2) for s in a.shape]
    return _rotate(a, euler_angles, center, ctx).astype(np.float64)


# ------------------------------------------------------------------ peaks

def _peak_host(a, ctx):
    d = _dims(a)
    buf = _f32_xfast(np.asarray(a).reshape(d, order="F"))
    val = ctypes.c_float()
    pos = (ctypes.c_int * 3)(0, 0, 0)
    ctx.check(lib().tomgpu_peak(ctx.handle, _ptr(buf), _cdims(d), ctypes.byref(val), pos))
    return tuple(pos[:]), float(val.value)


def tom_peakc(a, ctx: Context | None = None):
    """[pos val] via the tom_peakinc MEX semantics (strict '>' from -99999, 1-based)."""
    ctx = ctx or default_context()
    pos, val = _peak_host(a, ctx)
    nd = np.asarray(a).ndim
    return pos[:nd], val


def tom_peak(a, *args, ctx: Context | None = None):
    """[c val] = tom_peak(A); [c val] = tom_peak(A,'spline'); [c val M] = tom_peak(A,R);
    [c val M] = tom_peak(A,R,'spline')   (Analysis/tom_peak.m).  3-D volumes."""
    ctx = ctx or default_context()
    A = np.asarray(a, np.float64)
    if A.ndim != 3:
        raise ValueError("tom_peak: 3-D volumes on the GPU path")
    spline = any(isinstance(x, str) and x == "spline" for x in args)
    radius = None
    for x in args:
        if isinstance(x, str):
            if x != "spline":
                raise ValueError("unknown flag " + x)
        else:
            radius = float(x)
    dev = to_device(A, ctx.device)
    d = _cdims(A.shape)
    val = ctypes.c_float()
    pos = (ctypes.c_int * 3)(0, 0, 0)
    ctx.check(lib().tomgpu_peak_dev(ctx.handle, _tptr(dev), d, ctypes.byref(val), pos))
    c = tuple(pos[:])
    v = float(val.value)
    if spline:
        coord = (ctypes.c_double * 3)()
        sv = ctypes.c_double()
        ctx.check(lib().tomgpu_peak_spline_dev(ctx.handle, _tptr(dev), d, pos, coord, ctypes.byref(sv)))
        c, v = tuple(coord[:]), float(sv.value)
    if radius is None:
        return c, v
    # zero the ball around the integer maximum on the device (the spline variant
    # reports the sub-voxel position but zeroes around the integer peak, like
    # the reference)
    vr = ctypes.c_float()
    p1 = (ctypes.c_int * 3)()
    ctx.check(lib().tomgpu_peak_radius_dev(ctx.handle, _tptr(dev), d, float(radius), ctypes.byref(vr), p1))
    ctx.synchronize()
    M = from_device(dev).astype(np.float64)
    return c, v, np.asfortranarray(M)


def topk_peaks(vol_dev, K, radius, ctx: Context | None = None):
    """K peaks of a device volume by repeated tom_peak(A, R) (first maximum, then
    zero the ball of radius R).  Returns (vals[K], pos1[K,3])."""
    ctx = ctx or default_context()
    z, y, x = vol_dev.shape
    vals = (ctypes.c_float * K)()
    pos = (ctypes.c_int * (3 * K))()
    ctx.check(lib().tomgpu_topk_dev(ctx.handle, _tptr(vol_dev), _cdims((x, y, z)), int(K), float(radius), vals, pos))
    return np.array(vals[:], np.float32), np.array(pos[:], np.int32).reshape(K, 3)


# ------------------------------------------------------ weights and masks

def tom_calc_weight_functioninc(dims, angles, thickness, ctx: Context | None = None):
    """Exact (Radermacher) weighting, angles 2 x n (phi; theta) in degrees."""
    ctx = ctx or default_context()
    d = [int(x) for x in dims]
    ang = np.asarray(angles, np.float64)
    if ang.ndim != 2 or ang.shape[0] != 2:
        raise ValueError("angles must be 2 x n_tilt")
    flat = np.ascontiguousarray(ang.T)  # (phi, theta) pairs
    out = np.zeros(d, np.float32, order="F")
    ctx.check(lib().tomgpu_weight3d(ctx.handle, _cdims(d), flat.ctypes.data_as(_lib.c_double_p), flat.shape[0],
                                    float(thickness), _ptr(out)))
    return out


def _wedge(shape, a, b, av3, ctx):
    ctx = ctx or default_context()
    import torch
    d = _dims(np.empty(shape, np.int8))
    out = torch.empty((d[2], d[1], d[0]), dtype=torch.float32, device=f"cuda:{ctx.device}")
    ctx.check(lib().tomgpu_wedge_dev(ctx.handle, _cdims(d), float(a), float(b), int(av3), _tptr(out)))
    return from_device(out).astype(np.float64).reshape(shape, order="F")


def tom_wedge(image, angle, ctx: Context | None = None):
    """Binary missing wedge, 0 where tan(angle) > |x|/|z| (Filtrans/tom_wedge.m:62-77)."""
    return _wedge(np.shape(image), angle, 0.0, 0, ctx)


def av3_wedge(image, minangle, maxangle, ctx: Context | None = None):
    """av3 wedge (av3/utils/av3_wedge.m:23-26)."""
    return _wedge(np.shape(image), minangle, maxangle, 1, ctx)


def tom_os3_sphereMask(template):
    """[mask maskSize] = tom_os3_sphereMask(template): radius floor(min/2)-1 around
    floor(n/2)+1 (1-based), zero where distance >= radius; non-cubic input -> ones."""
    shape = np.shape(template)
    if len(set(shape)) != 1:
        m = np.ones(shape, np.float32)
        return m, int(m.size)
    radius = np.floor(min(shape) / 2) - 1
    center = [np.floor(s / 2) + 1 for s in shape]
    g = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij")
    dist = np.sqrt(sum((gi + 1 - c) ** 2 for gi, c in zip(g, center)))
    m = np.ones(shape, np.float32)
    m[dist >= radius] = 0
    return m, int((m > 0).sum())


def tom_apply_weight_function(in_, w_func, ctx: Context | None = None):
    """out = tom_apply_weight_function(in, w) (Filtrans/tom_apply_weight_function.m:56-62), FP64 on the GPU."""
    ctx = ctx or default_context()
    import torch
    a = np.asarray(in_, np.float32)
    if a.shape != np.shape(w_func):
        raise ValueError("volume and weight differ in size")
    ti, tw = to_device(a, ctx.device), to_device(np.asarray(w_func, np.float32), ctx.device)
    out = torch.empty_like(ti)
    ctx.check(lib().tomgpu_apply_weight_dev(ctx.handle, _tptr(ti), _tptr(tw), _cdims(_dims(a)), _tptr(out)))
    return np.asfortranarray(from_device(out).reshape(a.shape, order="F"))


def tom_emread(path):
    """EM file -> dict(Value=float32 [x,y,z], Header=dict(Size=...)) (IOfun/tom_emread.m)."""
    d = (ctypes.c_int * 3)()
    check(lib().tomgpu_em_read(str(path).encode(), d, None, 0))
    vol = np.zeros(tuple(d), np.float32, order="F")
    check(lib().tomgpu_em_read(str(path).encode(), d, _ptr(vol), vol.size))
    return {"Value": vol, "Header": {"Size": tuple(d)}}


def tom_emwrite(path, data, comment: str = ""):
    """Write a float32 EM file (IOfun/tom_emwrite.m), PC byte order."""
    a = _f32_xfast(np.asarray(data.get("Value") if isinstance(data, dict) else data))
    if a.ndim == 2:
        a = a.reshape(a.shape + (1,), order="F")
    check(lib().tomgpu_em_write(str(path).encode(), _ptr(a), _cdims(a.shape), comment.encode()[:80]))


def tom_fourier(a, ctx: Context | None = None):
    """fftn in FP64 on the GPU (Filtrans/tom_fourier.m)."""
    return _fft(a, -1, ctx)


def tom_ifourier(a, ctx: Context | None = None):
    """ifftn in FP64 on the GPU (Filtrans/tom_ifourier.m)."""
    return _fft(a, +1, ctx)


def _fft(a, direction, ctx):
    import torch
    ctx = ctx or default_context()
    A = np.asarray(a, np.complex128)
    shape = A.shape
    d = _dims(A)
    t = torch.from_numpy(np.ascontiguousarray(A.reshape(d, order="F").transpose(2, 1, 0))).to(f"cuda:{ctx.device}")
    t = torch.view_as_real(t).contiguous()
    ctx.check(lib().tomgpu_fft3d_c2c_dev(ctx.handle, _tptr(t), _cdims(d), int(direction), 64))
    ctx.synchronize()
    out = torch.view_as_complex(t).cpu().numpy().transpose(2, 1, 0)
    return out.reshape(shape, order="F")


# ---------------------------------------------------------------- angles

def _rotmatrix(phi, psi, theta):
    """tom_angles2rotmatrix (Sptrans/tom_sum_rotation.m): Rz(psi) Rx(theta) Rz(phi), double,
    with the reference's degree conversion a .* pi ./ 180 (in that order)."""
    ph, ps, th = (np.asarray([phi, psi, theta], np.float64) * np.pi) / 180
    rz = lambda a: np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])
    rx = np.array([[1, 0, 0], [0, np.cos(th), -np.sin(th)], [0, np.sin(th), np.cos(th)]])
    return rz(ps) @ rx @ rz(ph)


def _os3_axis(start, inc, end):
    """One axis of tom_os3_angleList (search/tom_os3_angleList.m, dim 2).
    start < end: start:inc:end mod 360.  Otherwise the reference walks
    start+1:inc:end+359 into a result preallocated with
    floor((360+end-start)/inc)+1 zeros, so when the walk is one step shorter
    (e.g. 300 -> 60 by 30: 301 331 1 31) the list keeps a trailing 0."""
    if start < end:
        vals = []
        i = start
        while i <= end + 1e-9:
            vals.append(np.mod(i, 360))
            i += inc
        return vals
    vals = []
    i = start + 1
    while i <= end + 360 - 1 + 1e-9:
        vals.append(np.mod(i, 360))
        i += inc
    size = int(np.floor((360 + end - start) / inc)) + 1
    return vals + [0.0] * max(0, size - len(vals))


def tom_os3_angleList(start, increment, end, dedup=True):
    """3-D angle list of tom_os3_angleList: phi outer, psi, theta inner; equivalent
    rotations (equal floor(R*1e4)) dropped.  Returns N x 3 [phi psi theta]."""
    phis = _os3_axis(start[0], increment[0], end[0])
    psis = _os3_axis(start[1], increment[1], end[1])
    ths = _os3_axis(start[2], increment[2], end[2])
    out, seen = [], set()
    for ph in phis:
        for ps in psis:
            for th in ths:
                if dedup:
                    key = tuple(np.floor(_rotmatrix(ph, ps, th) * 10000).astype(np.int64).ravel())
                    if key in seen:
                        continue
                    seen.add(key)
                out.append((ph, ps, th))
    return np.array(out, np.float64)


def tom_av3_angle_grid(start, incr, end):
    """Triplets in tom_av3_angle2index order: phi fastest, theta slowest, inclusive."""
    axes = [np.arange(s, e + i * 0.5, i) for s, i, e in zip(start, incr, end)]
    return np.array([(ph, ps, th) for th in axes[2] for ps in axes[1] for ph in axes[0]], np.float64)


def tom_av3_angle2index(angle, angle_start, angular_incr, angle_end):
    n = [int(round((e - s) / i)) + 1 for s, i, e in zip(angle_start, angular_incr, angle_end)]
    k = [int(round((a - s) / i)) for a, s, i in zip(angle, angle_start, angular_incr)]
    for kk, nn in zip(k, n):
        if kk < 0 or kk >= nn:
            return int(np.prod(n))  # the reference's loop runs to the end without a match
    return k[2] * n[0] * n[1] + k[1] * n[0] + k[0]


def tom_av3_index2angle(index, angle_start, angular_incr, angle_end):
    n = [(e - s) / i + 1 for s, i, e in zip(angle_start, angular_incr, angle_end)]
    a3 = np.floor(index / (n[0] * n[1]))
    rest = index - a3 * n[0] * n[1]
    a2 = np.floor(rest / n[0])
    a1 = rest - a2 * n[0]
    return np.array([a1, a2, a3]) * np.asarray(angular_incr) + np.asarray(angle_start)


# ------------------------------------------------------------- matching

class MatchPlan:
    """Device-resident FLCF search for one tomogram size and one template size.

    Tensors are torch CUDA float32, shaped (z, y, x).  Usage mirrors
    tom_os3_findTemplate: set_template (template, mask, optional psf) ->
    set_volume -> init_results -> run(eulers) [repeat] -> results.  A later
    set_template with the same mask keeps the volume; after one with another
    mask, set_volume again (run raises TomGpuError TOMGPU_ERR_STATE until then).
    """

    def __init__(self, vol_shape_xyz, tmpl_shape_xyz, batch: int = 0, ctx: Context | None = None,
                 generic: bool = False, path: int | None = None):
        self.ctx = ctx or default_context()
        self.vol_shape = tuple(int(s) for s in vol_shape_xyz)
        self.tmpl_shape = tuple(int(s) for s in tmpl_shape_xyz)
        p = MatchParams()
        p.batch = int(batch)
        p.path = int(path) if path is not None else (1 if generic else 0)
        h = ctypes.c_void_p()
        self.ctx.check(lib().tomgpu_match_plan_create(self.ctx.handle, _cdims(self.vol_shape),
                                                      _cdims(self.tmpl_shape), ctypes.byref(p), ctypes.byref(h)))
        self.handle = h
        self._keep = []

    def close(self):
        if getattr(self, "handle", None):
            lib().tomgpu_match_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def bytes(self):
        return int(lib().tomgpu_match_plan_bytes(self.handle))

    def set_template(self, tmpl_dev, mask_dev, psf_dev=None):
        self._keep = [tmpl_dev, mask_dev, psf_dev]
        self.ctx.check(lib().tomgpu_match_set_template_dev(self.handle, _tptr(tmpl_dev), _tptr(mask_dev),
                                                           _tptr(psf_dev) if psf_dev is not None else None))

    def autotune(self, eulers, candidates=(8, 16, 32)):
        """Pick the rotation batch with the fastest per-rotation time on these
        rotations (the plan keeps it); returns (best, {batch: ms per rotation})."""
        e = np.ascontiguousarray(np.asarray(eulers, np.float32).reshape(-1, 3))
        c = np.ascontiguousarray(np.asarray(candidates, np.int32))
        ms = np.zeros(len(c), np.float32)
        best = ctypes.c_int(0)
        self.ctx.check(lib().tomgpu_match_autotune(self.handle, e.ctypes.data_as(_lib.c_float_p), e.shape[0],
                                                   c.ctypes.data_as(_lib.c_int_p), len(c), ctypes.byref(best),
                                                   ms.ctypes.data_as(_lib.c_float_p)))
        return best.value, {int(b): float(m) for b, m in zip(c, ms) if m > 0}

    def set_template_raw(self, tmpl_dev, mask_dev):
        """Template statistics of this template as given (tom_os3_corr without cached statistics)."""
        self._keep = [tmpl_dev, mask_dev]
        self.ctx.check(lib().tomgpu_match_set_template_raw_dev(self.handle, _tptr(tmpl_dev), _tptr(mask_dev)))

    def set_volume(self, vol_dev):
        self.ctx.check(lib().tomgpu_match_set_volume_dev(self.handle, _tptr(vol_dev)))

    def new_analysis_results(self):
        """(maxcc, angidx, psr, autoc) device buffers, initialised like findTemplate."""
        import torch
        x, y, z = self.vol_shape
        dev = f"cuda:{self.ctx.device}"
        cc = torch.empty((z, y, x), dtype=torch.float32, device=dev)
        idx = torch.empty((z, y, x), dtype=torch.int32, device=dev)
        psr = torch.empty_like(cc)
        soc = torch.empty_like(cc)
        self.ctx.check(lib().tomgpu_match_init_analysis_dev(self.handle, _tptr(cc), _tptr(idx), _tptr(psr), _tptr(soc)))
        return cc, idx, psr, soc

    def run_analysis(self, eulers, maxcc_dev, angidx_dev, psr_dev, autoc_dev, ccc=True, psr=False,
                     autocorr=False, index_offset: int = 0):
        """Per-rotation FLCF, PSR and autocorrelation maps with tom_os3_bestPeak's
        update on the selected criteria (tom_os3_findTemplate's own loop)."""
        flags = (1 if ccc else 0) | (2 if psr else 0) | (4 if autocorr else 0)
        e = np.ascontiguousarray(np.asarray(eulers, np.float32).reshape(-1, 3))
        self.ctx.check(lib().tomgpu_match_run_analysis_dev(self.handle, e.ctypes.data_as(_lib.c_float_p), e.shape[0],
                                                           int(index_offset), flags, _tptr(maxcc_dev),
                                                           _tptr(angidx_dev), _tptr(psr_dev), _tptr(autoc_dev)))

    def new_results(self):
        import torch
        x, y, z = self.vol_shape
        cc = torch.empty((z, y, x), dtype=torch.float32, device=f"cuda:{self.ctx.device}")
        idx = torch.empty((z, y, x), dtype=torch.int32, device=f"cuda:{self.ctx.device}")
        self.ctx.check(lib().tomgpu_match_init_results_dev(self.handle, _tptr(cc), _tptr(idx)))
        return cc, idx

    def init_results(self, maxcc_dev, angidx_dev):
        """Reset result buffers of the volume's size (-1000 / -1), as new_results."""
        self.ctx.check(lib().tomgpu_match_init_results_dev(self.handle, _tptr(maxcc_dev), _tptr(angidx_dev)))

    def run(self, eulers, maxcc_dev, angidx_dev, index_offset: int = 0):
        e = np.ascontiguousarray(np.asarray(eulers, np.float32).reshape(-1, 3))
        self.ctx.check(lib().tomgpu_match_run_dev(self.handle, e.ctypes.data_as(_lib.c_float_p), e.shape[0],
                                                  int(index_offset), _tptr(maxcc_dev), _tptr(angidx_dev)))

    def corr(self, t_dev, out_dev):
        self.ctx.check(lib().tomgpu_match_corr_dev(self.handle, _tptr(t_dev), _tptr(out_dev)))

    def rescore_fp64(self, vol_dev, eulers, pos1):
        """FP64 direct-sum FLCF of candidates (eulers K x 3 degrees, pos1 K x 3 1-based)."""
        e = np.ascontiguousarray(np.asarray(eulers, np.float32).reshape(-1, 3))
        p = np.ascontiguousarray(np.asarray(pos1, np.int32).reshape(-1, 3))
        out = np.zeros(len(e), np.float64)
        self.ctx.check(lib().tomgpu_match_rescore_fp64_dev(
            self.handle, _tptr(vol_dev), e.ctypes.data_as(_lib.c_float_p), p.ctypes.data_as(_lib.c_int_p), len(e),
            out.ctypes.data_as(_lib.c_double_p)))
        return out

    def stats(self):
        import torch
        x, y, z = self.vol_shape
        m = torch.empty((z, y, x), dtype=torch.float32, device=f"cuda:{self.ctx.device}")
        s = torch.empty_like(m)
        self.ctx.check(lib().tomgpu_match_stats_dev(self.handle, _tptr(m), _tptr(s)))
        return m, s


def pick_peaks(maxcc_dev, angidx_dev, K, radius, ctx: Context | None = None):
    """Top-K candidates of a search: K rounds of tom_peak(A, R) on the max-CC
    volume (first maximum, then zero a ball of radius R), with the angle index
    recorded at each peak (tom_os3_returnPicklist.m's loop).  Returns
    (vals[K], pos1[K,3] 1-based [x,y,z], angle index[K] 0-based)."""
    vals, pos = topk_peaks(maxcc_dev, K, radius, ctx)
    p0 = pos - 1
    ok = (pos[:, 0] > 0)
    idx = np.full(K, -1, np.int64)
    if ok.any():
        import torch
        zz, yy, xx = (torch.as_tensor(p0[ok, 2]), torch.as_tensor(p0[ok, 1]), torch.as_tensor(p0[ok, 0]))
        idx[ok] = angidx_dev[zz.to(angidx_dev.device), yy.to(angidx_dev.device), xx.to(angidx_dev.device)].cpu().numpy()
    return vals, pos, idx


def picklist_to_motl(vals, pos1, eulers, class_no=0):
    """MOTL (20 x n) of a pick list, av3/alignment/av3_tomomatch.m:48-70 layout:
    row 1 CCC, 4 particle number, 8-10 x/y/z (1-based), 17-19 phi/psi/theta, 20 class."""
    n = len(vals)
    m = np.zeros((20, n))
    m[0] = vals
    m[3] = np.arange(1, n + 1)
    m[7:10] = np.asarray(pos1, np.float64).T
    m[16:19] = np.asarray(eulers, np.float64).reshape(-1, 3).T
    m[19] = class_no
    return m


def match_host(tomo, template, mask, eulers, psf=None, batch: int = 0, ctx: Context | None = None):
    """One-shot search through the C ABI with host buffers (tomgpu_match): returns
    (maxcc float32 [x,y,z], angle index int32 [x,y,z], 0-based, -1 where unset)."""
    ctx = ctx or default_context()
    vol = _f32_xfast(tomo)
    t = _f32_xfast(template)
    m = _f32_xfast(mask)
    p = _f32_xfast(psf) if psf is not None else None
    e = np.ascontiguousarray(np.asarray(eulers, np.float32).reshape(-1, 3))
    cc = np.zeros(vol.shape, np.float32, order="F")
    idx = np.zeros(vol.shape, np.int32, order="F")
    prm = MatchParams()
    prm.batch = int(batch)
    ctx.check(lib().tomgpu_match(ctx.handle, _ptr(vol), _cdims(vol.shape), _ptr(t), _cdims(t.shape), _ptr(m),
                                 _ptr(p) if p is not None else None, e.ctypes.data_as(_lib.c_float_p), e.shape[0],
                                 ctypes.byref(prm), _ptr(cc), _ptr(idx)))
    return cc, idx


def tom_os3_findTemplate(volume, template, angle_list, mask=None, psf=None, batch: int = 0,
                         analysis=None, ctx: Context | None = None):
    """[ccc angles] of tom_os3_findTemplate for in-memory inputs (the job/file
    plumbing of the reference is out of scope): template normalised with
    tom_norm(1e5*(t+1),'mean0+1std'), mask = tom_os3_sphereMask(template) when
    not given, psf = optional centred weight.  Returns ccc (float32 [x,y,z],
    -1000 where never updated) and angles (1-based angle-list index as float32,
    -1000 where never updated), the reference's conventions.

    analysis: None runs the fast search (options.analysis.ccc alone, the
    only output ccc/angles).  A dict like options.analysis, e.g.
    {'ccc': 1, 'psr': 1, 'autocorr': 0}, runs the reference's own loop with
    the PSR and autocorrelation maps of every rotation and tom_os3_bestPeak's
    update on the selected criteria, and returns (ccc, angles, psr, autoc)
    (result.ccc/.angles/.psr/.autoc)."""
    ctx = ctx or default_context()
    import torch
    vol = np.asarray(volume, np.float32)
    t = np.asarray(template, np.float32)
    if mask is None:
        mask, _ = tom_os3_sphereMask(t)
    if not np.any(vol):
        # tom_os3_findTemplate.m:221 and :309-313: a volume with mean 0 and
        # std 0 is not searched; ccc, psr and autoc are 0 and the angle map keeps -1000
        z = np.zeros(vol.shape, np.float32, order="F")
        ang = np.full(vol.shape, -1000, np.float32, order="F")
        return (z, ang) if analysis is None else (z, ang, z.copy(order="F"), z.copy(order="F"))
    plan = MatchPlan(vol.shape, t.shape, batch=batch, ctx=ctx)
    try:
        td, md = to_device(t, ctx.device), to_device(mask, ctx.device)
        pd = to_device(psf, ctx.device) if psf is not None else None
        plan.set_template(td, md, pd)
        plan.set_volume(to_device(vol, ctx.device))
        if analysis is None:
            cc, idx = plan.new_results()
            plan.run(angle_list, cc, idx)
            extra = ()
        else:
            flags = {k: bool(analysis.get(k, 0)) for k in ("ccc", "psr", "autocorr")}
            if not any(flags.values()):
                raise ValueError("analysis selects none of ccc, psr, autocorr")
            cc, idx, pm, am = plan.new_analysis_results()
            plan.run_analysis(angle_list, cc, idx, pm, am, **flags)
            extra = (pm, am)
        torch.cuda.synchronize(ctx.device)
        ccc = from_device(cc)
        ang = from_device(idx).astype(np.float32)
        ang = np.where(ang >= 0, ang + 1, -1000).astype(np.float32)
        out = (np.asfortranarray(ccc), np.asfortranarray(ang))
        return out + tuple(np.asfortranarray(from_device(e)) for e in extra)
    finally:
        plan.close()


def tom_os3_analyzePeak(img, peakMap, template, options, ctx: Context | None = None):
    """res = tom_os3_analyzePeak(img, peakMap, template, options) for
    options['analysis']['type'] 'PSR' or 'Autocorrelation'
    (Oscar3/matlabPicker/analyze/tom_os3_analyzePeak.m:61-101,174-190).
    options['correlation']['mask'] (template-sized) is the mask of the
    autocorrelation FLCF (tom_os3_sphereMask(template) when absent)."""
    import torch
    ctx = ctx or default_context()
    kind = options["analysis"]["type"]
    pk = np.asarray(peakMap, np.float32)
    t = np.asarray(template, np.float32)
    pd = to_device(pk, ctx.device)
    out = torch.empty_like(pd)
    if kind == "PSR":
        ctx.check(lib().tomgpu_analyze_psr_dev(ctx.handle, _tptr(pd), _cdims(pk.shape), _cdims(t.shape), _tptr(out)))
    elif kind == "Autocorrelation":
        mask = options.get("correlation", {}).get("mask")
        md = to_device(np.asarray(mask, np.float32), ctx.device) if mask is not None else None
        ctx.check(lib().tomgpu_analyze_autocorr_dev(ctx.handle, _tptr(pd), _cdims(pk.shape),
                                                    _tptr(to_device(t, ctx.device)), _cdims(t.shape),
                                                    _tptr(md) if md is not None else None, _tptr(out)))
    else:
        raise ValueError("analysis type must be 'PSR' or 'Autocorrelation'")
    ctx.synchronize()
    return np.asfortranarray(from_device(out))


def tom_os3_template_autocorr(template, ctx: Context | None = None):
    """tom_os3_corr(template, template) (same-size FLCF, default sphere mask)."""
    import torch
    ctx = ctx or default_context()
    t = np.asarray(template, np.float32)
    td = to_device(t, ctx.device)
    out = torch.empty_like(td)
    ctx.check(lib().tomgpu_template_autocorr_dev(ctx.handle, _tptr(td), _cdims(t.shape), _tptr(out)))
    ctx.synchronize()
    return np.asfortranarray(from_device(out))


def tom_os3_corr(img, template, options=None, ctx: Context | None = None):
    """FLCF map of one (already rotated, masked, filtered) template against img
    (search/tom_os3_corr.m FLCF branch).  options is a dict that caches the
    search statistics between calls like the reference's options.correlation:
    keys 'mask' (template-sized); the template statistics are those of
    findTemplate's preprocessing of options['template'] when given, else
    tom_os3_normUnderMask of this template (calculationAvailable false)."""
    import torch
    ctx = ctx or default_context()
    options = {} if options is None else options
    t = np.asarray(template, np.float32)
    vol = np.asarray(img, np.float32)
    mask = options.get("mask")
    if mask is None:
        mask, _ = tom_os3_sphereMask(t)
        options["mask"] = mask
    plan = options.get("_plan")
    if plan is None or plan.vol_shape != vol.shape or plan.tmpl_shape != t.shape:
        plan = MatchPlan(vol.shape, t.shape, ctx=ctx)
        if options.get("template") is not None:
            # statistics cached from findTemplate's preprocessed template
            plan.set_template(to_device(options["template"], ctx.device), to_device(mask, ctx.device),
                              to_device(options["psf"], ctx.device) if options.get("psf") is not None else None)
        else:
            plan.set_template_raw(to_device(t, ctx.device), to_device(mask, ctx.device))
        plan.set_volume(to_device(vol, ctx.device))
        options["_plan"] = plan
    out = torch.empty((vol.shape[2], vol.shape[1], vol.shape[0]), dtype=torch.float32, device=f"cuda:{ctx.device}")
    plan.corr(to_device(t, ctx.device), out)
    ctx.synchronize()
    return np.asfortranarray(from_device(out)), options


# ------------------------------------------------------ subtomogram alignment

def av3_average_add(particles, wedges, shifts, angles, average=None, wei=None, ctx: Context | None = None):
    """Accumulate the averaging step of av3_tomomatch (av3/alignment/av3_tomomatch.m:239-249):
    average += tom_rotate(tom_shift(p, -shift), [-psi -phi -theta]) and
    wei += (tom_rotate(wedge, [-psi -phi -theta]) >= 0.5) for each particle in
    order.  particles/wedges: lists of same-sized volumes ([x,y,z]);
    shifts: K x 3 (motl rows 11-13); angles: K x 3 phi, psi, theta (rows 17-19).
    Returns the device sums (float64 tensors [z,y,x]), to pass back in for
    more particles and to av3_average_final."""
    import torch
    ctx = ctx or default_context()
    K = len(particles)
    shape = np.shape(particles[0]) if K else np.shape(average)
    x, y, z = shape
    dev = f"cuda:{ctx.device}"
    if average is None:
        average = torch.zeros((z, y, x), dtype=torch.float64, device=dev)
        wei = torch.zeros_like(average)
    if K == 0:
        return average, wei
    pd = [to_device(np.asarray(p, np.float32), ctx.device) for p in particles]
    wcache = {}
    wd = []
    for w in wedges:
        key = id(w)
        if key not in wcache:
            wcache[key] = to_device(np.asarray(w, np.float32), ctx.device)
        wd.append(wcache[key])
    sh = np.asarray(shifts, np.float32).reshape(K, 3)
    an = np.asarray(angles, np.float32).reshape(K, 3)
    items = (_lib.AvgItem * K)()
    for k in range(K):
        items[k].particle = _tptr(pd[k])
        items[k].wedge = _tptr(wd[k])
        items[k].shift[:] = [float(v) for v in sh[k]]
        items[k].angles[:] = [float(v) for v in an[k]]
    ctx.check(lib().tomgpu_av3_average_add_dev(ctx.handle, _cdims(shape), items, K, _tptr(average), _tptr(wei)))
    return average, wei


def av3_average_final(average, wei, ctx: Context | None = None):
    """The weighting that ends an av3_tomomatch iteration (av3_tomomatch.m:263-265),
    FP64: returns the new reference ([x,y,z] float64)."""
    import torch
    ctx = ctx or default_context()
    z, y, x = average.shape
    out = torch.empty_like(average)
    ctx.check(lib().tomgpu_av3_average_final_dev(ctx.handle, _cdims((x, y, z)), _tptr(average), _tptr(wei),
                                                 _tptr(out)))
    ctx.synchronize()
    return np.asfortranarray(from_device(out))


def av3_tomomatch_average(particles, motl, wedgelist, threshold, iclass=0, meanv=None,
                          ctx: Context | None = None):
    """The selection and averaging of one av3_tomomatch iteration for an aligned
    motive list (av3_tomomatch.m:117-118,157-158,239-265).  particles[p] is the
    volume of motl column p; wedgelist is 3 x W (tomogram number, min and max
    tilt).  Particles of class 1, 2 or iclass whose CCC (row 1) exceeds
    threshold * meanv (meanv: mean CCC of those classes, computed from this
    motl unless given) are averaged and get class 1; the others of those
    classes get class 2.  Returns (average, wei, motl)."""
    motl = np.array(motl, np.float64, copy=True)
    sel = (motl[19] == 1) | (motl[19] == 2) | (motl[19] == iclass)
    if meanv is None:
        meanv = float(np.mean(motl[0, sel])) if sel.any() else 0.0
    wl = np.asarray(wedgelist, np.float64).reshape(3, -1)
    wedges = {}
    P, W, S, A = [], [], [], []
    for p in np.nonzero(sel)[0]:
        if motl[0, p] > threshold * meanv:
            itomo = motl[4, p]
            if itomo not in wedges:
                col = np.nonzero(wl[0] == itomo)[0][0]
                wedges[itomo] = av3_wedge(np.zeros(np.shape(particles[p])), wl[1, col], wl[2, col], ctx=ctx)
            part = np.asarray(particles[p], np.float64)
            part = np.where(part < -3, 0.0, np.minimum(part, 4.0))   # tom_limit(particle, -3, 4, 'z')
            P.append(part)
            W.append(wedges[itomo])
            S.append(motl[10:13, p])
            A.append(motl[16:19, p])
            motl[19, p] = 1
        else:
            motl[19, p] = 2
    avg, wei = av3_average_add(P, W, S, A, ctx=ctx) if P else av3_average_add(
        [], [], [], [], *_zero_sums(np.shape(particles[0]), ctx), ctx=ctx)
    return av3_average_final(avg, wei, ctx=ctx), np.asfortranarray(from_device(wei)), motl


def _zero_sums(shape, ctx):
    import torch
    ctx = ctx or default_context()
    x, y, z = shape
    a = torch.zeros((z, y, x), dtype=torch.float64, device=f"cuda:{ctx.device}")
    return a, torch.zeros_like(a)


def cpp_spheremask(shape, radius):
    """tom::init_spheremask(mask, radius, 0, 0): 1 where the squared distance
    from n/2 (integer centre) is <= radius^2, float arithmetic
    (Oscar3/c++Picker/src/tom/core/volume_fcn.cpp:979-1028)."""
    f32 = np.float32
    g = np.meshgrid(*[np.arange(n, dtype=f32) - f32(n // 2) for n in shape], indexing="ij")
    d2 = (g[0] * g[0] + (g[1] * g[1] + g[2] * g[2])).astype(f32)
    r = f32(max(radius, 0.0))
    return np.asfortranarray((d2 <= r * r).astype(f32) if r > 0 else np.zeros(shape, f32))


def tom_corr3d(templates, particles, angles, mask=None, wedge_ref=None, wedge_part=None, mask_cc=None,
               ctx: Context | None = None):
    """[out] = tom_mex_corr3d(size, templates, particles, angles, mask, wedge_ref,
    wedge_part, 'peak', mask_cc) (Oscar3/c++Picker/src/mex/tom_mex_corr3d.cpp),
    the C++ picker's batched aligner on the GPU.

    templates / particles: lists of same-sized volumes [x,y,z]; angles: R x 3
    [phi psi theta] degrees; mask: None, a radius (tom::init_spheremask) or a
    volume; wedge_ref / wedge_part: None ([]), one spec for all or a list of
    specs, a spec being None, an angle in degrees (SimpleWedge) or an
    fftshifted weight volume; mask_cc: None, a radius or an fftshifted volume.
    Returns an nt x np object array of dicts with the MEX's fields: peak
    (0-based [x y z]), ncc_val, angle (degrees), angle_idx (1-based)."""
    ctx = ctx or default_context()
    shape = tuple(np.shape(particles[0]))
    nt, npart = len(templates), len(particles)
    keep = []

    def dev(a):
        t = to_device(np.asarray(a, np.float32), ctx.device)
        keep.append(t)
        return t

    def vol_or_radius(m):
        if m is None:
            return None
        if np.ndim(m) == 0:
            return dev(cpp_spheremask(shape, float(m)))
        return dev(m)

    tp = (ctypes.c_void_p * nt)(*[_tptr(dev(t)).value for t in templates])
    pp = (ctypes.c_void_p * npart)(*[_tptr(dev(p)).value for p in particles])
    ang = np.ascontiguousarray(np.asarray(angles, np.float64).reshape(-1, 3))
    md, mcd = vol_or_radius(mask), vol_or_radius(mask_cc)

    def specs(w, count):
        if w is None:
            return None
        items = list(w) if isinstance(w, (list, tuple)) else [w] * count
        if len(items) == 1 and count > 1:
            items = items * count
        if len(items) != count:
            raise ValueError("one wedge for all volumes or one per volume")
        arr = (_lib.WedgeSpec * count)()
        for i, it in enumerate(items):
            if it is None:
                arr[i].kind = 0
            elif np.ndim(it) == 0:
                arr[i].kind, arr[i].angle_deg = 1, float(it)
            else:
                arr[i].kind, arr[i].volume = 2, _tptr(dev(it))
        return arr

    wt, wp = specs(wedge_ref, nt), specs(wedge_part, npart)
    peak = np.zeros((npart, nt, 3), np.float64)
    val = np.zeros((npart, nt), np.float64)
    idx = np.zeros((npart, nt), np.int32)
    ctx.check(lib().tomgpu_corr3d_peaks_dev(ctx.handle, _cdims(shape), tp, nt, pp, npart,
                                            ang.ctypes.data_as(_lib.c_double_p), len(ang),
                                            _tptr(md) if md is not None else None, wt, wp,
                                            _tptr(mcd) if mcd is not None else None,
                                            peak.ctypes.data_as(_lib.c_double_p), val.ctypes.data_as(_lib.c_double_p),
                                            idx.ctypes.data_as(_lib.c_int_p)))
    out = np.empty((nt, npart), dtype=object)
    for j in range(npart):
        for i in range(nt):
            k = int(idx[j, i])
            out[i, j] = {"peak": peak[j, i].copy(), "ncc_val": float(val[j, i]),
                         "angle": ang[k - 1].copy() if k > 0 else np.full(3, np.nan), "angle_idx": k}
    return out


def tom_spheremask_default(shape):
    """tom_spheremask(ones(n)) with the default radius floor((min(n)-1)/2) (Geom/tom_spheremask.m:41-67)."""
    shape = tuple(shape)
    radius = np.floor((min(shape) - 1) / 2)
    center = [np.floor(s / 2) + 1 for s in shape]
    g = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij")
    d = np.sqrt(sum((gi + 1 - c) ** 2 for gi, c in zip(g, center)))
    m = np.ones(shape, np.float32)
    m[d >= radius] = 0
    return m


def tom_corr(a, b, *args, ctx: Context | None = None):
    """ccf = tom_corr(a, b) | tom_corr(a, b, 'norm', mask) | tom_corr(a, b, 'norm', mask, psf1, psf2)
    (Analysis/tom_corr.m) on the GPU; returns a float32 volume [x, y, z]."""
    import torch
    ctx = ctx or default_context()
    A = np.asarray(a, np.float32)
    mask = psf1 = psf2 = None
    if args:
        if args[0] != "norm":
            raise ValueError("only the 'norm' flag is implemented")
        if len(args) not in (2, 4):
            raise ValueError("tom_corr(a, b, 'norm', mask[, psf1, psf2])")
        mask = args[1]
        if len(args) == 4:
            psf1, psf2 = args[2], args[3]
    dev = lambda x: None if x is None else to_device(np.asarray(x, np.float32), ctx.device)
    ta, tb_, tm, p1, p2 = dev(A), dev(b), dev(mask), dev(psf1), dev(psf2)
    out = torch.empty_like(ta)
    ptr = lambda t: _tptr(t) if t is not None else None
    ctx.check(lib().tomgpu_corr_dev(ctx.handle, _tptr(ta), _tptr(tb_), _cdims(A.shape), ptr(tm), ptr(p1), ptr(p2),
                                    _tptr(out)))
    ctx.synchronize()
    return np.asfortranarray(from_device(out))


def av3_align_batch(jobs, ctx: Context | None = None, path: int = 0, batch_bytes: int = 0, timings=None):
    """Run tom_av3_align jobs on the GPU.  Each job is a dict with numpy
    volumes 'ref', 'part', 'mask' (None: tom_spheremask default), 'mask_ccf'
    (None: ones), 'wedge_ref', 'wedge_part' (None: no wedges / same as
    wedge_ref) and angle ranges 'phi', 'psi', 'theta' ([start incr end]).
    path 0 batches the jobs of each compiled cubic edge, path 1 runs every job
    alone; batch_bytes bounds a batch's spectra (0: the library default).
    timings: an optional dict that receives the seconds of the uploads
    ('upload_s') and of the library call ('call_s').
    Returns (angles[n,3], shifts[n,3], ccf_peak[n])."""
    import time
    import torch
    ctx = ctx or default_context()
    t0 = time.perf_counter()
    arr = (_lib.AlignJob * len(jobs))()
    keep = []
    uploaded = {}  # id(array) -> (array, device tensor): a volume shared by jobs is uploaded once

    def dev(a):
        if a is None:
            return None
        hit = uploaded.get(id(a))
        if hit is not None and hit[0] is a:
            return hit[1]
        t = to_device(np.asarray(a, np.float32), ctx.device)
        uploaded[id(a)] = (a, t)
        return t

    for j, jb in enumerate(jobs):
        ref = jb["ref"]
        n = np.shape(ref)
        mask = jb.get("mask")
        mask = tom_spheremask_default(n) if mask is None else mask
        t = dict(ref=dev(ref), part=dev(jb["part"]), mask=dev(mask), mask_ccf=dev(jb.get("mask_ccf")),
                 wedge_ref=dev(jb.get("wedge_ref")), wedge_part=dev(jb.get("wedge_part")))
        keep.append(t)
        arr[j].n = (ctypes.c_int * 3)(*n)
        for k in ("ref", "part", "mask", "mask_ccf", "wedge_ref", "wedge_part"):
            setattr(arr[j], k, t[k].data_ptr() if t[k] is not None else None)
        arr[j].phi = (ctypes.c_float * 3)(*jb["phi"])
        arr[j].psi = (ctypes.c_float * 3)(*jb["psi"])
        arr[j].theta = (ctypes.c_float * 3)(*jb["theta"])
    angles = np.zeros((len(jobs), 3), np.float32)
    shifts = np.zeros((len(jobs), 3), np.float32)
    peaks = np.zeros(len(jobs), np.float32)
    prm = _lib.AlignParams(int(path), int(batch_bytes))
    torch.cuda.synchronize(ctx.device)
    t1 = time.perf_counter()
    ctx.check(lib().tomgpu_av3_align_ex_dev(ctx.handle, arr, len(jobs), ctypes.byref(prm),
                                            angles.ctypes.data_as(_lib.c_float_p),
                                            shifts.ctypes.data_as(_lib.c_float_p),
                                            peaks.ctypes.data_as(_lib.c_float_p)))
    torch.cuda.synchronize(ctx.device)
    if timings is not None:
        timings["upload_s"] = t1 - t0
        timings["call_s"] = time.perf_counter() - t1
    return angles, shifts, peaks


def av3_align_host(jobs, ctx: Context | None = None, path: int = 0, batch_bytes: int = 0):
    """av3_align_batch through the host-volume entry point tomgpu_av3_align
    (the one a MEX gateway calls): the library uploads every distinct array
    once.  Each array is passed as float32 in x-fastest order; an array used by
    several jobs (the same numpy object) is converted and uploaded once."""
    ctx = ctx or default_context()
    arr = (_lib.AlignJob * len(jobs))()
    conv = {}

    def host(a):
        if a is None:
            return None
        hit = conv.get(id(a))
        if hit is None or hit[0] is not a:
            hit = (a, np.asfortranarray(np.asarray(a, np.float32)))
            conv[id(a)] = hit
        return hit[1]

    for j, jb in enumerate(jobs):
        n = np.shape(jb["ref"])
        mask = jb.get("mask")
        if mask is None:
            mask = jb.setdefault("_default_mask", tom_spheremask_default(n))
        arr[j].n = (ctypes.c_int * 3)(*n)
        for k, a in (("ref", jb["ref"]), ("part", jb["part"]), ("mask", mask), ("mask_ccf", jb.get("mask_ccf")),
                     ("wedge_ref", jb.get("wedge_ref")), ("wedge_part", jb.get("wedge_part"))):
            h = host(a)
            setattr(arr[j], k, h.ctypes.data if h is not None else None)
        arr[j].phi = (ctypes.c_float * 3)(*jb["phi"])
        arr[j].psi = (ctypes.c_float * 3)(*jb["psi"])
        arr[j].theta = (ctypes.c_float * 3)(*jb["theta"])
    angles = np.zeros((len(jobs), 3), np.float32)
    shifts = np.zeros((len(jobs), 3), np.float32)
    peaks = np.zeros(len(jobs), np.float32)
    prm = _lib.AlignParams(int(path), int(batch_bytes))
    ctx.check(lib().tomgpu_av3_align(ctx.handle, arr, len(jobs), ctypes.byref(prm),
                                     angles.ctypes.data_as(_lib.c_float_p), shifts.ctypes.data_as(_lib.c_float_p),
                                     peaks.ctypes.data_as(_lib.c_float_p)))
    return angles, shifts, peaks


def tom_av3_align(ref, part, phi, psi, theta, mask=None, filter=None, mask_ccf=None, wedge_ref=None,
                  wedge_part=None, ctx: Context | None = None):
    """[angles shifts ccf_peak] = tom_av3_align(ref,part,phi,psi,theta,mask,filter,mask_ccf,wedge_ref,wedge_part)
    (av3_new/tom_av3_align.m) on the GPU; filter must be absent or have Apply = 0."""
    if filter is not None and getattr(filter, "Apply", filter.get("Apply", 0) if isinstance(filter, dict) else 0):
        raise ValueError("tom_av3_align on the GPU supports filter.Apply = 0 only")
    if wedge_ref is not None and wedge_part is None:
        wedge_part = wedge_ref  # the 8-argument form
    a, s, p = av3_align_batch([dict(ref=ref, part=part, phi=phi, psi=psi, theta=theta, mask=mask,
                                    mask_ccf=mask_ccf, wedge_ref=wedge_ref, wedge_part=wedge_part)], ctx)
    return a[0], s[0], float(p[0])
