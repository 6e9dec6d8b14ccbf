"""Kernel-level parity on the GPU: rotation (bit-exact with rot3d), FFTs,
peaks, weighting and wedges, all through the C ABI."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TABLE = [0, 30, 45, 60, 90, 120, 135, 150, 180, 210, 225, 240, 270, 300, 315, 330]


def test_rotate_bit_exact(gpu, oracle):
    rng = np.random.default_rng(11)
    for trial in range(24):
        s = tuple(int(x) for x in rng.integers(4, 20, 3))
        v = rng.standard_normal(s).astype(np.float32)
        e = rng.choice(TABLE, 3) if trial % 2 else rng.random(3) * 360
        c = [float(np.ceil(x / 2)) for x in s] if trial % 3 else [float(x) for x in rng.integers(0, 5, 3)]
        out = np.zeros(s, np.float32, order="F")
        gpu.tom_rotatec(v, out, e, "linear", c)
        ref = oracle.rotate(v, e, c)
        assert np.array_equal(out.view(np.uint32), ref.view(np.uint32)), (s, e, c)
        if oracle.ref_available():
            assert np.array_equal(out, oracle.ref_rotate(v, e, c))
        m = oracle.euler_matrix(e).reshape(3, 3, order="F")
        out2 = np.zeros(s, np.float32, order="F")
        gpu.tom_rotatec(v, out2, m, "linear", c)
        assert np.array_equal(out2, oracle.rotate_matrix(v, oracle.euler_matrix(e), c))


def test_rotate_batch_with_mask(gpu, oracle):
    import ctypes
    import torch
    from tom_b200 import _lib
    from tom_b200.tom import _cdims, _tptr
    ctx = gpu.default_context()
    rng = np.random.default_rng(12)
    T = 24
    t = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 10).astype(np.float32)
    eul = np.column_stack([rng.choice(TABLE, 7), rng.random(7) * 360, rng.choice(TABLE, 7)]).astype(np.float32)
    td, md = gpu.to_device(t), gpu.to_device(mask)
    out = torch.empty((7, T, T, T), dtype=torch.float32, device="cuda")
    c = (ctypes.c_float * 3)(12, 12, 12)
    ctx.check(_lib.lib().tomgpu_rotate3d_batch_dev(ctx.handle, _tptr(td), _tptr(out), _cdims((T, T, T)),
                                                   eul.ctypes.data_as(_lib.c_float_p), 7, c, _tptr(md)))
    torch.cuda.synchronize()
    for r in range(7):
        ref = oracle.rotate(t, eul[r], (12, 12, 12)) * mask
        got = gpu.from_device(out[r])
        assert np.array_equal(got, ref.astype(np.float32))


@pytest.mark.parametrize("L", [8, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 232, 256, 464, 512, 928])
def test_fft_lengths(gpu, L):
    rng = np.random.default_rng(L)
    for shape in [(L, 8, 8), (8, L, 16), (16, 8, L)]:
        a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        f = gpu.tom_fourier(a)
        ref = np.fft.fftn(a)
        assert np.abs(f - ref).max() <= 1e-11 * np.abs(ref).max()
        b = gpu.tom_ifourier(f)
        assert np.abs(b - a).max() <= 1e-11 * np.abs(a).max()


@pytest.mark.parametrize("shape", [(64, 48, 40), (32, 32, 32), (128, 16, 24), (96, 80, 160)])
@pytest.mark.parametrize("prec", [32, 64])
def test_fft_r2c_c2r(gpu, shape, prec):
    import ctypes
    import torch
    from tom_b200 import _lib
    from tom_b200.tom import _cdims, _tptr
    ctx = gpu.default_context()
    rng = np.random.default_rng(7)
    a = rng.standard_normal(shape)
    dt = torch.float32 if prec == 32 else torch.float64
    x = torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).to("cuda", dt)
    nh = shape[0] // 2 + 1
    half = torch.empty((shape[2], shape[1], nh, 2), dtype=dt, device="cuda")
    ctx.check(_lib.lib().tomgpu_fft3d_r2c_dev(ctx.handle, _tptr(x), _tptr(half), _cdims(shape), prec))
    torch.cuda.synchronize()
    got = torch.view_as_complex(half).cpu().numpy().transpose(2, 1, 0)
    ref = np.fft.rfftn(a, axes=(2, 1, 0))
    tol = 2e-6 if prec == 32 else 1e-13
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
    back = torch.empty_like(x)
    ctx.check(_lib.lib().tomgpu_fft3d_c2r_dev(ctx.handle, _tptr(half), _tptr(back), _cdims(shape), prec))
    torch.cuda.synchronize()
    assert np.abs(back.cpu().numpy().transpose(2, 1, 0) - a).max() <= tol * 10 * np.abs(a).max()


def test_peak_matches_reference(gpu, oracle):
    rng = np.random.default_rng(13)
    for _ in range(10):
        v = rng.integers(-4, 5, (17, 9, 11)).astype(np.float32)
        pos, val = gpu.tom_peakc(v)
        rv, rp = oracle.find_max(v)
        assert val == rv and pos == tuple(p + 1 for p in rp)
    big = rng.standard_normal((256, 200, 130)).astype(np.float32)
    big[77, 3, 100] = 50.0
    big[5, 150, 129] = 50.0  # a later tie: the first in x-fastest order wins
    pos, val = gpu.tom_peakc(big)
    assert val == 50.0 and pos == (78, 4, 101)


def test_tom_peak_kat_and_radius(gpu, oracle):
    A = np.array([[1, 2, 3, 4, 17], [5, 6, 7, 8, 18], [10, 9, 40, 6, 20], [12, 16, 17, 20, 30],
                  [5, 23, 35, 12, 6]], float)
    A3 = A[:, :, None].repeat(1, axis=2)
    c, v = gpu.tom_peak(A3)
    assert c == (3, 3, 1) and v == 40
    c, v = gpu.tom_peak(A3, "spline")
    assert np.allclose(c[:2], [3.0890, 2.9770], atol=5e-5) and abs(v - 40.2232) < 5e-5
    # radius zeroing in 3-D against the oracle
    rng = np.random.default_rng(14)
    B = rng.standard_normal((15, 13, 11))
    c, v, M = gpu.tom_peak(B, 3)
    rc, rv, rM = oracle.tom_peak_radius(B.astype(np.float32).astype(np.float64), 3)
    assert c == rc and abs(v - rv) < 1e-6
    assert np.array_equal(M == 0, rM == 0)


def test_topk_matches_oracle(gpu, oracle):
    rng = np.random.default_rng(15)
    vol = rng.standard_normal((40, 36, 30)).astype(np.float32)
    vals, pos = gpu.topk_peaks(gpu.to_device(vol), 12, 4.0)
    ref = oracle.topk_peaks(vol, 12, 4.0)
    for k, (c, v) in enumerate(ref):
        assert tuple(pos[k]) == c and vals[k] == np.float32(v)


def test_topk_radius_beyond_the_volume_and_rejected_radii(gpu, oracle):
    """A radius beyond the volume's diagonal zeroes the whole volume after the
    first peak (the zeroing box is clamped to the volume on each axis), so the
    later rounds find 0 at (1, 1, 1), as tom_peak does on the zeroed matrix;
    a radius far beyond the int range behaves the same.  Negative, NaN and
    infinite radii are rejected before anything is launched."""
    rng = np.random.default_rng(16)
    vol = rng.standard_normal((20, 17, 12)).astype(np.float32)
    diag = float(np.sqrt(20 ** 2 + 17 ** 2 + 12 ** 2))
    for radius in (diag + 5.0, 1e6, 3e9):
        vals, pos = gpu.topk_peaks(gpu.to_device(vol), 4, radius)
        ref = oracle.topk_peaks(vol, 4, radius)
        for k, (c, v) in enumerate(ref):
            assert tuple(pos[k]) == c and vals[k] == np.float32(v), (radius, k)
        assert list(vals[1:]) == [0.0, 0.0, 0.0] and all(tuple(p) == (1, 1, 1) for p in pos[1:])
    for bad in (float("inf"), float("nan"), -1.0):
        with pytest.raises(gpu.TomGpuError) as e:
            gpu.topk_peaks(gpu.to_device(vol), 3, bad)
        assert e.value.status == gpu._lib.TOMGPU_ERR_ARG, bad


def test_weight3d_vs_reference(gpu, oracle):
    for dims, ang, th in [((16, 12, 10), [[0, 0, 0, 0], [-60, -20, 20, 60]], 16),
                          ((32, 32, 32), np.vstack([np.zeros(41), np.arange(-60, 61, 3)]), 64)]:
        ang = np.asarray(ang, float)
        got = gpu.tom_calc_weight_functioninc(dims, ang, th)
        ref = oracle.ref_weight3d(dims, ang, th) if oracle.ref_available() else oracle.weight3d(dims, ang, th)
        ulp = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
        assert ulp.max() <= 1


def test_wedges_vs_oracle(gpu, oracle):
    for shape in [(32, 32, 32), (40, 24, 36), (17, 9, 13)]:
        for ang in (30.0, 35.0, 25.0):
            assert np.array_equal(gpu.tom_wedge(np.zeros(shape), ang), oracle.tom_wedge(shape, ang))
        for mn, mx in ((-60, 60), (-45, 55)):
            assert np.array_equal(gpu.av3_wedge(np.zeros(shape), mn, mx), oracle.av3_wedge(shape, mn, mx))


def test_apply_weight_function(gpu, oracle):
    rng = np.random.default_rng(71)
    v = rng.standard_normal((24, 20, 32)).astype(np.float32)
    w = oracle.tom_wedge(v.shape, 30.0)
    got = gpu.tom_apply_weight_function(v, w)
    ref = oracle.apply_weight_function(v, w)
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


def test_empty_volume_rule(gpu, oracle):
    """tom_os3_findTemplate.m: a volume with mean 0 and std 0 is not searched."""
    T = 16
    tmpl = np.random.default_rng(1).standard_normal((T, T, T)).astype(np.float32)
    ccc, ang = gpu.tom_os3_findTemplate(np.zeros((32, 32, 32), np.float32), tmpl, [(0, 0, 0)])
    assert np.all(ccc == 0) and np.all(ang == -1000)
