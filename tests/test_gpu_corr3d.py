"""The C++ picker's batched aligner (tom_mex_corr3d 'peak') on the GPU against
the oracle's restatement of tom::corr3d_batch.

Tolerance: |ncc_gpu - ncc_oracle| <= 1e-4 (FP32 spectra against FP64); the
best angle and the peak position must agree wherever the oracle's best value
beats every other angle's by more than 1e-3."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _data(seed, n, nt, npart):
    rng = np.random.default_rng(seed)
    temps = [rng.standard_normal(n).astype(np.float32) for _ in range(nt)]
    parts = [rng.standard_normal(n).astype(np.float32) for _ in range(npart)]
    return temps, parts, rng


def _compare(gpu_out, ref):
    nt, npart = ref["val"].shape
    for i in range(nt):
        for j in range(npart):
            g = gpu_out[i, j]
            assert abs(g["ncc_val"] - ref["val"][i, j]) <= 1e-4, (i, j, g["ncc_val"], ref["val"][i, j])
            if ref["val"][i, j] - ref["second"][i, j] > 1e-3:
                assert g["angle_idx"] == ref["angle_idx"][i, j] + 1
                assert tuple(g["peak"].astype(int)) == tuple(ref["peak"][i, j])


@pytest.mark.parametrize("case", ["plain", "mask_simple_wedges", "volume_wedges"])
def test_corr3d_vs_oracle(gpu, oracle, case):
    n = (24, 24, 20)
    temps, parts, rng = _data(61, n, 2, 3)
    angles = rng.uniform(-180, 180, (5, 3))
    kw = {}
    if case == "mask_simple_wedges":
        kw = dict(mask=gpu.cpp_spheremask(n, 9), wedge_ref=30.0, wedge_part=[45.0, None, 50.0],
                  mask_cc=gpu.cpp_spheremask(n, 4))
        ref_kw = dict(mask=kw["mask"], wedge_t=[("simple", 30.0)] * 2,
                      wedge_p=[("simple", 45.0), None, ("simple", 50.0)], mask_cc=kw["mask_cc"])
    elif case == "volume_wedges":
        w1 = oracle.av3_wedge(n, -60, 60).astype(np.float32)
        w2 = oracle.av3_wedge(n, -45, 55).astype(np.float32)
        kw = dict(wedge_ref=w1, wedge_part=[w2, w1, np.ones(n, np.float32)])
        ref_kw = dict(wedge_t=[("volume", w1)] * 2, wedge_p=[("volume", w2), ("volume", w1), ("volume", np.ones(n))])
    else:
        ref_kw = {}
    out = gpu.tom_corr3d(temps, parts, angles, **kw)
    ref = oracle.corr3d_peaks(temps, parts, angles, **ref_kw)
    _compare(out, ref)


def test_corr3d_recovers_rotation(gpu, oracle):
    n = (32, 32, 32)
    rng = np.random.default_rng(62)
    t = np.zeros(n, np.float32)
    t[8:24, 10:22, 12:20] = rng.standard_normal((16, 12, 8))
    angles = [(0, 0, 0), (30, 20, 40), (90, 0, 45), (10, 80, 20)]
    m, v = oracle.cpp_stat(t)
    part = oracle.cpp_rotate(((t - m) / np.sqrt(v)).astype(np.float32), *np.deg2rad(angles[2]))
    out = gpu.tom_corr3d([t], [part], angles, mask=14.0)
    assert out[0, 0]["angle_idx"] == 3
    assert tuple(out[0, 0]["peak"].astype(int)) == (0, 0, 0)
    assert out[0, 0]["ncc_val"] > 0.95


def test_corr3d_host_entry_point_equals_device_one(gpu, oracle):
    """tomgpu_corr3d_peaks (the host-volume form the tom_mex_corr3d gateway
    calls) gives the device form's results bit for bit, with a mask, wedge
    volumes for the templates, simple wedges for the particles and a peak mask."""
    import ctypes
    from tom_b200 import _lib
    from tom_b200.tom import _cdims
    n = (20, 18, 16)
    temps, parts, rng = _data(63, n, 2, 3)
    angles = rng.uniform(-180, 180, (4, 3))
    mask = gpu.cpp_spheremask(n, 7)
    mcc = gpu.cpp_spheremask(n, 3)
    w1 = oracle.av3_wedge(n, -60, 60).astype(np.float32)
    ref = gpu.tom_corr3d(temps, parts, angles, mask=mask, wedge_ref=w1, wedge_part=[40.0, None, 55.0], mask_cc=mcc)
    host = [np.asfortranarray(np.asarray(v, np.float32)) for v in temps + parts + [mask, mcc, w1]]
    ptr = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    tp = (ctypes.c_void_p * 2)(*[ptr(h).value for h in host[:2]])
    pp = (ctypes.c_void_p * 3)(*[ptr(h).value for h in host[2:5]])
    wt = (_lib.WedgeSpec * 2)()
    for i in range(2):
        wt[i].kind, wt[i].volume = 2, ptr(host[7])
    wp = (_lib.WedgeSpec * 3)()
    wp[0].kind, wp[0].angle_deg = 1, 40.0
    wp[1].kind = 0
    wp[2].kind, wp[2].angle_deg = 1, 55.0
    ang = np.ascontiguousarray(angles, np.float64)
    peak = np.zeros((3, 2, 3), np.float64)
    val = np.zeros((3, 2), np.float64)
    idx = np.zeros((3, 2), np.int32)
    ctx = gpu.default_context()
    ctx.check(_lib.lib().tomgpu_corr3d_peaks(ctx.handle, _cdims(n), tp, 2, pp, 3, ang.ctypes.data_as(_lib.c_double_p),
                                             len(ang), ptr(host[5]), wt, wp, ptr(host[6]),
                                             peak.ctypes.data_as(_lib.c_double_p), val.ctypes.data_as(_lib.c_double_p),
                                             idx.ctypes.data_as(_lib.c_int_p)))
    for i in range(2):
        for j in range(3):
            r = ref[i, j]
            assert idx[j, i] == r["angle_idx"] and val[j, i] == r["ncc_val"]
            assert np.array_equal(peak[j, i], r["peak"])


def test_corr3d_odd_box(gpu, oracle):
    """An odd box (the FFT lengths 25, 21 and 19, 19 through Bluestein)."""
    n = (25, 21, 19)
    temps, parts, rng = _data(64, n, 1, 2)
    angles = rng.uniform(-180, 180, (4, 3))
    out = gpu.tom_corr3d(temps, parts, angles, mask=gpu.cpp_spheremask(n, 8), wedge_ref=30.0, wedge_part=45.0)
    ref = oracle.corr3d_peaks(temps, parts, angles, mask=gpu.cpp_spheremask(n, 8), wedge_t=[("simple", 30.0)],
                              wedge_p=[("simple", 45.0)] * 2)
    _compare(out, ref)
