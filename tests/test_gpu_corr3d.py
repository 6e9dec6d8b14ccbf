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
