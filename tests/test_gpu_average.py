"""Averaging step after alignment (av3_tomomatch) on the GPU against the oracle.

The rotation is bit-exact given the same float input; the Fourier shift runs in
FP64 on both sides, so the rotated particles agree to float rounding of the
shifted volume: tolerance 1e-6 of the largest value for the sums and the
weighted average, exact equality for the wedge counts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _items(oracle, K, n, seed):
    rng = np.random.default_rng(seed)
    w1 = oracle.av3_wedge((n, n, n), -60, 60).astype(np.float32)
    w2 = oracle.av3_wedge((n, n, n), -45, 55).astype(np.float32)
    parts = [rng.standard_normal((n, n, n)).astype(np.float32) for _ in range(K)]
    wedges = [w1 if k % 2 == 0 else w2 for k in range(K)]
    shifts = rng.uniform(-3, 3, (K, 3)).astype(np.float32)
    angles = rng.uniform(-180, 180, (K, 3)).astype(np.float32)
    return parts, wedges, shifts, angles


def test_average_sums_and_final(gpu, oracle):
    n, K = 32, 7
    parts, wedges, shifts, angles = _items(oracle, K, n, 51)
    ref_avg, ref_wei = oracle.av3_average_add(list(zip(parts, wedges, shifts, angles)), (n, n, n))
    avg, wei = gpu.av3_average_add(parts[:4], wedges[:4], shifts[:4], angles[:4])
    avg, wei = gpu.av3_average_add(parts[4:], wedges[4:], shifts[4:], angles[4:], avg, wei)  # accumulates
    g_avg = np.asfortranarray(gpu.from_device(avg))
    g_wei = np.asfortranarray(gpu.from_device(wei))
    assert np.array_equal(g_wei, ref_wei)
    assert np.abs(g_avg - ref_avg).max() <= 1e-6 * np.abs(ref_avg).max()
    out = gpu.av3_average_final(avg, wei)
    ref = oracle.av3_average_final(ref_avg, ref_wei)
    assert np.abs(out - ref).max() <= 1e-6 * np.abs(ref).max()


def test_tomomatch_average_selection(gpu, oracle):
    """Class 1/2 assignment by threshold * mean CCC and the tom_limit of the particles."""
    n, K = 24, 6
    parts, _, shifts, angles = _items(oracle, K, n, 52)
    parts = [p * 3 for p in parts]            # values beyond -3 .. 4 are limited
    motl = np.zeros((20, K))
    motl[0] = [0.5, 0.1, 0.6, 0.55, 0.05, 0.4]
    motl[4] = [1, 1, 2, 2, 1, 2]
    motl[10:13] = shifts.T
    motl[16:19] = angles.T
    motl[19] = [1, 1, 2, 0, 1, 3]             # the last is another class: untouched
    wl = np.array([[1, 2], [-60, -45], [60, 55]], np.float64)
    avg, wei, m2 = gpu.av3_tomomatch_average(parts, motl, wl, threshold=0.8)
    sel = np.array([True, True, True, False, True, False])  # classes 1, 2 (iclass 0 selects class-0 too)
    sel[3] = True
    meanv = motl[0, sel].mean()
    keep = [p for p in range(K) if sel[p] and motl[0, p] > 0.8 * meanv]
    assert list(np.nonzero(m2[19] == 1)[0]) == keep
    assert set(np.nonzero(m2[19] == 2)[0]) == {p for p in range(K) if sel[p]} - set(keep)
    assert m2[19, 5] == 3
    w = {1: oracle.av3_wedge((n, n, n), -60, 60), 2: oracle.av3_wedge((n, n, n), -45, 55)}
    items = [(oracle.tom_limit(parts[p], -3, 4, "z"), w[int(motl[4, p])], shifts[p], angles[p]) for p in keep]
    ra, rw = oracle.av3_average_add(items, (n, n, n))
    assert np.array_equal(wei, rw)
    ref = oracle.av3_average_final(ra, rw)
    assert np.abs(avg - ref).max() <= 1e-6 * np.abs(ref).max()
