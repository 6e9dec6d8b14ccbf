"""Peak analysis (tom_os3_analyzePeak 'PSR' / 'Autocorrelation') and the
findTemplate loop that carries it, on the GPU against the FP64 oracle.

Tolerance: |x_gpu - x_oracle| <= 1e-4 * max|x_oracle| for every map; the
search's indices must agree on every voxel whose update decisions were all
clear-cut in the oracle (margin above 5e-4).  The templates here are dense
(wedge-filtered or random), so every window of the template autocorrelation
sees nonzero voxels: where a window sees only zeros the reference divides 0 by
0 and its result there is rounding noise."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REL = 1e-4


def _close(got, ref, rel=REL):
    scale = np.abs(ref).max()
    err = np.abs(np.asarray(got, np.float64) - ref).max()
    assert err <= rel * scale, f"max err {err:.3e} > {rel * scale:.3e}"


def _cc_map(oracle, seed, N=(64, 48, 40), T=16):
    rng = np.random.default_rng(seed)
    vol = rng.standard_normal(N)
    t = rng.standard_normal((T, T, T))
    mask = oracle.sphere_mask((T, T, T), 7)
    st = oracle.FLCF(vol, mask)
    _, tm, ts = oracle.norm_under_mask(t, mask)
    return st.corr(t, tm, ts).astype(np.float32), t.astype(np.float32), mask.astype(np.float32)


def test_psr_map(gpu, oracle):
    pk, t, _ = _cc_map(oracle, 41)
    ref = oracle.analyze_psr(pk.astype(np.float64), t.shape)
    got = gpu.tom_os3_analyzePeak(None, pk, t, {"analysis": {"type": "PSR"}})
    _close(got, ref)


def test_template_autocorr(gpu, oracle):
    rng = np.random.default_rng(42)
    t = rng.standard_normal((16, 16, 16)).astype(np.float32)
    ref = oracle.os3_corr_same(t.astype(np.float64), t.astype(np.float64))
    got = gpu.tom_os3_template_autocorr(t)
    assert abs(got[8, 8, 8] - 1) < 1e-6
    _close(got, ref, 1e-6)


def test_autocorr_map(gpu, oracle):
    pk, t, mask = _cc_map(oracle, 43)
    ref = oracle.analyze_autocorr(pk.astype(np.float64), t.astype(np.float64), mask.astype(np.float64))
    got = gpu.tom_os3_analyzePeak(None, pk, t, {"analysis": {"type": "Autocorrelation"},
                                                "correlation": {"mask": mask}})
    _close(got, ref)


def test_os3_corr_own_statistics(gpu, oracle):
    """tom_os3_corr(img, t, options) without cached template statistics."""
    rng = np.random.default_rng(44)
    vol = rng.standard_normal((64, 48, 40)).astype(np.float32)
    t = (rng.standard_normal((16, 16, 16)) * 3 + 2).astype(np.float32)
    mask = oracle.sphere_mask((16, 16, 16), 7).astype(np.float32)
    st = oracle.FLCF(vol.astype(np.float64), mask.astype(np.float64))
    _, tm, ts = oracle.norm_under_mask(t.astype(np.float64), mask)
    ref = st.corr(t.astype(np.float64), tm, ts)
    got, _ = gpu.tom_os3_corr(vol, t, {"mask": mask})
    _close(got, ref)


@pytest.mark.parametrize("flags", [dict(ccc=1), dict(ccc=1, psr=1), dict(ccc=1, psr=1, autocorr=1),
                                   dict(psr=1)])
def test_find_template_analysis(gpu, oracle, flags):
    rng = np.random.default_rng(45)
    N, T = (48, 40, 32), 16
    vol = rng.standard_normal(N).astype(np.float32)
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    psf = oracle.tom_wedge((T, T, T), 30).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (60, 60, 45), (300, 60, 90))[:6]
    sel = {k: bool(flags.get(k, 0)) for k in ("ccc", "psr", "autocorr")}
    rc, ri, rp, ra, margin = oracle.find_template_analysis(vol, tmpl, mask, angles, psf=psf, margins=True, **sel)
    ccc, ang, psr, soc = gpu.tom_os3_findTemplate(vol, tmpl, angles, mask=mask, psf=psf, analysis=flags)
    idx = np.where(ang > 0, ang - 1, -1).astype(np.int64)
    clear = margin > 5e-4
    assert clear.mean() > 0.8
    assert np.array_equal(idx[clear], ri[clear]), f"{(idx[clear] != ri[clear]).sum()} index mismatches"
    for got, ref in ((ccc, rc), (psr, rp), (soc, ra)):
        scale = np.abs(ref[clear]).max()
        assert np.abs(got[clear] - ref[clear]).max() <= REL * scale


def test_find_template_analysis_ccc_equals_fast(gpu, oracle):
    """The analysis loop with only the ccc criterion finds what the fast search finds."""
    rng = np.random.default_rng(46)
    N, T = (48, 40, 32), 16
    vol = rng.standard_normal(N).astype(np.float32)
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (60, 60, 45), (300, 60, 90))[:5]
    c1, a1 = gpu.tom_os3_findTemplate(vol, tmpl, angles, mask=mask)
    c2, a2, _, _ = gpu.tom_os3_findTemplate(vol, tmpl, angles, mask=mask, analysis={"ccc": 1})
    assert np.abs(c1 - c2).max() <= 1e-5 * np.abs(c1).max()
    assert (a1 != a2).mean() < 1e-3


def test_find_template_analysis_empty_volume(gpu):
    z = np.zeros((32, 32, 32), np.float32)
    t = np.ones((16, 16, 16), np.float32)
    ccc, ang, psr, soc = gpu.tom_os3_findTemplate(z, t, [[0, 0, 0]], analysis={"ccc": 1, "psr": 1})
    assert not ccc.any() and not psr.any() and not soc.any() and np.all(ang == -1000)
