"""Subtomogram alignment (tom_av3_align semantics) on the GPU against the FP64
oracle restatement: same best angles, shifts within the spline step, peak
values within 1e-4 relative; the max-CC volume of the scan within 1e-4."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _particle(oracle, n, euler, shift, seed, wedge=None):
    rng = np.random.default_rng(seed)
    from tom_b200 import synth
    ph = synth.BlobPhantom(rng, 6, n / 4)
    ref = ph.template(n)
    part = np.zeros((n, n, n), np.float32, order="F")
    c = [np.ceil(n / 2) + s for s in shift]
    ph.render((n, n, n), c, euler, out=part)
    part = part + 0.3 * rng.standard_normal((n, n, n)).astype(np.float32)
    if wedge is not None:
        part = np.real(np.fft.ifftn(np.fft.fftn(part) * np.fft.ifftshift(wedge))).astype(np.float32)
    return ref, part


@pytest.mark.parametrize("n,wedges", [(24, True), (32, True), (32, False)])
def test_av3_align_matches_oracle(gpu, oracle, n, wedges):
    euler = (9.0, 6.0, 12.0)
    w = oracle.av3_wedge((n, n, n), -55, 60).astype(np.float32) if wedges else None
    ref, part = _particle(oracle, n, euler, (1, -1, 0), seed=n, wedge=w)
    mask = oracle.sphere_mask((n, n, n), n / 2 - 2).astype(np.float32)
    mccf = oracle.sphere_mask((n, n, n), 4.0, strict=True).astype(np.float32)
    phi, psi, theta = (3, 3, 12), (3, 3, 9), (6, 3, 15)
    ra, rs, rp, extra = oracle.av3_align(ref, part, phi, psi, theta, mask, mccf, w if wedges else None,
                                         w if wedges else None) if wedges else (None, None, None, None)
    if not wedges:
        # the oracle's no-wedge form: tom_corr 'norm' without psfs in the scan
        ra, rs, rp, extra = _oracle_no_wedge(oracle, ref, part, phi, psi, theta, mask, mccf)
    ga, gs, gp = gpu.tom_av3_align(ref, part, phi, psi, theta, mask=mask, mask_ccf=mccf,
                                   wedge_ref=w if wedges else None, wedge_part=w if wedges else None)
    assert np.allclose(ga, ra), (ga, ra)
    assert np.abs(gs - rs).max() <= 0.0015, (gs, rs)
    assert abs(gp - rp) <= 1e-4 * abs(rp), (gp, rp)


def _oracle_no_wedge(O, ref, part, phi, psi, theta, mask, mccf):
    ref = np.asarray(ref, np.float64)
    part = np.asarray(part, np.float64)
    n = ref.shape
    cmax = np.full(n, -2.0)
    amax = np.full(n, -2.0)
    st, inc, en = (phi[0], psi[0], theta[0]), (phi[1], psi[1], theta[1]), (phi[2], psi[2], theta[2])
    for a in O.av3_axis(phi):
        for b in O.av3_axis(psi):
            for c in O.av3_axis(theta):
                R = O.rotmatrix_double((a, b, c))
                rr = O.rotate_matrix(ref, R.astype(np.float32).flatten(order="F")).astype(np.float64)
                ccf = O.tom_corr_norm(rr, part, mask)
                nm = np.where(ccf > cmax, ccf, cmax)
                amax = np.where(ccf >= nm, O.av3_angle2index((a, b, c), st, inc, en), amax)
                cmax = nm
    pos, _ = O.tom_peak(cmax * mccf)
    ang = O.av3_index2angle(amax[tuple(p - 1 for p in pos)], st, inc, en)
    ccf_s = O.tom_corr_norm(O.rotate(ref, ang).astype(np.float64), part, mask)
    pos, peak = O.tom_peak_spline(ccf_s * mccf)
    return ang, np.array(pos) - (np.floor(np.array(n) / 2) + 1), peak, None


def test_av3_align_batch_mixed_sizes(gpu, oracle):
    jobs, expect = [], []
    for k, n in enumerate((32, 48, 32)):
        e = (6.0 + 3 * k, 3.0, 9.0)
        ref, part = _particle(oracle, n, e, (0, 1, -1), seed=100 + k)
        jobs.append(dict(ref=ref, part=part, phi=(0, 3, 15), psi=(0, 3, 6), theta=(6, 3, 12),
                         mask=oracle.sphere_mask((n, n, n), n / 2 - 2).astype(np.float32),
                         mask_ccf=oracle.sphere_mask((n, n, n), 4.0, strict=True).astype(np.float32)))
        expect.append(e)
    angles, shifts, peaks = gpu.av3_align_batch(jobs)
    for k in range(3):
        assert np.allclose(angles[k], expect[k]), (k, angles[k], expect[k])
        assert np.abs(shifts[k] - np.array([0, 1, -1])).max() < 0.6
        assert peaks[k] > 0.5


@pytest.mark.parametrize("form", ["plain", "mask", "psf"])
def test_tom_corr_forms(gpu, oracle, form):
    rng = np.random.default_rng(61)
    n = (32, 24, 40)
    a = rng.standard_normal(n)
    b = np.roll(a, (2, -1, 3), axis=(0, 1, 2)) + 0.2 * rng.standard_normal(n)
    if form == "plain":
        ref = np.real(np.fft.fftshift(np.fft.ifftn(np.fft.fftn(b) * np.conj(np.fft.fftn(a))))) / a.size
        got = gpu.tom_corr(a, b)
    else:
        mask = oracle.sphere_mask(n, 10).astype(np.float32)
        if form == "mask":
            ref = oracle.tom_corr_norm(a.astype(np.float32), b.astype(np.float32), mask)
            got = gpu.tom_corr(a, b, "norm", mask)
        else:
            w = oracle.av3_wedge(n, -50, 50)
            p1 = np.real(np.fft.ifftn(np.fft.ifftshift(w)))
            p2 = np.real(np.fft.ifftn(np.fft.ifftshift(oracle.av3_wedge(n, -60, 45))))
            ref = oracle.tom_corr_norm(a.astype(np.float32), b.astype(np.float32), mask, p1.astype(np.float32),
                                       p2.astype(np.float32))
            got = gpu.tom_corr(a, b, "norm", mask, p1, p2)
    assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max()
