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


def _job(oracle, n, k, wedge, rng_seed, phi=(0, 3, 6), psi=(0, 3, 6), theta=(6, 3, 12), mccf="sphere"):
    e = (3.0 * (k % 3), 3.0, 9.0)
    w = oracle.av3_wedge((n, n, n), -50, 55).astype(np.float32) if wedge else None
    ref, part = _particle(oracle, n, e, (1, 0, -1), seed=rng_seed, wedge=w)
    sph = oracle.sphere_mask((n, n, n), 4.0, strict=True).astype(np.float32)
    m = {"sphere": sph, "negative": -sph, "none": None}[mccf]
    return dict(ref=ref, part=part, phi=phi, psi=psi, theta=theta,
                mask=oracle.sphere_mask((n, n, n), n / 2 - 2).astype(np.float32),
                mask_ccf=m, wedge_ref=w, wedge_part=w)


def test_batched_engine_equals_per_job(gpu, oracle):
    """The batched engine (one entry stream per box edge and wedge form, a
    batch smaller than a particle's scan so that batches span particles and
    entry groups) gives the per-job results: same angles, shifts and peaks to
    FP32 rounding.  A 28^3 job (no compiled edge) runs per job in both."""
    jobs = []
    spec = [(32, True), (32, True), (24, True), (32, False), (32, True), (48, True), (28, True), (32, False),
            (24, False)]
    for k, (n, wedge) in enumerate(spec):
        jobs.append(_job(oracle, n, k, wedge, 300 + k))
    # a negative mask_ccf (every in-mask product below zero: the maximum is the
    # first zero voxel, outside the mask) at 40^3, and 64^3 without mask_ccf
    # (no pruning of the final inverse)
    jobs.append(_job(oracle, 40, 1, True, 320, mccf="negative"))
    jobs.append(_job(oracle, 40, 2, True, 321))
    jobs.append(_job(oracle, 64, 0, True, 322, mccf="none", phi=(0, 3, 3), psi=(0, 3, 3)))
    # a graded reference wedge (not exact in half precision: full-precision
    # corner bricks for the 40^3 edge; the binary wedges elsewhere use halves)
    soft = _job(oracle, 40, 0, True, 323)
    soft["wedge_ref"] = (0.7 * soft["wedge_ref"] + 0.1234567).astype(np.float32)
    jobs.append(soft)
    # a particle wedge other than the reference wedge (the 8-argument form
    # with both), and a graded mask (the reference times the mask values,
    # the statistics over its non-zero voxels)
    two = _job(oracle, 32, 2, True, 327)
    two["wedge_part"] = oracle.av3_wedge((32, 32, 32), -40, 65).astype(np.float32)
    jobs.append(two)
    graded = _job(oracle, 48, 1, True, 328)
    r = np.sqrt(((np.indices((48, 48, 48)) - 24.0) ** 2).sum(0))
    graded["mask"] = np.asfortranarray(np.clip((22.0 - r) / 4.0, 0.0, 1.0).astype(np.float32))
    jobs.append(graded)
    # the larger edges (radices 8 x 7, 4 x 5 x 5, 16 x 8), the last without
    # mask_ccf (the full last inverse on two lines per complex line)
    few = dict(phi=(0, 3, 3), psi=(0, 3, 3), theta=(6, 3, 9))
    jobs.append(_job(oracle, 56, 1, True, 324, **few))
    jobs.append(_job(oracle, 100, 2, True, 325, **few))
    jobs.append(_job(oracle, 128, 0, False, 326, mccf="none", **few))
    half32 = 17 * 32 * 32 * 8
    a0, s0, p0 = gpu.av3_align_batch(jobs, path=0, batch_bytes=2 * half32 * 10)
    a1, s1, p1 = gpu.av3_align_batch(jobs, path=1)
    assert np.array_equal(a0, a1), (a0, a1)
    assert np.abs(s0 - s1).max() <= 2e-3, (s0, s1)
    assert np.allclose(p0, p1, rtol=2e-4, atol=0), (p0, p1)
    # the default batch (every scan in one batch) and the batched engine
    # without the pruned last inverse agree too
    for path in (0, 2):
        a2, s2, p2 = gpu.av3_align_batch(jobs, path=path)
        assert np.array_equal(a2, a1), path
        assert np.abs(s2 - s1).max() <= 2e-3, path
        assert np.allclose(p2, p1, rtol=2e-4, atol=0), path


def test_batched_engine_matches_oracle_without_and_with_wedges(gpu, oracle):
    """Batched engine against the FP64 oracle of tom_av3_align at 40^3 with
    wedges (the oracle's own cross-wedged scan) and several particles."""
    n = 40
    w = oracle.av3_wedge((n, n, n), -55, 60).astype(np.float32)
    jobs, want = [], []
    for k in range(2):
        euler = (9.0 - 3 * k, 6.0, 12.0)
        ref, part = _particle(oracle, n, euler, (1, -1, 0), seed=500 + k, wedge=w)
        mask = oracle.sphere_mask((n, n, n), n / 2 - 2).astype(np.float32)
        mccf = oracle.sphere_mask((n, n, n), 4.0, strict=True).astype(np.float32)
        phi, psi, theta = (3, 3, 9), (3, 3, 9), (9, 3, 15)
        want.append(oracle.av3_align(ref, part, phi, psi, theta, mask, mccf, w, w)[:3])
        jobs.append(dict(ref=ref, part=part, phi=phi, psi=psi, theta=theta, mask=mask, mask_ccf=mccf,
                         wedge_ref=w, wedge_part=w))
    ga, gs, gp = gpu.av3_align_batch(jobs, batch_bytes=2 * 21 * 40 * 40 * 8 * 7)
    for k in range(2):
        ra, rs, rp = want[k]
        assert np.allclose(ga[k], ra), (k, ga[k], ra)
        assert np.abs(gs[k] - rs).max() <= 0.0015, (gs[k], rs)
        assert abs(gp[k] - rp) <= 1e-4 * abs(rp), (gp[k], rp)


def test_host_entry_point_equals_device_entry_point(gpu, oracle):
    """tomgpu_av3_align (host volumes, each distinct array uploaded once: here
    one reference and one mask shared by three particles, one mask_ccf
    omitted) gives what tomgpu_av3_align_ex_dev gives on device copies."""
    n = 32
    base = _job(oracle, n, 0, True, 400)
    jobs = []
    for k in range(3):
        jb = _job(oracle, n, k, True, 401 + k)
        jb["ref"], jb["mask"] = base["ref"], base["mask"]
        jobs.append(jb)
    jobs[2]["mask_ccf"] = None
    jobs.append(_job(oracle, 24, 1, False, 405))
    a0, s0, p0 = gpu.av3_align_batch(jobs)
    a1, s1, p1 = gpu.av3_align_host(jobs)
    assert np.array_equal(a0, a1)
    assert np.array_equal(s0, s1)
    assert np.array_equal(p0, p1)


def test_batched_engine_remaining_edges(gpu, oracle):
    """The compiled edges not covered above (radices 8 x 3 x 3, 16 x 5,
    16 x 6, 16 x 7, 8 x 3 x 5) give the job-by-job results."""
    few = dict(phi=(0, 3, 3), psi=(0, 3, 3), theta=(6, 3, 9))
    jobs = [_job(oracle, n, k, True, 600 + k, **few) for k, n in enumerate((72, 80, 96, 112, 120))]
    jobs.append(_job(oracle, 96, 1, False, 610, mccf="none", **few))
    a0, s0, p0 = gpu.av3_align_batch(jobs, path=0)
    a1, s1, p1 = gpu.av3_align_batch(jobs, path=1)
    assert np.array_equal(a0, a1), (a0, a1)
    assert np.abs(s0 - s1).max() <= 2e-3, (s0, s1)
    assert np.allclose(p0, p1, rtol=2e-4, atol=0), (p0, p1)
