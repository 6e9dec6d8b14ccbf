"""The oracle pinned against the reference: its C restatements equal the
compiled reference routines bit for bit, and its MATLAB-level restatements
reproduce every known-answer example of the reference's docstrings."""
import os

import numpy as np
import pytest

TABLE = [0, 30, 45, 60, 90, 120, 135, 150, 180, 210, 225, 240, 270, 300, 315, 330]


def test_rot3d_bit_exact_vs_reference(ref_libs):
    O = ref_libs
    rng = np.random.default_rng(1)
    for trial in range(40):
        s = tuple(int(x) for x in rng.integers(4, 18, 3))
        v = rng.standard_normal(s).astype(np.float32)
        if trial % 2:
            e = rng.choice(TABLE + [10, 17.5, -20, 33.3], 3)
        else:
            e = rng.random(3) * 360
        c = None if trial % 3 else tuple(float(x) for x in rng.integers(0, 6, 3))
        a = O.rotate(v, e, c)
        b = O.ref_rotate(v, e, c)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (s, e, c)
        m = O.euler_matrix(e)
        assert np.array_equal(O.rotate_matrix(v, m, c), O.ref_rotate(v, m, c))


def test_find_max_vs_reference(ref_libs):
    O = ref_libs
    rng = np.random.default_rng(2)
    for _ in range(20):
        v = rng.integers(-3, 4, (6, 5, 4)).astype(np.float32)  # many ties
        assert O.find_max(v) == O.ref_find_max(v)
    v = np.full((3, 3, 3), -1e6, np.float32)
    v[1, 2, 0] = -99998.0
    assert O.ref_find_max(v)[1] == (1, 2, 0)


def test_weight3d_vs_reference(ref_libs):
    O = ref_libs
    for dims, ang, th in [((16, 12, 10), [[0, 0, 0, 0], [-60, -20, 20, 60]], 16),
                          ((9, 8, 7), [[10, 30], [-45, 50]], 5),
                          ((20, 20, 20), np.vstack([np.zeros(41), np.arange(-60, 61, 3)]), 64)]:
        a = O.weight3d(dims, np.asarray(ang, float), th)
        b = O.ref_weight3d(dims, np.asarray(ang, float), th)
        assert np.array_equal(a, b)


def test_tom_peak_kats(oracle):
    """Analysis/tom_peak.m:27-50."""
    A = np.array([[1, 2, 3, 4, 17], [5, 6, 7, 8, 18], [10, 9, 40, 6, 20], [12, 16, 17, 20, 30],
                  [5, 23, 35, 12, 6]], float)
    assert oracle.tom_peak(A) == ((3, 3), 40.0)
    c, v = oracle.tom_peak_spline(A)
    assert np.allclose(c, [3.0890, 2.9770], atol=5e-5) and abs(v - 40.2232) < 5e-5
    _, _, M = oracle.tom_peak_radius(A, 2)
    expect = np.array([[1, 2, 0, 4, 17], [5, 0, 0, 0, 18], [0, 0, 0, 0, 0], [12, 0, 0, 0, 30],
                       [5, 23, 0, 12, 6]], float)
    assert np.array_equal(M, expect)


def test_tom_fourier_kat():
    """Filtrans/tom_fourier.m:18-22.  Two printed entries contradict the table's own
    Hermitian symmetry for a real input (c(1,2) must be conj(c(1,4)) and c(2,2)
    conj(c(4,4))); the other 14 entries are pinned exactly."""
    a = np.array([[11, 3, -6, -14], [1, -13, 9, 6], [0, 8, 13, -3], [-8, 17, -15, 7]], float)
    c = np.fft.fft2(a)
    expect = np.array([[16, 3 + 19j, -6, 3 + 19j], [-24 - 2j, 50 + 9j, 8 - 64j, 1 + 21j],
                       [8, 5 - 37j, 54, 5 + 37j], [-24 + 2j, 1 - 21j, 8 + 64j, 59 - 9j]])
    ok = np.ones((4, 4), bool)
    ok[0, 1] = ok[1, 1] = False
    assert np.allclose(c[ok], expect[ok])
    assert np.isclose(c[0, 1], np.conj(expect[0, 3])) and np.isclose(c[1, 1], np.conj(expect[3, 3]))


def test_tom_norm_kat(oracle):
    """Sptrans/tom_norm.m:29-43: c = tom_norm(a, 10) maps [min, max] = [0, 19]
    to [0, 10].  23 of the 25 printed values are the map's values truncated
    to 3 decimals; two are print slips: the input 8 prints as 4.210 five
    times and once (row 5, column 2) as 4.219, and the input 2 prints as
    1.056 where 10 * 2 / 19 = 1.0526 is the value of the same linear map that
    fits the other 23."""
    a = np.array([[10, 1, 19, 8, 5], [12, 9, 17, 10, 10], [3, 3, 2, 0, 8], [15, 8, 0, 7, 8],
                  [0, 8, 6, 15, 8]], float)
    printed = np.array([[5.263, 0.526, 10.00, 4.210, 2.631], [6.315, 4.736, 8.947, 5.263, 5.263],
                        [1.578, 1.578, 1.056, 0, 4.210], [7.894, 4.210, 0, 3.684, 4.210],
                        [0, 4.219, 3.157, 7.894, 4.210]])
    c = oracle.tom_norm(a, 10)
    slips = np.zeros(a.shape, bool)
    slips[2, 2] = slips[4, 1] = True
    # the printed values are truncated to 3 decimals (7.8947 -> 7.894, 4.7368 -> 4.736)
    d = c[~slips] - printed[~slips]
    assert np.all((d > -1e-12) & (d < 1e-3))
    assert np.isclose(c[4, 1], 4.2105, atol=1e-4) and np.isclose(c[2, 2], 1.0526, atol=1e-4)
    # the constant and the already-scaled cases of the same branch (:142-147)
    assert np.array_equal(oracle.tom_norm(np.full((3, 3), 4.0), 2), np.full((3, 3), 2.0))
    b = np.array([1.0, 2.0, 3.0])
    assert np.array_equal(oracle.tom_norm(b, 2), b)


def test_tom_norm_branches(oracle):
    """The string branches of tom_norm against their definitions, and the
    'mean0+1std' branch against the restatement the template statistics use."""
    rng = np.random.default_rng(4)
    a = rng.standard_normal((6, 5, 4)) * 3 + 1
    assert np.allclose(oracle.tom_norm(a, "mean0+1std"), oracle.tom_norm_mean0_1std(a), rtol=0, atol=1e-12)
    assert np.allclose(oracle.tom_norm(a), oracle.tom_norm_mean0_1std(a), rtol=0, atol=1e-12)
    m, s = a.mean(), a.std()
    assert np.allclose(oracle.tom_norm(a, "phase"), (a - m) / (m + 1e-12))
    for k in (1, 2, 3):
        assert np.allclose(oracle.tom_norm(a, f"{k}std"), np.clip(a, m - k * s, m + k * s) - m)
    mask = np.zeros(a.shape)
    mask[1:4, 1:4, 1:3] = 1
    v = a[mask > 0]
    mm, ms = v.mean(), v.std()
    assert np.allclose(oracle.tom_norm(a, "2std", mask), np.clip(a, mm - 2 * ms, mm + 2 * ms) - mm)
    c = np.clip(a, m - 3 * s, m + 3 * s) - m + 100
    assert np.allclose(oracle.tom_norm(a, "oscar"), (c - c.mean()) / (c.mean() + 1e-12))
    with pytest.raises(ValueError):
        oracle.tom_norm(a, "4std")


def test_rotation_axis_conventions(oracle):
    """Sptrans/tom_rotate.m:59-61: X axis ~ phi=0 psi=0 the=a; Y ~ phi=270 psi=90 the=a; Z ~ phi=a."""
    for a in (20.0, 37.0, 90.0):
        for e, axis in (((0, 0, a), 0), ((270, 90, a), 1), ((a, 0, 0), 2)):
            m = oracle.euler_matrix(e).reshape(3, 3).T  # rows: r = M p
            u = np.zeros(3)
            u[axis] = 1
            assert np.allclose(m @ u, u, atol=1e-6), (e, axis)


def test_local_stats_direct(oracle):
    """tom_os3_mean/std via FFT equal the direct masked sums (Roseman FLCF denominators)."""
    rng = np.random.default_rng(3)
    vol = rng.standard_normal((12, 10, 8))
    mask = oracle.sphere_mask((6, 6, 6), 2.5)
    mean, std, M = oracle.local_stats(vol, mask)
    c = 3
    for p in [(0, 0, 0), (5, 4, 3), (11, 9, 7)]:
        vals = []
        for j in np.argwhere(mask != 0):
            q = [(p[d] + j[d] - c) % vol.shape[d] for d in range(3)]
            vals.append(vol[tuple(q)])
        vals = np.array(vals)
        assert abs(mean[p] - vals.mean()) < 1e-12
        assert abs(std[p] - vals.std()) < 1e-10


def test_flcf_direct(oracle):
    """tom_os3_corr's FLCF equals the direct correlation sum at every voxel."""
    rng = np.random.default_rng(4)
    vol = rng.standard_normal((10, 12, 8))
    t = rng.standard_normal((6, 6, 6))
    mask = oracle.sphere_mask((6, 6, 6), 2.9)
    st = oracle.FLCF(vol, mask)
    tm, ts = 0.1, 1.3
    cc = st.corr(t, tm, ts)
    c = 3
    for p in [(0, 0, 0), (4, 7, 2), (9, 11, 7)]:
        s = 0.0
        for j in np.argwhere(mask != 0):
            q = [(p[d] + j[d] - c) % vol.shape[d] for d in range(3)]
            s += t[tuple(j)] * vol[tuple(q)]
        num = s / st.M - st.mean[p] * tm
        assert abs(cc[p] - num / (ts * st.std[p])) < 1e-10


def test_angle_grids(oracle):
    g0 = oracle.av3_angle_grid((0, 0, 0), (30, 30, 30), (330, 330, 180))
    assert len(g0) == 1008
    g1 = oracle.av3_angle_grid((0, 0, 0), (10, 10, 10), (350, 350, 180))
    assert len(g1) == 24624
    st, inc, en = (0, 0, 0), (30, 30, 30), (330, 330, 180)
    for i in (0, 1, 11, 12, 143, 144, 1007):
        a = g0[i]
        assert oracle.av3_angle2index(a, st, inc, en) == i
        assert np.allclose(oracle.av3_index2angle(i, st, inc, en), a)


# ------------------------------------------------------------- peak analysis

def _ifftshift_conv_direct(img, big_mask, x):
    """real(ifftshift(ifftn(fftn(img).*fftn(big_mask))))(x), written out."""
    N = img.shape
    s = 0.0
    for j in np.argwhere(big_mask != 0):
        q = tuple((x[d] + N[d] // 2 - j[d]) % N[d] for d in range(3))
        s += big_mask[tuple(j)] * img[q]
    return s


@pytest.mark.parametrize("N", [(12, 10, 14), (11, 13, 9)])
def test_psr_direct(oracle, N):
    """PSR of tom_os3_analyzePeak from tom_os3_mean/std written as sums over the
    pasted N-sized mask (odd and even sizes pin the ifftshift)."""
    rng = np.random.default_rng(31)
    pk = rng.standard_normal(N)
    T = (8, 8, 8)
    big = oracle.paste_center(N, oracle.psr_mask_box(T))
    M = (big != 0).sum()
    res = oracle.analyze_psr(pk, T)
    box = oracle.psr_mask_box(T)
    assert box.sum() == oracle.os3_sphere_mask(T)[0].sum() - 8   # 2x2x2 centre box zeroed
    for x in [(0, 0, 0), (5, 3, 7), (N[0] - 1, N[1] - 1, N[2] - 1)]:
        m = _ifftshift_conv_direct(pk, big, x) / M
        e2 = _ifftshift_conv_direct(pk * pk, big, x) / M
        sd = np.float32(np.sqrt(max(e2 - m * m, 0)))
        assert abs(res[x] - (pk[x] - m) / float(sd)) < 1e-9 * max(1, abs(res[x]))


def test_template_autocorr_direct(oracle):
    """tom_os3_corr(t, t): 1 at the centre; circular sums elsewhere."""
    rng = np.random.default_rng(32)
    T = (8, 8, 8)
    t = rng.standard_normal(T)
    A = oracle.os3_corr_same(t, t)
    c = 4
    assert abs(A[c, c, c] - 1) < 1e-12
    S = oracle.os3_sphere_mask(T)[0]
    M = S.sum()
    _, tm, ts = oracle.norm_under_mask(t, S)
    for x in [(0, 0, 0), (2, 5, 7), (7, 1, 3)]:
        num = sum(t[tuple((x[d] + c + j[d]) % 8 for d in range(3))] * t[tuple(j)] for j in np.argwhere(S != 0)) / M
        m = _ifftshift_conv_direct(t, S, x) / M
        e2 = _ifftshift_conv_direct(t * t, S, x) / M
        assert abs(A[x] - (num - m * tm) / (ts * np.sqrt(e2 - m * m))) < 1e-10


def test_analysis_ccc_only_is_find_template(oracle):
    rng = np.random.default_rng(33)
    vol = rng.standard_normal((16, 14, 12))
    T = 8
    tmpl = rng.standard_normal((T, T, T))
    mask = oracle.sphere_mask((T, T, T), 3)
    angles = oracle.av3_angle_grid((0, 0, 0), (90, 90, 90), (270, 90, 90))[:5]
    c1, i1 = oracle.find_template(vol, tmpl, mask, angles)
    c2, i2, p2, a2 = oracle.find_template_analysis(vol, tmpl, mask, angles)
    assert np.array_equal(i1, i2)
    assert np.abs(c1 - c2).max() < 1e-6
    assert np.all(np.isfinite(p2)) and np.all(np.isfinite(a2))


def test_tom_shift_integer(oracle):
    """tom_shift by whole voxels is a circular shift."""
    rng = np.random.default_rng(34)
    a = rng.standard_normal((8, 6, 10))
    b = oracle.tom_shift(a, (2, -1, 3))
    assert np.abs(b - np.roll(a, (2, -1, 3), axis=(0, 1, 2))).max() < 1e-12


def test_tom_limit(oracle):
    a = np.array([-4.0, -3.0, 0.5, 4.0, 5.0])
    assert np.array_equal(oracle.tom_limit(a, -3, 4, "z"), [0, -3, 0.5, 4, 4])
    assert np.array_equal(oracle.tom_limit(a, -3, 4), [-3, -3, 0.5, 4, 4])
    # the nested limits of the wedge weight are an indicator of >= 0.5
    w = np.array([0.0, 0.49, 0.5, 0.7, 1.0])
    assert np.array_equal(2 * oracle.tom_limit(oracle.tom_limit(w, 0.5, 1, "z"), 0, 0.5), [0, 0, 1, 1, 1])


# ------------------------------------------------------- C++ picker (corr3d)

def test_cpp_rotate_matches_reference_transform(ref_libs):
    """The C++ tom::rotate restatement against the reference's compiled transform.c."""
    o = ref_libs
    if not os.path.exists(os.path.join(o.REF_DIR, "libref_transform.so")):
        pytest.skip("libref_transform.so not built")
    rng = np.random.default_rng(35)
    v = rng.standard_normal((16, 12, 10)).astype(np.float32)
    # the matrix is composed directly here and by double inversion in the
    # reference: source coordinates agree to ~1e-16, so a rare voxel differs
    # by an ulp of its interpolation weight
    for ang in [(0.3, 0.7, 1.1), (1.0, -2.0, 0.5), (0.0, 0.0, 0.0), (2.5, 0.4, -1.3),
                (np.pi / 2, 0, np.pi / 2)]:
        a, b = o.cpp_rotate(v, *ang), o.ref_cpp_rotate(v, *ang)
        assert np.abs(a - b).max() <= 2e-7 * np.abs(v).max()
        assert (a != b).mean() < 0.05


def test_cpp_simple_wedge_halves(oracle):
    """The reduced SimpleWedge is the first nz/2+1 z-planes of the full one."""
    shape = (16, 12, 10)
    for ang in [(0.0, 0.0, 0.0), (0.4, 1.0, 0.3)]:
        full = oracle.cpp_simple_wedge(shape, np.deg2rad(30), 5, *ang, reduced=False)
        red = oracle.cpp_simple_wedge(shape, np.deg2rad(30), 5, *ang, reduced=True)
        assert np.array_equal(full[:, :, :shape[2] // 2 + 1], red)
        assert 0 < red.mean() < 1


def test_corr3d_finds_the_rotation(oracle):
    """A particle that is the template rotated by one of the angles is found at
    that angle with no shift and a coefficient near 1."""
    rng = np.random.default_rng(36)
    n = (16, 16, 16)
    t = np.zeros(n, np.float32)
    t[4:12, 5:11, 6:10] = rng.standard_normal((8, 6, 4))
    angles = [(0, 0, 0), (30, 20, 40), (90, 0, 45)]
    a = np.deg2rad(angles[1])
    m, v = oracle.cpp_stat(t)
    part = oracle.cpp_rotate(((t - m) / np.sqrt(v)).astype(np.float32), *a)
    res = oracle.corr3d_peaks([t], [part], angles)
    assert res["angle_idx"][0, 0] == 1
    assert tuple(res["peak"][0, 0]) == (0, 0, 0)
    assert res["val"][0, 0] > 0.99


# ------------------------------------------------------- learned proposer oracle

def test_cnn_conv_grads_finite_difference(oracle):
    """The FP64 convolution gradients against central differences."""
    rng = np.random.default_rng(37)
    x = rng.standard_normal((2, 5, 6, 7))
    w = rng.standard_normal((3, 2, 27)) * 0.3
    b = rng.standard_normal(3)
    g = rng.standard_normal((3, 5, 6, 7))
    for dil in (1, 2):
        gx, gw, gb = oracle.cnn_conv3d_grads(x, w, dil, g)
        f = lambda xx, ww, bb: float((g * oracle.cnn_conv3d(xx, ww, bb, dil)).sum())
        h = 1e-6
        for idx in [(0, 1, 2, 3), (1, 4, 5, 6), (0, 0, 0, 0)]:
            e = np.zeros_like(x)
            e[idx] = h
            assert abs((f(x + e, w, b) - f(x - e, w, b)) / (2 * h) - gx[idx]) < 1e-6
        for idx in [(0, 1, 13), (2, 0, 0), (1, 1, 26)]:
            e = np.zeros_like(w)
            e[idx] = h
            assert abs((f(x, w + e, b) - f(x, w - e, b)) / (2 * h) - gw[idx]) < 1e-6
        assert np.allclose(gb, g.sum(axis=(1, 2, 3)))


def test_cnn_losses_finite_difference(oracle):
    rng = np.random.default_rng(38)
    z = rng.standard_normal(50)
    y = (rng.random(50) > 0.8).astype(float)
    loss, g = oracle.cnn_bce(z, y, 5.0)
    h = 1e-6
    for i in (0, 7, 33):
        e = np.zeros(50)
        e[i] = h
        fd = (oracle.cnn_bce(z + e, y, 5.0)[0] - oracle.cnn_bce(z - e, y, 5.0)[0]) / (2 * h)
        assert abs(fd - g[i]) < 1e-8
    lg = rng.standard_normal((6, 4))
    lab = np.array([0, 5, 2, 2])
    loss, g = oracle.cnn_softmax_ce(lg, lab)
    for idx in [(0, 0), (5, 1), (3, 2)]:
        e = np.zeros_like(lg)
        e[idx] = h
        fd = (oracle.cnn_softmax_ce(lg + e, lab)[0] - oracle.cnn_softmax_ce(lg - e, lab)[0]) / (2 * h)
        assert abs(fd - g[idx]) < 1e-8


def test_constant_template_rule(oracle):
    """A constant template: tom_norm(...,'mean0+1std') leaves zeros
    (Sptrans/tom_norm.m:114-119 with std 0), its std under the mask is 0, so
    every FLCF denominator is 0 and tom_os3_corr.m:169-176 leaves 0 at every
    voxel; tom_os3_bestPeak's strict update then keeps the first angle
    everywhere (ccc 0, angle index 0)."""
    rng = np.random.default_rng(12)
    vol = rng.standard_normal((12, 10, 8))
    tmpl = np.full((6, 6, 6), 3.0)
    mask = oracle.sphere_mask((6, 6, 6), 2.5)
    angles = oracle.av3_angle_grid((0, 0, 0), (30, 30, 30), (330, 330, 180))[:7]
    t, tmean, tstd = oracle.prepare_template(tmpl, mask)
    assert not t.any() and tmean == 0 and tstd == 0
    ccc, idx = oracle.find_template(vol, tmpl, mask, angles)
    assert not ccc.any() and not idx.any()
