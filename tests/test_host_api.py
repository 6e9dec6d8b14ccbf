"""Host-side functions of tom_b200.tom that need no GPU: angle lists and
their index conventions, the mask builders and the motive-list layout,
against the reference's definitions and the oracle."""
import numpy as np

from conftest import needs_library
from tom_b200 import tom


def test_os3_axis_follows_the_reference_loop():
    """search/tom_os3_angleList.m (dim 2): start < end walks start:inc:end mod
    360; otherwise start+1:inc:end+359 into floor((360+end-start)/inc)+1
    preallocated zeros, which can leave a trailing 0."""
    assert tom._os3_axis(0, 30, 330) == list(range(0, 331, 30))
    assert tom._os3_axis(10, 20, 50) == [10, 30, 50]
    assert tom._os3_axis(300, 30, 60) == [301, 331, 1, 31, 0]   # 5 slots, 4 filled
    full = tom._os3_axis(0, 30, 0)                               # 13 slots, 12 filled
    assert full == list(range(1, 332, 30)) + [0]
    assert tom._os3_axis(350, 7, 20) == [351, 358, 5, 12, 19]    # slots = walk, no padding


def test_os3_angle_list_dedup():
    """Nested phi, psi, theta; a triplet is dropped when floor(R * 1e4) equals
    that of an earlier one.  The kept order is the nested order, every
    dropped triplet is the same rotation as a kept one, and no kept pair is
    the same rotation with the same floor key."""
    start, inc, end = (0, 0, 0), (30, 30, 30), (330, 330, 180)
    full = tom.tom_os3_angleList(start, inc, end, dedup=False)
    assert len(full) == 12 * 12 * 7
    assert np.array_equal(full[:3], [[0, 0, 0], [0, 0, 30], [0, 0, 60]])  # theta innermost
    kept = tom.tom_os3_angleList(start, inc, end)
    assert 744 <= len(kept) < len(full)  # 744 distinct rotations on this grid
    key = lambda a: tuple(np.floor(tom._rotmatrix(*a) * 10000).astype(np.int64).ravel())
    keys = [key(a) for a in kept]
    assert len(set(keys)) == len(keys)
    # kept triplets appear in the nested order
    pos = {tuple(a): i for i, a in enumerate(full)}
    order = [pos[tuple(a)] for a in kept]
    assert order == sorted(order)
    # every triplet of the grid has the key of a kept one, and is that rotation
    where = {k: i for i, k in enumerate(keys)}
    for a in full:
        i = where[key(a)]
        assert np.abs(tom._rotmatrix(*a) - tom._rotmatrix(*kept[i])).max() < 1e-9


@needs_library
def test_rotmatrix_is_the_zxz_matrix():
    """Rz(psi) Rx(theta) Rz(phi) (Sptrans/tom_sum_rotation.m) against the
    float32 matrix of tom_rotatec (rm.. order: column-major rows of R)."""
    rng = np.random.default_rng(3)
    for _ in range(20):
        e = rng.random(3) * 360
        R = tom._rotmatrix(*e)
        m = tom.euler_matrix(e).reshape(3, 3).T
        assert np.abs(R - m).max() < 1e-6


def test_av3_indices_round_trip_on_the_full_grid(oracle):
    """tom_av3_angle2index / index2angle (av3_new/tom_av3_angle2index.m:45-51,
    tom_av3_index2angle.m:47-54) over the 24,624-triplet 10-degree grid, and
    equal to the oracle's; an angle off the grid gives the count of triplets
    (the reference's search loop runs to its end)."""
    st, inc, en = (0, 0, 0), (10, 10, 10), (350, 350, 180)
    grid = tom.tom_av3_angle_grid(st, inc, en)
    assert len(grid) == 24624
    assert np.array_equal(grid, oracle.av3_angle_grid(st, inc, en))
    for i in list(range(0, 24624, 97)) + [1, 35, 36, 1295, 1296, 24623]:
        a = grid[i]
        assert tom.tom_av3_angle2index(a, st, inc, en) == i == oracle.av3_angle2index(a, st, inc, en)
        assert np.allclose(tom.tom_av3_index2angle(i, st, inc, en), a)
        assert np.allclose(tom.tom_av3_index2angle(i, st, inc, en), oracle.av3_index2angle(i, st, inc, en))
    assert tom.tom_av3_angle2index((360, 0, 0), st, inc, en) == 24624
    assert tom.tom_av3_angle2index((0, 0, 190), st, inc, en) == 24624


def test_sphere_masks(oracle):
    """tom_os3_sphereMask (search/tom_os3_sphereMask.m:4-37) equals the
    oracle's, with the count of its nonzeros; a non-cubic template gives
    ones.  tom_spheremask's default (Geom/tom_spheremask.m:41-67): radius
    floor((min n - 1)/2) about floor(n/2)+1, zero at distance >= radius."""
    for n in (6, 7, 16, 32, 33, 40):
        m, cnt = tom.tom_os3_sphereMask(np.zeros((n, n, n)))
        ref, _ = oracle.os3_sphere_mask((n, n, n))
        assert np.array_equal(m, ref) and cnt == int(ref.sum())
    m, cnt = tom.tom_os3_sphereMask(np.zeros((8, 8, 6)))
    assert m.all() and cnt == 8 * 8 * 6
    for shape in ((9, 9, 9), (10, 12, 8), (16, 16, 16)):
        r = np.floor((min(shape) - 1) / 2)
        ref = oracle.sphere_mask(shape, r, strict=False)
        assert np.array_equal(tom.tom_spheremask_default(shape), ref)


def test_picklist_to_motl_layout():
    """av3/alignment/av3_tomomatch.m:48-70: row 1 CCC, 4 particle number,
    8-10 x y z (1-based), 17-19 phi psi theta, 20 class; the rest 0."""
    vals = np.array([0.9, 0.7, 0.5])
    pos1 = np.array([[10, 20, 30], [1, 2, 3], [5, 6, 7]])
    eul = np.array([[10.0, 20.0, 30.0], [0.0, 90.0, 45.0], [350.0, 0.0, 180.0]])
    m = tom.picklist_to_motl(vals, pos1, eul, class_no=2)
    assert m.shape == (20, 3)
    assert np.array_equal(m[0], vals) and np.array_equal(m[3], [1, 2, 3])
    assert np.array_equal(m[7:10], pos1.T) and np.array_equal(m[16:19], eul.T)
    assert np.array_equal(m[19], [2, 2, 2])
    others = np.ones(20, bool)
    others[[0, 3, 7, 8, 9, 16, 17, 18, 19]] = False
    assert not m[others].any()
