"""The synthetic benchmark inputs follow their definitions: the missing wedge
applied to the tomogram is the reference's tom_wedge(., 90 - tilt) =
av3_wedge(-tilt, +tilt) on the spectrum, and particle centres keep their
spacing and borders."""
import numpy as np
import pytest

from tom_b200 import synth


@pytest.mark.parametrize("shape", [(16, 12, 10), (15, 12, 9), (32, 8, 20)])
@pytest.mark.parametrize("tilt", [45, 55, 60])
def test_wedge_fourier_is_tom_wedge(oracle, shape, tilt):
    """wedge_fourier on an impulse returns the kept half spectrum; it equals
    Filtrans/tom_wedge.m:62-77 at 90 - tilt, moved from the centred grid to
    the FFT layout (ifftshift) and cut to the half x axis."""
    imp = np.zeros(shape, np.float32, order="F")
    imp[0, 0, 0] = 1.0
    out = synth.wedge_fourier(imp, tilt)
    spec = np.fft.rfftn(out.astype(np.float64), axes=(2, 1, 0))
    kept = np.abs(spec) > 0.5
    assert np.all((np.abs(spec) < 1e-4) | (np.abs(spec - 1) < 1e-4))
    w = np.fft.ifftshift(oracle.tom_wedge(shape, 90 - tilt))[: shape[0] // 2 + 1]
    assert np.array_equal(kept, w > 0)


@pytest.mark.parametrize("tilt", [45, 55, 60])
def test_av3_wedge_is_tom_wedge_complement(oracle, tilt):
    """av3/utils/av3_wedge.m:23-26 with (-tilt, +tilt) zeroes the same voxels
    as tom_wedge at 90 - tilt (the z = 0 plane kept by both)."""
    for shape in ((16, 12, 10), (15, 13, 9)):
        assert np.array_equal(oracle.av3_wedge(shape, -tilt, tilt), oracle.tom_wedge(shape, 90 - tilt))


def test_place_copies_spacing_and_borders():
    N, T = (128, 96, 64), 24
    a = synth.place_copies(np.random.default_rng(5), N, T, 20)
    b = synth.place_copies(np.random.default_rng(5), N, T, 20)
    assert np.array_equal(a, b) and len(a) == 20
    for d in range(3):
        assert a[:, d].min() >= T / 2 - 0.5 and a[:, d].max() <= N[d] - T / 2 + 0.5
    dist = np.linalg.norm(a[:, None] - a[None], axis=-1)
    assert dist[np.triu_indices(len(a), 1)].min() >= T


def test_rotation_matrices_and_geodesic_neighbours():
    """proposer.rotation_matrices is the transpose of synth.rot3d_matrix (the
    same rotation, column-major as tom_rotatec lists it) and neighbours()
    returns exactly the fine triplets within the geodesic radius."""
    from tom_b200 import proposer as pr
    import tom_b200 as tb
    rng = np.random.default_rng(5)
    e = np.column_stack([rng.uniform(0, 360, 20), rng.uniform(0, 360, 20), rng.uniform(0, 180, 20)])
    R = pr.rotation_matrices(e)
    for k in range(len(e)):
        assert np.allclose(R[k], synth.rot3d_matrix(e[k]).T, atol=1e-12)
        assert np.allclose(R[k] @ R[k].T, np.eye(3), atol=1e-12)
    fine = tb.tom_av3_angle_grid((0, 0, 0), (20, 20, 20), (340, 340, 180))
    centres = e[:5]
    Rf = pr.rotation_matrices(fine)
    for c, ids in zip(centres, pr.neighbours(fine, centres, 25.0)):
        Rc = pr.rotation_matrices([c])[0]
        ang = np.degrees(np.arccos(np.clip((np.einsum("kij,ij->k", Rf, Rc) - 1) / 2, -1, 1)))
        assert set(ids.tolist()) == set(np.nonzero(ang <= 25.0 + 1e-7)[0].tolist())
