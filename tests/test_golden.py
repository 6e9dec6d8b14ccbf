"""The oracle's C restatement against golden outputs of the reference's own C
routines (tests/golden/reference_c.npz, made by tests/golden/make_golden.py
from the reference sources compiled into oracle/_ref).  Needs no reference
tree: this keeps the oracle pinned on any machine."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_c.npz")


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def _cases(g, prefix, suffix):
    return sorted({k[len(prefix):].split("_")[0] for k in g if k.startswith(prefix) and k.endswith(suffix)},
                  key=int)


def test_rot3d_golden(oracle, golden):
    """Sptrans/tom_rotatec.c rot3d, Euler and matrix mode: bit for bit."""
    g = golden
    cases = _cases(g, "rot", "_vol")
    assert len(cases) == 12
    for c in cases:
        vol, euler, cen = g[f"rot{c}_vol"], g[f"rot{c}_euler"], g[f"rot{c}_center"]
        center = None if np.isnan(cen).any() else tuple(float(x) for x in cen)
        got = oracle.rotate(vol, euler, center)
        assert np.array_equal(got.view(np.uint32), g[f"rot{c}_out"].view(np.uint32)), c
        got_m = oracle.rotate_matrix(vol, oracle.euler_matrix(euler), center)
        assert np.array_equal(got_m.view(np.uint32), g[f"rot{c}_matrix_out"].view(np.uint32)), c


def test_find_max_golden(oracle, golden):
    """Analysis/tom_peakinc.c find_max: the first strict maximum, value and position."""
    g = golden
    cases = _cases(g, "max", "_v")
    assert len(cases) == 6
    for c in cases:
        val, pos = oracle.find_max(g[f"max{c}_v"])
        assert np.float32(val) == g[f"max{c}_val"] and tuple(pos) == tuple(g[f"max{c}_pos"]), c


def test_weight3d_golden(oracle, golden):
    """Filtrans/tom_calc_weight_functioninc.c weight3d: bit for bit."""
    g = golden
    cases = _cases(g, "w", "_dims")
    assert len(cases) == 3
    for c in cases:
        got = oracle.weight3d(tuple(int(x) for x in g[f"w{c}_dims"]), g[f"w{c}_angles"], float(g[f"w{c}_thickness"]))
        assert np.array_equal(got, g[f"w{c}_out"]), c
