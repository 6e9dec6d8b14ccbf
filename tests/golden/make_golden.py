"""Generate tests/golden/reference_c.npz: outputs of the reference's own C
routines, compiled from its sources into oracle/_ref by oracle/Makefile
(`make -C oracle ref REF=<TOM source tree>`), on seeded inputs:

* rot3d (Sptrans/tom_rotatec.c:146-401): Euler and matrix mode, table and
  free angles, default and explicit centres, cubic and non-cubic volumes;
* find_max (Analysis/tom_peakinc.c:23-52): inputs with many ties;
* weight3d (Filtrans/tom_calc_weight_functioninc.c:152-252).

tests/test_golden.py checks the oracle's C restatement against these values,
so the oracle stays pinned where the reference sources are absent.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

TABLE = [0, 30, 45, 60, 90, 120, 135, 150, 180, 210, 225, 240, 270, 300, 315, 330]


def main():
    import tm_oracle as O
    if not O.ref_available():
        raise SystemExit("oracle/_ref not built: run `make -C oracle ref REF=<TOM source tree>`")
    rng = np.random.default_rng(2024)
    out = {}
    # rot3d
    for c in range(12):
        shape = tuple(int(x) for x in rng.integers(4, 11, 3)) if c % 3 else (8, 8, 8)
        vol = rng.standard_normal(shape).astype(np.float32)
        if c % 2:
            euler = rng.choice(TABLE, 3).astype(np.float32)
        else:
            euler = (rng.random(3) * 360).astype(np.float32)
        center = None if c % 4 < 2 else tuple(float(x) for x in rng.integers(0, 5, 3))
        res = O.ref_rotate(vol, euler, center)
        out[f"rot{c}_vol"] = np.asfortranarray(vol)
        out[f"rot{c}_euler"] = euler
        out[f"rot{c}_center"] = np.array(center if center is not None else [np.nan] * 3, np.float32)
        out[f"rot{c}_out"] = np.asfortranarray(res)
        m9 = O.euler_matrix(euler)
        out[f"rot{c}_matrix_out"] = np.asfortranarray(O.ref_rotate(vol, m9, center))
    # find_max
    for c in range(6):
        v = rng.integers(-3, 4, tuple(int(x) for x in rng.integers(3, 8, 3))).astype(np.float32)
        val, pos = O.ref_find_max(v)
        out[f"max{c}_v"] = np.asfortranarray(v)
        out[f"max{c}_val"] = np.float32(val)
        out[f"max{c}_pos"] = np.array(pos, np.int32)
    # weight3d
    cases = [((16, 12, 10), [[0, 0, 0, 0], [-60, -20, 20, 60]], 16.0),
             ((9, 8, 7), [[10, 30], [-45, 50]], 5.0),
             ((12, 12, 12), np.vstack([np.zeros(21), np.arange(-60, 61, 6)]), 32.0)]
    for c, (dims, ang, th) in enumerate(cases):
        out[f"w{c}_dims"] = np.array(dims, np.int32)
        out[f"w{c}_angles"] = np.asarray(ang, np.float64)
        out[f"w{c}_thickness"] = np.float64(th)
        out[f"w{c}_out"] = O.ref_weight3d(dims, np.asarray(ang, np.float64), th)
    path = os.path.join(HERE, "reference_c.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
