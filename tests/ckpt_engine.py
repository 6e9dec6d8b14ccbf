"""A checkpointable search engine for the CPU tests of tom_b200.checkpoint:
the oracle's tom_os3_findTemplate loop (tom_os3_findTemplate.m:255-307 with
tom_os3_bestPeak's strict update) run one chunk of angles at a time, results
kept in float32 / int32 like the device search.  Test infrastructure."""
import os

import numpy as np


def small_job(oracle, seed=6, n_angles=23):
    rng = np.random.default_rng(seed)
    vol = rng.standard_normal((12, 10, 8))
    tmpl = rng.standard_normal((6, 6, 6))
    mask = oracle.sphere_mask((6, 6, 6), 2.5)
    angles = oracle.av3_angle_grid((0, 0, 0), (30, 30, 30), (330, 330, 180))[:n_angles]
    return vol, tmpl, mask, angles


class OracleEngine:
    """fail_at: raise RuntimeError when a chunk at or past this angle offset
    starts; exit_at: end the whole process there (os._exit), as a killed
    process would, with no exception handling or clean-up."""

    def __init__(self, oracle, vol, tmpl, mask, fail_at=None, exit_at=None):
        self.O = oracle
        self.shape = tuple(vol.shape)
        self.t, self.tm, self.ts = oracle.prepare_template(tmpl, mask)
        self.st = oracle.FLCF(vol, mask)
        self.mask = mask
        self.fail_at, self.exit_at = fail_at, exit_at
        self.offsets = []

    def init(self):
        self.cc = np.full(self.shape, -1000.0, np.float32, order="F")
        self.idx = np.full(self.shape, -1, np.int32, order="F")

    def run(self, eulers, index_offset):
        if self.exit_at is not None and index_offset >= self.exit_at:
            os._exit(3)
        if self.fail_at is not None and index_offset >= self.fail_at:
            raise RuntimeError("simulated failure")
        self.offsets.append(index_offset)
        for i, ang in enumerate(np.asarray(eulers, np.float64)):
            tr = self.O.rotate(self.t.astype(np.float32), ang).astype(np.float64) * self.mask
            c = self.st.corr(tr.astype(np.float32).astype(np.float64), self.tm, self.ts).astype(np.float32)
            upd = self.cc < c
            self.cc[upd] = c[upd]
            self.idx[upd] = index_offset + i

    def read(self):
        return self.cc.copy(order="F"), self.idx.copy(order="F")

    def write(self, cc, idx):
        self.cc = np.array(cc, np.float32, order="F")
        self.idx = np.array(idx, np.int32, order="F")
