"""Checkpoint and resume of an angle search (tom_b200/checkpoint.py), on the
CPU with the oracle's FLCF loop as the engine: a search that fails or whose
process is killed resumes at its last checkpoint and ends bit-identical to
the uninterrupted search; a finished search is not rerun; checkpoints of
another search and damaged checkpoints are refused."""
import os
import subprocess
import sys

import numpy as np
import pytest

from tom_b200.checkpoint import (CheckpointCorrupt, CheckpointMismatch, SearchCheckpoint, job_key,
                                 run_checkpointed)

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from ckpt_engine import OracleEngine, small_job  # noqa: E402


@pytest.fixture(scope="module")
def job(oracle):
    return small_job(oracle)


@pytest.fixture(scope="module")
def reference(oracle, job, tmp_path_factory):
    vol, tmpl, mask, angles = job
    path = str(tmp_path_factory.mktemp("ref") / "ref.npz")
    cc, idx, info = run_checkpointed(OracleEngine(oracle, vol, tmpl, mask), angles, 5, path)
    assert info == {"resumed_at": 0, "chunks_run": 5, "checkpoints": 5}
    return cc, idx


def test_engine_is_the_oracle_search(oracle, job, reference):
    """The chunked engine finds the maxima of the oracle's one-call search
    (float32 running values: equal CC to float32 rounding, same angles)."""
    vol, tmpl, mask, angles = job
    ccc, idx = oracle.find_template(vol, tmpl, mask, angles)
    assert np.abs(reference[0] - ccc).max() <= 1e-6 * np.abs(ccc).max()
    assert (reference[1] != idx).mean() < 0.01


@pytest.mark.parametrize("chunk,every,fail_at", [(5, 1, 10), (5, 2, 15), (4, 1, 4), (3, 3, 20), (23, 1, 0)])
def test_resume_after_failure_is_bit_identical(oracle, job, reference, tmp_path, chunk, every, fail_at):
    vol, tmpl, mask, angles = job
    path = str(tmp_path / "ck.npz")
    if chunk != 5:  # the reference search used chunks of 5; recompute for this chunking
        ref = run_checkpointed(OracleEngine(oracle, vol, tmpl, mask), angles, chunk, str(tmp_path / "r.npz"))[:2]
    else:
        ref = reference
    with pytest.raises(RuntimeError, match="simulated failure"):
        run_checkpointed(OracleEngine(oracle, vol, tmpl, mask, fail_at=fail_at), angles, chunk, path, every=every)
    # the checkpoint holds the last multiple of `every` chunks finished before the failure
    done = (fail_at + chunk - 1) // chunk
    expect = (done // every) * every * chunk
    ck = SearchCheckpoint(path).load()
    if expect == 0:
        assert ck is None
    else:
        assert ck[0]["cursor"] == expect
    eng = OracleEngine(oracle, vol, tmpl, mask)
    cc, idx, info = run_checkpointed(eng, angles, chunk, path, every=every)
    assert info["resumed_at"] == expect
    assert eng.offsets and eng.offsets[0] == expect  # nothing finished is run again
    assert np.array_equal(cc, ref[0]) and np.array_equal(idx, ref[1])


def test_killed_process_resumes(oracle, job, reference, tmp_path):
    """The search runs in a child process that ends itself with os._exit in the
    middle of the angle list (no exception, no clean-up); the parent resumes."""
    path = str(tmp_path / "ck.npz")
    root = os.path.dirname(HERE)
    code = (
        "import sys\n"
        f"sys.path[:0] = [{root!r}, {os.path.join(root, 'oracle')!r}, {HERE!r}]\n"
        "import tm_oracle as O\n"
        "from ckpt_engine import OracleEngine, small_job\n"
        "from tom_b200.checkpoint import run_checkpointed\n"
        "vol, tmpl, mask, angles = small_job(O)\n"
        f"run_checkpointed(OracleEngine(O, vol, tmpl, mask, exit_at=15), angles, 5, {path!r})\n"
    )
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert p.returncode == 3, p.stderr[-2000:]
    assert SearchCheckpoint(path).load()[0]["cursor"] == 15
    vol, tmpl, mask, angles = job
    eng = OracleEngine(oracle, vol, tmpl, mask)
    cc, idx, info = run_checkpointed(eng, angles, 5, path)
    assert info["resumed_at"] == 15 and eng.offsets == [15, 20]
    assert np.array_equal(cc, reference[0]) and np.array_equal(idx, reference[1])


def test_finished_search_is_not_rerun(oracle, job, reference, tmp_path):
    vol, tmpl, mask, angles = job
    path = str(tmp_path / "ck.npz")
    run_checkpointed(OracleEngine(oracle, vol, tmpl, mask), angles, 5, path)
    cc, idx, info = run_checkpointed(OracleEngine(oracle, vol, tmpl, mask, fail_at=0), angles, 5, path)
    assert info == {"resumed_at": len(angles), "chunks_run": 0, "checkpoints": 0}
    assert np.array_equal(cc, reference[0]) and np.array_equal(idx, reference[1])


def test_checkpoint_of_another_search_is_refused(oracle, job, tmp_path):
    vol, tmpl, mask, angles = job
    path = str(tmp_path / "ck.npz")
    with pytest.raises(RuntimeError):
        run_checkpointed(OracleEngine(oracle, vol, tmpl, mask, fail_at=10), angles, 5, path)
    other = angles[::-1].copy()
    with pytest.raises(CheckpointMismatch):
        run_checkpointed(OracleEngine(oracle, vol, tmpl, mask), other, 5, path)
    with pytest.raises(CheckpointMismatch):  # same angles, another chunk
        run_checkpointed(OracleEngine(oracle, vol, tmpl, mask), angles, 4, path)
    with pytest.raises(CheckpointMismatch):  # same angles, the caller's key differs
        run_checkpointed(OracleEngine(oracle, vol, tmpl, mask), angles, 5, path, key={"tomogram_crc": 1})
    eng = OracleEngine(oracle, vol, tmpl, mask)
    cc, idx, info = run_checkpointed(eng, other, 5, path, on_mismatch="restart")
    assert info["resumed_at"] == 0 and eng.offsets[0] == 0
    assert SearchCheckpoint(path).load()[0]["job"] == job_key(vol.shape, other, 5)


def test_damaged_checkpoint_is_refused(oracle, job, tmp_path):
    vol, tmpl, mask, angles = job
    path = str(tmp_path / "ck.npz")
    with pytest.raises(RuntimeError):
        run_checkpointed(OracleEngine(oracle, vol, tmpl, mask, fail_at=10), angles, 5, path)
    good = open(path, "rb").read()
    # truncated file
    with open(path, "wb") as f:
        f.write(good[: len(good) // 2])
    with pytest.raises(CheckpointCorrupt):
        run_checkpointed(OracleEngine(oracle, vol, tmpl, mask), angles, 5, path)
    # one result value changed, the stored checksum kept
    with open(path, "wb") as f:
        f.write(good)
    with np.load(path, allow_pickle=False) as z:
        parts = {k: np.array(z[k]) for k in ("meta", "cc", "idx", "crc")}
    parts["cc"][1, 2, 3] += 1.0
    with open(path, "wb") as f:
        np.savez(f, **parts)
    with pytest.raises(CheckpointCorrupt, match="checksum"):
        SearchCheckpoint(path).load()
    # not a checkpoint at all
    with open(path, "wb") as f:
        np.savez(f, x=np.zeros(3))
    with pytest.raises(CheckpointCorrupt):
        SearchCheckpoint(path).load()


def test_interrupted_write_leaves_the_last_checkpoint(oracle, job, reference, tmp_path):
    """A save that died before its rename leaves a partial .tmp beside the last
    complete checkpoint: the resume reads the complete one and the next save
    replaces the partial file."""
    vol, tmpl, mask, angles = job
    path = str(tmp_path / "ck.npz")
    with pytest.raises(RuntimeError):
        run_checkpointed(OracleEngine(oracle, vol, tmpl, mask, fail_at=10), angles, 5, path)
    with open(path + ".tmp", "wb") as f:
        f.write(b"PK\x03\x04 partial")
    cc, idx, info = run_checkpointed(OracleEngine(oracle, vol, tmpl, mask), angles, 5, path)
    assert info["resumed_at"] == 10
    assert np.array_equal(cc, reference[0]) and np.array_equal(idx, reference[1])
    assert not os.path.exists(path + ".tmp")


class _HostCtx:
    device = 0

    def synchronize(self):
        pass


class _HostPlan:
    """The MatchPlan calls MatchPlanEngine makes, on host torch tensors in the
    device layout (z, y, x), each rotation's CC map from the oracle engine."""

    def __init__(self, oracle, vol, tmpl, mask):
        self.vol_shape = tuple(vol.shape)
        self.ctx = _HostCtx()
        self.maps = OracleEngine(oracle, vol, tmpl, mask)

    def new_results(self):
        import torch
        x, y, z = self.vol_shape
        cc, idx = torch.empty((z, y, x)), torch.empty((z, y, x), dtype=torch.int32)
        self.init_results(cc, idx)
        return cc, idx

    def init_results(self, cc, idx):
        cc.fill_(-1000.0)
        idx.fill_(-1)

    def run(self, eulers, cc, idx, index_offset=0):
        import torch
        for i, ang in enumerate(np.asarray(eulers)):
            self.maps.init()
            self.maps.run(ang[None], 0)
            c = torch.from_numpy(np.ascontiguousarray(self.maps.cc.transpose(2, 1, 0)))
            upd = cc < c
            cc[upd] = c[upd]
            idx[upd] = index_offset + i


def test_match_plan_engine_layout_and_resume(oracle, job, reference, tmp_path):
    """MatchPlanEngine reads the device layout (z, y, x) back as [x, y, z] and
    writes a resumed checkpoint into it: an interrupted and resumed search
    through it equals the oracle engine's search bit for bit."""
    from tom_b200.checkpoint import MatchPlanEngine
    vol, tmpl, mask, angles = job
    path = str(tmp_path / "ck.npz")

    class Failing(_HostPlan):
        def run(self, eulers, cc, idx, index_offset=0):
            if index_offset >= 15:
                raise RuntimeError("simulated failure")
            super().run(eulers, cc, idx, index_offset)

    with pytest.raises(RuntimeError):
        run_checkpointed(MatchPlanEngine(Failing(oracle, vol, tmpl, mask)), angles, 5, path)
    cc, idx, info = run_checkpointed(MatchPlanEngine(_HostPlan(oracle, vol, tmpl, mask)), angles, 5, path)
    assert info["resumed_at"] == 15
    assert cc.dtype == np.float32 and idx.dtype == np.int32 and cc.shape == vol.shape
    assert np.array_equal(cc, reference[0]) and np.array_equal(idx, reference[1])


def test_checkpointed_find_template_empty_volume(tmp_path):
    """tom_os3_findTemplate.m:221 and :309-313: an empty volume is not searched
    (ccc 0, angles -1000), so no device and no checkpoint are needed."""
    from tom_b200.checkpoint import find_template_checkpointed
    path = str(tmp_path / "ck.npz")
    ccc, ang, info = find_template_checkpointed(np.zeros((12, 10, 8), np.float32), np.ones((6, 6, 6)),
                                                np.zeros((4, 3)), path)
    assert ccc.shape == (12, 10, 8) and not ccc.any() and (ang == -1000).all()
    assert info["chunks_run"] == 0 and not os.path.exists(path)
