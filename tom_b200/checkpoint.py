"""Checkpoint and resume of a long angle search.

The reference keeps a long search restartable with per-job result files that
are saved, read back and re-saved until the read succeeds
(Oscar3/matlabPicker/tools/tom_os3_secureSave.m, up to 10 retries), a list of
jobs without a result (results/tom_os3_checkMissingResults.m) and a rest-job
list the picker resumes from (tom_os3_picker.m:147-148).  Here one search is
the job and the angle list is cut into fixed chunks:

* after every `every` chunks the running (max CC, angle index) volumes and
  the cursor (angles done) are written to one .npz file under a temporary
  name, read back and checked against their CRC-32, and only then renamed
  over the previous checkpoint, so a checkpoint on disk is always complete;
  a failed write or read-back is retried up to 10 times;
* a search started on the same job (volume and template sizes, the angle
  list, the chunk, and the caller's own key such as input checksums) resumes
  at the cursor; a checkpoint of another job is refused (or ignored on
  request), a damaged one raises;
* a finished search leaves a checkpoint with the cursor at the end, and a
  rerun returns its volumes without running anything.

Every chunk is run as the same call with the same global angle offset
whether or not the search was interrupted, and the running maximum keeps the
first angle on ties, so the resumed result equals the uninterrupted one bit
for bit.

The search itself is an engine: any object with ``shape`` (x, y, z) and the
methods ``init()`` (results to their initial values), ``run(eulers,
index_offset)``, ``read() -> (cc, idx)`` (host copies, [x, y, z]) and
``write(cc, idx)`` (restore).  ``MatchPlanEngine`` drives a
:class:`tom_b200.tom.MatchPlan` on the device.
"""
from __future__ import annotations

import hashlib
import json
import os
import zipfile
import zlib

import numpy as np

FORMAT = "tomgpu-search-checkpoint-1"
RETRIES = 10



def _fsync_dir(d: str) -> None:
    """Flush a directory entry (the rename of a new checkpoint) to disk, so a
    power loss after save() returns does not bring back the older checkpoint.
    POSIX only: elsewhere directories cannot be opened and this does nothing."""
    if os.name != "posix":
        return
    fd = os.open(d, os.O_RDONLY)
    try:
        os.fsync(fd)
    finally:
        os.close(fd)

class CheckpointMismatch(RuntimeError):
    """The checkpoint on disk belongs to another search."""


class CheckpointCorrupt(RuntimeError):
    """The checkpoint on disk is incomplete or fails its checksum."""


def _crc(meta_json: str, cc: np.ndarray, idx: np.ndarray) -> int:
    c = zlib.crc32(meta_json.encode())
    for a in (cc, idx):
        c = zlib.crc32(memoryview(np.ascontiguousarray(a).reshape(-1).view(np.uint8)), c)
    return c


def job_key(shape, eulers, chunk: int, extra: dict | None = None) -> dict:
    """What identifies a search: sizes, the angle list (SHA-256 of its float32
    bytes), the chunk and the caller's own entries."""
    e = np.ascontiguousarray(np.asarray(eulers, np.float32).reshape(-1, 3))
    key = {"shape": [int(s) for s in shape], "angles": int(e.shape[0]),
           "angles_sha256": hashlib.sha256(e.tobytes()).hexdigest(), "chunk": int(chunk)}
    if extra:
        key["extra"] = json.loads(json.dumps(extra, sort_keys=True))
    return key


class SearchCheckpoint:
    """One checkpoint file: atomic save with read-back, verified load."""

    def __init__(self, path: str):
        self.path = os.fspath(path)

    def exists(self) -> bool:
        return os.path.exists(self.path)

    def load(self):
        """(meta, cc, idx) of the checkpoint, or None if there is none."""
        if not self.exists():
            return None
        return self._read(self.path)

    @staticmethod
    def _read(path):
        try:
            with np.load(path, allow_pickle=False) as z:
                meta_json = str(z["meta"][()])
                cc = np.asfortranarray(z["cc"])
                idx = np.asfortranarray(z["idx"])
                crc = int(z["crc"][()])
            meta = json.loads(meta_json)
            fmt = meta.get("format") if isinstance(meta, dict) else None
            shape = tuple(meta["job"]["shape"]) if fmt == FORMAT else None
            int(meta["cursor"]) if fmt == FORMAT else None
        except (OSError, ValueError, KeyError, TypeError, EOFError, zipfile.BadZipFile) as e:
            raise CheckpointCorrupt(f"{path}: unreadable checkpoint ({e})") from e
        if fmt != FORMAT:
            raise CheckpointCorrupt(f"{path}: not a search checkpoint")
        if _crc(meta_json, cc, idx) != crc:
            raise CheckpointCorrupt(f"{path}: checksum mismatch")
        if cc.shape != shape or idx.shape != shape or cc.dtype != np.float32 or idx.dtype != np.int32:
            raise CheckpointCorrupt(f"{path}: result volumes do not match the recorded sizes")
        return meta, cc, idx

    def save(self, job: dict, cursor: int, cc: np.ndarray, idx: np.ndarray) -> None:
        cc = np.asarray(cc, np.float32)
        idx = np.asarray(idx, np.int32)
        meta_json = json.dumps({"format": FORMAT, "job": job, "cursor": int(cursor)}, sort_keys=True)
        crc = _crc(meta_json, cc, idx)
        tmp = self.path + ".tmp"
        last = None
        for _ in range(RETRIES):
            try:
                with open(tmp, "wb") as f:
                    np.savez(f, meta=np.array(meta_json), cc=np.ascontiguousarray(cc),
                             idx=np.ascontiguousarray(idx), crc=np.array(crc, np.int64))
                    f.flush()
                    os.fsync(f.fileno())
                meta, _, _ = self._read(tmp)  # read back before it replaces the last good one
                if meta["cursor"] != int(cursor):
                    raise CheckpointCorrupt(f"{tmp}: cursor read back wrong")
                os.replace(tmp, self.path)
                _fsync_dir(os.path.dirname(os.path.abspath(self.path)))
                return
            except (OSError, CheckpointCorrupt) as e:
                last = e
                try:
                    os.remove(tmp)
                except OSError:
                    pass
        raise OSError(f"{self.path}: checkpoint not written after {RETRIES} attempts ({last})")

    def remove(self) -> None:
        for p in (self.path, self.path + ".tmp"):
            try:
                os.remove(p)
            except FileNotFoundError:
                pass


def run_checkpointed(engine, eulers, chunk: int, path: str, every: int = 1, key: dict | None = None,
                     on_mismatch: str = "error"):
    """Search all of `eulers` (R x 3, degrees) in chunks of `chunk` rotations,
    checkpointing to `path` after every `every` chunks and at the end, and
    resuming from the checkpoint there.  Returns (cc, idx, info): the result
    volumes ([x, y, z] float32 / int32, 0-based angle index, -1 where never
    updated) and {"resumed_at", "chunks_run", "checkpoints"}.

    on_mismatch: "error" raises CheckpointMismatch when the checkpoint on disk
    belongs to another search; "restart" starts over and replaces it."""
    if chunk <= 0 or every <= 0:
        raise ValueError("chunk and every must be positive")
    if on_mismatch not in ("error", "restart"):
        raise ValueError("on_mismatch is 'error' or 'restart'")
    e = np.ascontiguousarray(np.asarray(eulers, np.float32).reshape(-1, 3))
    R = e.shape[0]
    job = job_key(engine.shape, e, chunk, key)
    ck = SearchCheckpoint(path)
    state = ck.load()
    if state is not None and state[0]["job"] != job:
        if on_mismatch == "error":
            raise CheckpointMismatch(f"{path} holds a checkpoint of another search")
        state = None
    start = 0
    if state is not None:
        meta, cc, idx = state
        start = int(meta["cursor"])
        if start >= R:
            return cc, idx, {"resumed_at": start, "chunks_run": 0, "checkpoints": 0}
    engine.init()
    if start:
        engine.write(cc, idx)
    info = {"resumed_at": start, "chunks_run": 0, "checkpoints": 0}
    pending = 0
    for s in range(start, R, chunk):
        engine.run(e[s:s + chunk], s)
        info["chunks_run"] += 1
        pending += 1
        done = min(s + chunk, R)
        if pending >= every or done == R:
            cc, idx = engine.read()
            ck.save(job, done, cc, idx)
            info["checkpoints"] += 1
            pending = 0
    if R == 0:
        cc, idx = engine.read()
    return cc, idx, info


class MatchPlanEngine:
    """A device-resident search (MatchPlan with its template and volume set)
    as a checkpointable engine; results live in device buffers between
    chunks and cross to the host only at a checkpoint."""

    def __init__(self, plan):
        self.plan = plan
        self.shape = tuple(plan.vol_shape)
        self.cc = self.idx = None

    def init(self):
        if self.cc is None:
            self.cc, self.idx = self.plan.new_results()
        else:
            self.plan.init_results(self.cc, self.idx)

    def run(self, eulers, index_offset):
        self.plan.run(eulers, self.cc, self.idx, index_offset=index_offset)

    def _sync(self):
        import torch
        if self.cc.is_cuda:
            torch.cuda.synchronize(self.cc.device)

    def read(self):
        from .tom import from_device
        self.plan.ctx.synchronize()
        self._sync()
        return (np.asfortranarray(from_device(self.cc)).astype(np.float32, copy=True),
                np.asfortranarray(from_device(self.idx)).astype(np.int32, copy=True))

    def write(self, cc, idx):
        import torch
        self.plan.ctx.synchronize()
        for dst, src, dt in ((self.cc, cc, np.float32), (self.idx, idx, np.int32)):
            host = torch.from_numpy(np.ascontiguousarray(np.asarray(src, dt).transpose(2, 1, 0)))
            dst.copy_(host)
        self._sync()


def _crc32(a) -> int:
    return zlib.crc32(memoryview(np.ascontiguousarray(a).reshape(-1).view(np.uint8)))


def find_template_checkpointed(volume, template, angle_list, path, mask=None, psf=None, batch: int = 0,
                               chunk: int = 1024, every: int = 1, on_mismatch: str = "error", ctx=None):
    """[ccc angles] of tom_os3_findTemplate (the ccc-only search, as
    tom_b200.tom.tom_os3_findTemplate) run in chunks of `chunk` rotations with
    a checkpoint at `path` after every `every` chunks; a call with the same
    inputs resumes there.  The job key holds CRC-32s of the tomogram,
    template, mask and psf, so a checkpoint is never resumed with other
    inputs.  Returns (ccc, angles, info): the reference's conventions
    (angles 1-based as float32, -1000 where never updated) and the resume
    record of run_checkpointed."""
    from .tom import MatchPlan, default_context, tom_os3_sphereMask, to_device
    vol = np.asarray(volume, np.float32)
    t = np.asarray(template, np.float32)
    if mask is None:
        mask, _ = tom_os3_sphereMask(t)
    mask = np.asarray(mask, np.float32)
    if not np.any(vol):
        # tom_os3_findTemplate.m:221 and :309-313: an empty volume is not searched
        return (np.zeros(vol.shape, np.float32, order="F"), np.full(vol.shape, -1000, np.float32, order="F"),
                {"resumed_at": 0, "chunks_run": 0, "checkpoints": 0})
    key = {"tomogram_crc32": _crc32(vol), "template_shape": list(t.shape), "template_crc32": _crc32(t),
           "mask_crc32": _crc32(mask), "psf_crc32": None if psf is None else _crc32(np.asarray(psf, np.float32))}
    ctx = ctx or default_context()
    plan = MatchPlan(vol.shape, t.shape, batch=batch, ctx=ctx)
    try:
        plan.set_template(to_device(t, ctx.device), to_device(mask, ctx.device),
                          to_device(psf, ctx.device) if psf is not None else None)
        plan.set_volume(to_device(vol, ctx.device))
        cc, idx, info = run_checkpointed(MatchPlanEngine(plan), angle_list, chunk, path, every=every, key=key,
                                         on_mismatch=on_mismatch)
    finally:
        plan.close()
    ang = np.where(idx >= 0, idx.astype(np.float32) + 1, -1000).astype(np.float32)
    return np.asfortranarray(cc), np.asfortranarray(ang), info
