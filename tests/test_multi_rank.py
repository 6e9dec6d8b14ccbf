"""Angle-partitioned search on world-size-2 gloo ranks (CPU): each rank scans
its slice of the angle list with the oracle and the ranks merge with one
all-reduce; the result equals the single-process search over all angles."""
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _case():
    import tm_oracle as O
    rng = np.random.default_rng(31)
    vol = rng.standard_normal((24, 20, 16))
    tmpl = rng.standard_normal((8, 8, 8))
    mask = O.sphere_mask((8, 8, 8), 3.5)
    angles = O.av3_angle_grid((0, 0, 0), (90, 90, 90), (270, 90, 90))
    return vol, tmpl, mask, angles


def _worker(rank, world, port, out_dir, root):
    import sys
    sys.path[:0] = [root, os.path.join(root, "oracle")]
    import torch.distributed as dist
    import tm_oracle as O
    from tom_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    vol, tmpl, mask, angles = _case()
    lo, hi = shard.angle_slice(len(angles), world, rank)
    cc, idx = O.find_template(vol, tmpl, mask, angles[lo:hi])
    idx = np.where(idx >= 0, idx + lo, -1)
    c, i = shard.merge_results(torch.from_numpy(cc.astype(np.float32)), torch.from_numpy(idx.astype(np.int32)))
    np.save(os.path.join(out_dir, f"cc{rank}.npy"), c.numpy())
    np.save(os.path.join(out_dir, f"idx{rank}.npy"), i.numpy())
    dist.destroy_process_group()


def test_two_rank_merge_equals_single_search(tmp_path, oracle):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path), root), nprocs=2, start_method="spawn")
    vol, tmpl, mask, angles = _case()
    ref_cc, ref_idx = oracle.find_template(vol, tmpl, mask, angles)
    for r in range(2):
        cc = np.load(tmp_path / f"cc{r}.npy")
        idx = np.load(tmp_path / f"idx{r}.npy")
        assert np.array_equal(cc, ref_cc.astype(np.float32))
        assert np.array_equal(idx, ref_idx)


def test_key_packing_order():
    from tom_b200 import shard
    rng = np.random.default_rng(3)
    cc = np.concatenate([rng.standard_normal(200).astype(np.float32), [0.0, -0.0, 1.5, 1.5, -1000.0]])
    idx = np.concatenate([rng.integers(0, 5000, 200), [3, 2, 7, 4, -1]]).astype(np.int32)
    k = shard.pack_keys(torch.from_numpy(cc), torch.from_numpy(idx)).numpy()
    c2, i2 = shard.unpack_keys(torch.from_numpy(k))
    assert np.array_equal(c2.numpy(), np.where(cc == 0, 0, cc).astype(np.float32))
    assert np.array_equal(i2.numpy(), idx)
    # order: larger CC first, then smaller index
    order = sorted(range(len(cc)), key=lambda j: (float(cc[j]), -int(idx[j])))
    assert np.all(np.diff(k[order]) >= 0)


def _bestpeak_merge(parts):
    """The checker: merge [(cc, idx), ...] in rank order with tom_os3_bestPeak's
    rule (search/tom_os3_bestPeak.m:42-47: a strictly larger CC replaces, so on
    equal CC the earlier rank's, i.e. earlier angle's, pair stays)."""
    cc = parts[0][0].astype(np.float32).copy()
    idx = parts[0][1].astype(np.int32).copy()
    for c, i in parts[1:]:
        better = c > cc
        cc = np.where(better, c, cc)
        idx = np.where(better, i, idx)
    return cc, idx


def test_key_max_merge_is_the_bestpeak_merge():
    """One elementwise MAX over the ranks' packed keys (what the all-reduce
    computes) equals the rank-order bestPeak merge, with CCs quantised so
    ranks tie often, signed zeros, and voxels a rank never updated."""
    from tom_b200 import shard
    rng = np.random.default_rng(8)
    n, world, n_angles = 4000, 4, 1000
    parts = []
    for r in range(world):
        lo, hi = shard.angle_slice(n_angles, world, r)
        cc = (np.round(rng.standard_normal(n) * 4) / 8).astype(np.float32)
        cc[rng.random(n) < 0.05] = -0.0
        idx = rng.integers(lo, hi, n).astype(np.int32)
        unset = rng.random(n) < 0.02
        cc[unset], idx[unset] = -1000.0, -1
        parts.append((cc, idx))
    keys = np.max(np.stack([shard.pack_keys(torch.from_numpy(c), torch.from_numpy(i)).numpy() for c, i in parts]),
                  axis=0)
    c2, i2 = shard.unpack_keys(torch.from_numpy(keys))
    ref_cc, ref_idx = _bestpeak_merge(parts)
    assert np.array_equal(c2.numpy(), np.where(ref_cc == 0, 0, ref_cc).astype(np.float32))
    # where every rank left -1000 / -1 the merge keeps -1; elsewhere the indices agree
    assert np.array_equal(i2.numpy(), ref_idx)


def test_angle_slices_cover_exactly():
    from tom_b200 import shard
    for n in (1, 7, 1008, 24624):
        for w in (1, 2, 3, 8):
            s = [shard.angle_slice(n, w, r) for r in range(w)]
            covered = np.concatenate([np.arange(lo, hi) for lo, hi in s])
            assert np.array_equal(covered, np.arange(n))
