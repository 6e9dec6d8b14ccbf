"""Angle partitioning across ranks and the final max/arg-max merge.

The search partitions by angle like the reference's job lists
(Oscar3/matlabPicker/search/tom_os3_createJobList.m:100-119): every rank holds
the whole tomogram and scans its own slice of the angle list; the only
exchange is one merge of the per-voxel (max CC, angle index) pairs at the end,
with tom_os3_bestPeak's rule (strictly larger CC wins; on equal CC the
earlier angle wins, search/tom_os3_bestPeak.m:42-47,94-96).

The merge packs each pair into one int64 key whose order is the rule's order
— high 32 bits: the CC mapped to an order-preserving integer, low 32 bits: the
complemented index — so a single all-reduce MAX (NCCL on GPUs, gloo on CPUs)
performs it.
"""
from __future__ import annotations


def angle_slice(n_angles: int, world: int, rank: int):
    """Contiguous slice [lo, hi) of the angle list for `rank`."""
    per = -(-n_angles // world)
    lo = min(n_angles, rank * per)
    return lo, min(n_angles, lo + per)


def pack_keys(cc, idx):
    """torch float32 CC and int32/64 index (>= -1) -> int64 keys."""
    import torch
    cc = cc.contiguous().to(torch.float32)
    cc = torch.where(cc == 0, torch.zeros_like(cc), cc)  # -0 == +0
    u = cc.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    neg = (u & 0x80000000) != 0
    ordk = torch.where(neg, (~u) & 0xFFFFFFFF, u | 0x80000000)
    hi = ordk - 0x80000000  # signed
    lo = (0x7FFFFFFF - idx.to(torch.int64)) & 0xFFFFFFFF
    return hi * (1 << 32) + lo


def unpack_keys(keys):
    import torch
    lo = keys & 0xFFFFFFFF
    hi = (keys - lo) // (1 << 32) + 0x80000000
    neg = (hi & 0x80000000) == 0
    u = torch.where(neg, (~hi) & 0xFFFFFFFF, hi & 0x7FFFFFFF)
    u = torch.where(u >= 0x80000000, u - (1 << 32), u).to(torch.int32)
    cc = u.view(torch.float32)
    idx = (0x7FFFFFFF - lo).to(torch.int64)
    idx = torch.where(idx > 0x7FFFFFFF, idx - (1 << 32), idx)
    return cc, idx.to(torch.int32)


def merge_results(cc, idx, group=None):
    """All-reduce the per-rank (max CC, index) volumes into the global result
    (in place semantics: returns new tensors)."""
    import torch.distributed as dist
    keys = pack_keys(cc, idx)
    dist.all_reduce(keys, op=dist.ReduceOp.MAX, group=group)
    return unpack_keys(keys)
