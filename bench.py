#!/usr/bin/env python
"""Exhaustive FLCF template-matching benchmark (rot*voxel/s).

Workload: the 512x512x256 FP32 tomogram / 40^3 template search (8-blob
phantom, 40 copies, SNR 0.1, +-55 degree wedge, mask radius 16) over its 10
degree ZXZ grid (36 x 36 x 19 = 24,624 triplets), synthetic seeded data.

A step is one pass of the hot path (rotate -> mask -> FFT correlation -> FLCF
-> running max/arg-max) over one chunk of `--rot-per-step` Euler triplets
against the whole tomogram; step s on rank r takes chunk s*world + r of the
grid (angle partitioning, so per-GPU work is fixed as N grows: weak scaling;
every rank holds the same tomogram spectrum).

  python bench.py --gpus N --steps K --warmup W [--impl reference]

Rank 0 prints one JSON line.  `value` is rot*voxel/s of the timed region
(device time, CUDA events, max over ranks); `e2e` is the same metric through
the one-shot C-ABI call tomgpu_match with pinned host buffers (upload of the
tomogram, FP64 statistics, the search, download of max-CC and angle index
inside the timed region).  Before the timed region the rotation batch is
autotuned over 8, 16, 32 and 64 (those that fit); the device-resident plan is
released before the end-to-end leg builds its own.

Other workloads (`--workload`, each its own JSON line; not the headline):
exhaustive_928x928x464 and exhaustive_128 (the same search at other sizes),
pruned_928x928x464 (the pruned search against the exhaustive one),
align_2048 (batched subtomogram alignment), learned_256 (the coarse-map CNN
proposer), unet (the U-Net's tensor-core forward and training throughput)
and learned_928x928x464 (the U-Net proposer on the full-size tomogram: its
learned-pruned search, its candidates alone, and its ranking of the coarse
search's candidates against their CC at equal counts).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "exhaustive_512x512x256"
METRIC = "TM rot*voxel/s (exhaustive FLCF, 512x512x256 tomogram, 40^3 template)"
UNIT = "rot*voxel/s"

# DRAM bytes (read + write) per launch of a kernel class at a rotation batch,
# from ncu captures of thinner volumes with the same x and y edges, scaled by
# the voxel count (every term of these kernels' traffic scales with it):
# 512x128x64 (batch 16, 32: the cp.async x-line kernel) and 512x512x48
# (batch 64: the TMA x-line kernel and the y-column kernel), 512x64x256 at
# batch 16 (the z-line kernel; its traffic also scales with the batch) for
# the 512x512x256 tomogram; 928x928x48 (batch 32) for the 928x928x464 one.
TRAFFIC = {"exhaustive_512x512x256": {"c2r_flcf": {16: 16 * (336639232 + 22247680),
                                                  32: 16 * (606162432 + 24264960),
                                                  64: 256 / 48 * (3435212032 + 94609920)},
                                     "corr_y": {64: 256 / 48 * (303350272 + 3173413120)},
                                     "inv_z": {64: 32 * (538986496 + 487509760)}},
           "exhaustive_928x928x464": {"c2r_flcf": {32: 464 / 48 * (5964541184 + 316938496)},
                                      "corr_y": {32: 464 / 48 * (440176384 + 5247565312)}}}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--rot-per-step", type=int, default=64)
    p.add_argument("--batch", type=int, default=0,
                   help="rotation batch; 0 = autotune over 8, 16, 32, 64 before the timed region")
    p.add_argument("--path", type=int, default=0, choices=[0, 1, 2, 3],
                   help="kernel path of the plan: 0 fastest (TMA x-line tiles at the 512 x edge), 1 generic, "
                        "2 as 0 with cp.async x-line tiles, 3 as 0 with the tcgen05 inverse z-DFT")
    p.add_argument("--e2e-rot", type=int, default=0,
                   help="rotations per end-to-end call; 0: the whole angle grid in one call (a whole search, "
                        "as tom_os3_findTemplate makes it) when it holds at most 25,000 triplets, else 2048")
    p.add_argument("--e2e-steps", type=int, default=0,
                   help="end-to-end calls timed; 0: one for a whole-grid call, else 3")
    p.add_argument("--cpu-seconds", type=float, default=20.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--rescore-k", type=int, default=None,
                   help="top-K peaks rescored in FP64 after the timed region (default 200; 1000 for the "
                        "928x928x464 workload)")
    p.add_argument("--learned-train", type=int, default=8, help="training tomograms of the learned_256 workload")
    p.add_argument("--learned-steps", type=int, default=400, help="timed training steps of the learned_256 workload")
    p.add_argument("--align-particles", type=int, default=40,
                   help="particles timed for --workload align_2048 (extrapolated to 2048 from the per-edge "
                        "times; 2048 times the whole workload once)")
    p.add_argument("--align-batch-mb", type=int, default=0,
                   help="align_2048: device MB of a batch's spectra in the batched engine (0: the library default)")
    p.add_argument("--align-path", type=int, default=0, choices=[0, 1, 2],
                   help="align_2048: 0 the batched engine (entries of all particles of a box edge), 1 one job at "
                        "a time, 2 batched without the pruned last inverse DFT")
    p.add_argument("--pruned-step", type=int, default=21, help="pruned_928x928x464: coarse grid step (degrees)")
    p.add_argument("--pruned-cands", type=float, default=2.0,
                   help="pruned_928x928x464: candidates per particle of the tomogram")
    p.add_argument("--pruned-radius", type=float, default=21.0,
                   help="pruned_928x928x464: fine triplets within this many degrees of a candidate's coarse "
                        "rotation are searched")
    p.add_argument("--unet-train", type=int, default=32,
                   help="learned_928x928x464: training tomograms (128^3 network inputs: 256^3 binned by 2 with "
                        "--unet-bin 2; the workload's species, SNR 0.05-0.2)")
    p.add_argument("--unet-steps", type=int, default=3000, help="learned_928x928x464: U-Net training steps")
    p.add_argument("--unet-bins", type=int, default=4,
                   help="learned_928x928x464: orientation bins (30 degree grid) refined per candidate")
    p.add_argument("--unet-lr", type=float, default=1e-3, help="learned_928x928x464: Adam learning rate")
    p.add_argument("--unet-pos-weight", type=float, default=300.0,
                   help="learned_928x928x464: weight of the centre target's positive voxels")
    p.add_argument("--unet-target-radius", type=float, default=3.0,
                   help="learned_928x928x464: radius of the centre target's balls")
    p.add_argument("--unet-edge", type=int, default=256, help="unet: the volume edge")
    p.add_argument("--rerank-step", type=int, default=28,
                   help="learned_928x928x464: coarse sub-grid step of the ranking comparison (degrees)")
    p.add_argument("--rerank-radius", type=float, default=28.0,
                   help="learned_928x928x464: fine triplets within this many degrees of a kept candidate's "
                        "coarse rotation")
    p.add_argument("--unet-bin", type=int, default=2, choices=[1, 2],
                   help="learned_928x928x464: run the network on the tomogram binned by this factor")
    p.add_argument("--unet-snr", default="0.05,0.2",
                   help="learned_928x928x464: SNR range of the training tomograms (lo,hi)")
    p.add_argument("--unet-window", type=int, default=7,
                   help="learned_928x928x464: refine window (+- voxels) around a candidate")
    p.add_argument("--pruned-window", type=int, default=2,
                   help="pruned_928x928x464: refine window (+- voxels) around a candidate (the crop is the FFT "
                        "length >= T + 2 window + 1: 64 for the 48^3 template up to window 7)")
    p.add_argument("--pruned-ref-out", default="", help="pruned_928x928x464: save the exhaustive peaks (.npz)")
    p.add_argument("--pruned-ref-in", default="", help="pruned_928x928x464: reuse saved exhaustive peaks")
    p.add_argument("--workload", default=WORKLOAD,
                   help="exhaustive_512x512x256 (the benchmark), profile_256x256x128 (profiler captures) or "
                        "align_2048 (batched subtomogram alignment, not the headline metric)")
    return p.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    INTERVAL_MS = 50

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []  # (host time, csv line)
        self.window = None

    def start(self):
        """Start sampling and return once the first sample has arrived (at
        most 5 s), so that the timed region that follows is covered."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.INTERVAL_MS)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        t_end = time.time() + 5.0
        while not self.lines and time.time() < t_end and self.proc.poll() is None:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, t0, t1):
        """Host-time window of the timed region (from before its first launch
        to after the synchronize that ends it)."""
        self.window = (t0, t1)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        # one more interval, so that a sample taken just before the window closed is read
        time.sleep(2 * self.INTERVAL_MS / 1e3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        lines = self.lines
        if self.window:
            inside = [x for x in lines if self.window[0] <= x[0] <= self.window[1]]
            # a timed region shorter than one interval keeps the samples nearest to it
            lines = inside or sorted(lines, key=lambda x: abs(x[0] - 0.5 * sum(self.window)))[:2]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, ln in lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "interval_ms": self.INTERVAL_MS}


def make_workload(name=WORKLOAD):
    from tom_b200 import synth
    cfg = synth.CONFIGS[name]
    grid = __import__("tom_b200").tom_av3_angle_grid(*cfg["angles"])
    d = synth.make_tomogram(cfg["N"], cfg["T"], cfg["n_copies"], cfg["n_blobs"], cfg["rho"], cfg["snr"],
                            cfg["max_tilt"], seed=2024, euler_pool=grid, mask_radius=cfg["mask_radius"])
    mask = synth.sphere_mask(cfg["T"], cfg["mask_radius"])
    return cfg, grid, d, mask


def chunk(grid, s, world, rank, rps):
    start = ((s * world + rank) * rps) % len(grid)
    idx = (start + np.arange(rps)) % len(grid)
    return grid[idx], start


def algorithmic_bytes(kind, cfg, nb):
    """Compulsory HBM bytes of one launch of a hot kernel class over a batch of nb rotations."""
    nx, ny, nz = cfg["N"]
    T = cfg["T"]
    nh1 = nx // 2 + 1
    half = 8 * nh1 * ny * nz  # one FP32 complex half spectrum
    nvox = nx * ny * nz
    if kind == "corr_y":
        return half + nb * (8 * nh1 * nz * T) + nb * half
    if kind == "inv_z":
        return 2 * nb * half
    if kind == "c2r_flcf":
        return nb * half + 8 * nvox + 8 * nvox + 8 * nvox
    if kind == "spec_z":
        return nb * 8 * nh1 * T * T + nb * 8 * nh1 * nz * T
    return 0


def cpu_baseline(d, mask, grid, seconds):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_baseline as CB
    cpu = CB.CpuFLCF(d["tomo"], d["template"], mask)
    t1 = cpu.run(grid[:1], 0)
    n = max(1, min(len(grid) - 1, int(seconds / max(t1, 1e-3))))
    tn = cpu.run(grid[1:1 + n], 1)
    nvox = int(np.prod(d["tomo"].shape))
    return {"value": n * nvox / tn, "unit": UNIT, "cores": cpu.workers,
            "kind": "reference" if cpu.use_ref else "port",
            "sample": f"{n} of {len(grid)} triplets on the full {'x'.join(map(str, d['tomo'].shape))} tomogram "
                      f"({tn:.1f} s; rotation by the "
                      f"reference's compiled rot3d, FP32 pocketfft rfftn/irfftn on {cpu.workers} threads, "
                      "numpy FLCF + max)"}


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    cfg, grid, d, mask = make_workload()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_baseline as CB
    cpu = CB.CpuFLCF(d["tomo"], d["template"], mask)
    nvox = int(np.prod(cfg["N"]))
    rps = 1
    for s in range(args.warmup):
        cpu.run(grid[s:s + rps], s)
    t = 0.0
    for s in range(args.steps):
        e, start = chunk(grid, args.warmup + s, 1, 0, rps)
        t += cpu.run(e, start)
    value = args.steps * rps * nvox / t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rot_per_step": rps, "angles": len(grid),
                       "tomogram": list(cfg["N"]), "template": cfg["T"]},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cpu.workers,
                             "kind": "reference" if cpu.use_ref else "port",
                             "sample": f"{args.steps} steps x {rps} triplet of the {len(grid)}-triplet grid"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_learned(args):
    """The learned proposer on a 256^3 tomogram (one 32^3 species, SNR 0.1,
    +-60 degree wedge): training throughput of the network's own kernels
    (FLOP/s of forward + backward), and the pruned search (coarse 30 degree
    search, proposals, fine search in the proposed bins around the proposals)
    against the exhaustive fine (15 degree) search: time and recall of the
    exhaustive search's top peaks, with the network's proposals and with the
    coarse map's own peaks as the candidates."""
    import torch
    import tom_b200 as tb
    from tom_b200 import proposer as pr
    from tom_b200 import synth
    world, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    ctx = tb.default_context(local)
    T = 32
    coarse = tb.tom_av3_angle_grid((0, 0, 0), (30, 30, 30), (330, 330, 180))
    fine = tb.tom_av3_angle_grid((0, 0, 0), (15, 15, 15), (345, 345, 180))
    members = pr.bin_members(fine, coarse)
    ph = synth.BlobPhantom(np.random.default_rng(5), 8, 12)
    mask = synth.sphere_mask(T, T // 2 - 1)

    def sample(N, n_copies, seed):
        d = synth.make_tomogram(N, T, n_copies, 8, 12, 0.1, 60, seed=seed, euler_pool=fine,
                                mask_radius=T // 2 - 1, phantom=ph)
        ccc, idc = pr.search(d["tomo"], d["template"], mask, coarse, ctx=ctx)
        return d, ccc, idc

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t0

    # training set: 128^3 tomograms labelled by the fine search
    net = pr.ProposerNet(len(coarse), ctx, seed=1)
    train = []
    for s in range(args.learned_train):
        d, ccc, idc = sample((128, 128, 128), 12, 500 + s)
        ccf, idf = pr.search(d["tomo"], d["template"], mask, fine, ctx=ctx)
        pos, bins, _ = pr.make_labels(ccf, idf, 12, T / 2, fine, coarse, ctx)
        train.append((ccc, pos, bins))
    N = (128, 128, 128)

    def step(i):
        ccc, pos, bins = train[i % len(train)]
        x = torch.from_numpy(np.ascontiguousarray(pr.normalise(tb.from_device(ccc).transpose(2, 1, 0)))).to(net.dev)
        return net.train_step(x, pr.heat_target(N, pos, net.dev), torch.from_numpy(pr.flat_index(pos, N)).to(net.dev),
                              torch.from_numpy(bins.astype(np.int32)).to(net.dev), pos_weight=200.0, lr=5e-4)

    for i in range(args.warmup):
        step(i)
    losses, t_train = timed(lambda: [step(i) for i in range(args.warmup, args.warmup + args.learned_steps)])
    train_flops = 3 * net.flops_per_voxel() * int(np.prod(N)) * args.learned_steps
    # test tomogram, 256^3
    NT = (256, 256, 256)
    d, ccc, idc = sample(NT, 60, 999)
    (ccf, idf), t_exh = timed(lambda: pr.search(d["tomo"], d["template"], mask, fine, batch=16, ctx=ctx))
    K = 60
    ref_vals, ref_pos, ref_idx = tb.pick_peaks(ccf, idf, K, T / 2, ctx)
    ref_pos = ref_pos - 1
    (ccc2, idc2), t_coarse = timed(lambda: pr.search(d["tomo"], d["template"], mask, coarse, batch=16, ctx=ctx))
    (cpos, _, cbins), t_prop = timed(lambda: pr.propose(net, ccc2, 2 * K, T / 2, 3, ctx))
    idc_h = tb.from_device(idc2)

    def refine_from(cands, extra_bins):
        sets = []
        for c, b in zip(cands, extra_bins):
            bs = set(int(x) for x in b) | {int(idc_h[c[0], c[1], c[2]])}
            ids = np.concatenate([members[k] for k in sorted(bs)])
            sets.append((fine[ids], ids))
        return pr.refine(d["tomo"], d["template"], mask, cands, sets, ctx=ctx)

    (rpos, rcc, ridx), t_ref = timed(lambda: refine_from(cpos, cbins))
    _, bpos, _ = tb.pick_peaks(ccc2, idc2, 2 * K, T / 2, ctx)
    bpos = bpos - 1
    (bres_pos, bcc, bidx), t_bref = timed(lambda: refine_from(bpos, [[]] * len(bpos)))

    def recall(pos, idx):
        dd = np.linalg.norm(ref_pos[:, None, :] - np.asarray(pos)[None].astype(float), axis=2)
        j = np.argmin(dd, axis=1)
        found = dd[np.arange(len(ref_pos)), j] <= 2
        same = np.asarray(idx)[j] == ref_idx
        return float(found.mean()), float((found & same).mean())

    rc, ra = recall(rpos, ridx)
    bc, ba = recall(bres_pos, bidx)
    # equal candidate counts with the fine triplets within 30 degrees of each
    # candidate's coarse rotation: the coarse map's own first peaks against the
    # network's ranking of the first 4 x that many coarse peaks
    cmp = {}
    for C in (K // 2, K, 2 * K):
        _, bp, bi = tb.pick_peaks(ccc2, idc2, C, T / 2, ctx)
        okb = bi >= 0
        bp, bi = bp[okb] - 1, bi[okb]
        npos, nidx, _ = pr.rerank(net, ccc2, idc2, C, 4 * C, T / 2, ctx)
        out = {}
        for name, cp_, ci_ in (("coarse_peaks", bp, bi), ("network_ranked", npos, nidx)):
            near = pr.neighbours(fine, coarse[ci_], 30.0)
            rp, _, ri = pr.refine(d["tomo"], d["template"], mask, cp_, [(fine[i], i) for i in near], ctx=ctx)
            pc, pa = recall(rp, ri)
            out[name] = {"position": pc, "position_and_angle": pa}
        cmp[str(C)] = out
    t_pruned = t_coarse + t_prop + t_ref
    line = {"metric": "learned-pruned search speed-up over the exhaustive fine search (256^3, 32^3 template)",
            "value": t_exh / t_pruned, "unit": "x", "higher_is_better": True, "n_gpus": 1,
            "steps": args.learned_steps, "warmup": args.warmup, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "learned_256", "tomogram": list(NT), "template": T, "coarse_angles": len(coarse),
                       "fine_angles": len(fine), "candidates": 2 * K, "reference_peaks": K,
                       "train_tomograms": args.learned_train, "train_volume": list(N)},
            "exhaustive_s": t_exh, "pruned_s": {"coarse": t_coarse, "network": t_prop, "refine": t_ref},
            "recall_network": {"position": rc, "position_and_angle": ra},
            "recall_coarse_peaks_without_network": {"position": bc, "position_and_angle": ba,
                                                    "pruned_s": t_coarse + t_bref},
            "recall_by_candidates_radius_30deg": cmp,
            "training": {"flop_per_s": train_flops / t_train, "s_per_step": t_train / args.learned_steps,
                         "last_loss": losses[-1]},
            "scaling": "weak", "vs_baseline": None}
    print(json.dumps(line), flush=True)


def run_pruned(args):
    """Pruned search on the full-size tomogram (928x928x464, one 48^3 species,
    the 7 degree grid of 70,304 triplets): a coarse search on a sub-grid (every
    --pruned-step degrees), its top candidates (tom_peak rounds with radius
    T/2), and the fine search around each candidate only (proposer.refine: a
    crop holding every voxel the FLCF there reads, the fine triplets within
    --pruned-radius degrees of the candidate's coarse rotation, the best CC
    within 2 voxels).  Against the exhaustive fine search: seconds and recall
    of its top-K peaks (K = the particle count), by position (within 2 voxels)
    and by position and triplet.  --pruned-ref-out / --pruned-ref-in save and
    reuse the exhaustive search's peaks (and its time) for the same seeded
    tomogram."""
    import torch
    import tom_b200 as tb
    from tom_b200 import proposer as pr
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    ctx = tb.default_context(local)
    name = "exhaustive_928x928x464"
    cfg, fine, d, mask = make_workload(name)
    T, K = cfg["T"], cfg["n_copies"]
    step = args.pruned_step
    fstart, finc, fend = cfg["angles"]
    if step % finc[0]:
        raise SystemExit("--pruned-step must be a multiple of the fine step (%d)" % finc[0])
    coarse = pr.coarse_grid(fstart, finc, fend, step // finc[0])

    def timed(fn):
        torch.cuda.synchronize()
        t = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t

    batch = args.batch or 32
    if args.pruned_ref_in:
        z = np.load(args.pruned_ref_in)
        ref_pos, ref_idx, ref_vals, t_exh = z["pos"], z["idx"], z["vals"], float(z["t_exh"])
    else:
        (ccf, idf), t_exh = timed(lambda: pr.search(d["tomo"], d["template"], mask, fine, batch=batch, ctx=ctx))
        ref_vals, ref_pos, ref_idx = tb.pick_peaks(ccf, idf, K, T / 2, ctx)
        ref_pos = ref_pos - 1
        del ccf, idf
        if args.pruned_ref_out:
            np.savez(args.pruned_ref_out, pos=ref_pos, idx=ref_idx, vals=ref_vals, t_exh=t_exh)
    torch.cuda.empty_cache()
    C = int(round(args.pruned_cands * K))
    tm = {}
    rpos, rcc, ridx = pr.pruned_search(d["tomo"], d["template"], mask, fine, coarse, C, args.pruned_radius,
                                       window=args.pruned_window, batch=batch, ctx=ctx, timings=tm)
    dd = np.linalg.norm(ref_pos[:, None, :].astype(float) - np.asarray(rpos)[None].astype(float), axis=2)
    j = np.argmin(dd, axis=1)
    found = dd[np.arange(len(ref_pos)), j] <= 2
    same = np.asarray(ridx)[j] == ref_idx
    t_pruned = tm["total"]
    line = {"metric": "pruned-search speed-up over the exhaustive fine search (928x928x464, 48^3 template)",
            "value": t_exh / t_pruned, "unit": "x", "higher_is_better": True, "n_gpus": 1,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "pruned_928x928x464", "fine_angles": len(fine), "coarse_angles": len(coarse),
                       "coarse_step_deg": step, "candidates": tm["candidates_n"], "reference_peaks": K,
                       "refine_radius_deg": args.pruned_radius, "refine_window": args.pruned_window,
                       "refine_triplets_per_candidate": tm["triplets_per_candidate"]},
            "exhaustive_s": t_exh,
            "pruned_s": {k: tm[k] for k in ("total", "coarse", "candidates", "triplet_sets", "refine")},
            "recall": {"position": float(found.mean()), "position_and_triplet": float((found & same).mean())},
            "scaling": "weak", "vs_baseline": None}
    print(json.dumps(line), flush=True)


def run_learned_928(args):
    """The learned-pruned search on the full-size tomogram (928x928x464, the
    48^3 species, 7 degree grid of 70,304 triplets).  The U-Net (BF16 on the
    tensor cores) is trained on --unet-train synthetic 128^3 tomograms of the
    same species (SNR drawn from 0.05-0.2, +-60 degree wedge) labelled by the
    search itself (the peaks of the exhaustive fine search and the 30 degree
    bins of their angles); on the test tomogram it proposes candidates and orientation
    bins, and the fine search runs only on crops around the candidates, over
    the fine triplets within --pruned-radius degrees of the --unet-bins most
    probable bins.  Against the exhaustive fine search: seconds and recall of
    its top-K peaks (K = the particle count), by position (within 2 voxels)
    and by position and triplet; the network's training FLOP/s and inference
    time; and the candidate recall of the network alone and of the coarse
    search's peaks at the same count."""
    import torch
    import tom_b200 as tb
    from tom_b200 import proposer as pr
    from tom_b200 import synth
    from tom_b200 import unet
    world, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    ctx = tb.default_context(local)
    name = "exhaustive_928x928x464"
    cfg, fine, d, mask = make_workload(name)
    T, K = cfg["T"], cfg["n_copies"]
    bins30 = tb.tom_av3_angle_grid((0, 0, 0), (30, 30, 30), (330, 330, 180))

    def timed(fn):
        torch.cuda.synchronize()
        t = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t

    # the workload's species (the first draw of make_tomogram's generator)
    ph = synth.BlobPhantom(np.random.default_rng(2024), cfg["n_blobs"], cfg["rho"])
    rng = np.random.default_rng(31)
    snr_lo, snr_hi = (float(x) for x in args.unet_snr.split(","))
    nb = args.unet_bin
    E = 128 * nb  # training tomograms: 128^3 network inputs
    # labels: the exhaustive fine search on unbinned training tomograms; the
    # exhaustive 30 degree search (peaks within 4 voxels, 2 after binning) on
    # the 8x larger binned ones
    (samples), t_data = timed(lambda: [
        unet.training_sample((E, E, E), T, 6 * nb ** 3, cfg["n_blobs"], cfg["rho"],
                             float(rng.uniform(snr_lo, snr_hi)), 60, 7000 + s, ph, mask, bins30,
                             fine if nb == 1 else None, ctx, binning=nb) for s in range(args.unet_train)])
    net = unet.UNetProposer(len(bins30), ctx, seed=1)
    kw = dict(lr=args.unet_lr, pos_weight=args.unet_pos_weight, target_radius=args.unet_target_radius)
    unet.train(net, samples, max(1, args.warmup), **kw)
    losses, t_train = timed(lambda: unet.train(net, samples, args.unet_steps, start=args.warmup, **kw))
    train_flops = 3 * net.flops_per_voxel() * 128 ** 3 * args.unet_steps
    # the network on a training tomogram: its own labels recalled (a check of
    # the pipeline's coordinate conventions and of what training reached)
    v0, p0, _ = samples[0]
    tpos, _, _ = unet.propose(net, v0, 2 * len(p0), T / 2 / nb, 1, border=16 // nb)
    td = np.linalg.norm(np.asarray(p0)[:, None, :].astype(float) - np.asarray(tpos)[None].astype(float), axis=2)
    train_recall = float((td.min(axis=1) <= 2).mean())
    del samples, v0
    torch.cuda.empty_cache()
    batch = args.batch or 32
    if args.pruned_ref_in:
        z = np.load(args.pruned_ref_in)
        ref_pos, ref_idx, t_exh = z["pos"], z["idx"], float(z["t_exh"])
    else:
        (ccf, idf), t_exh = timed(lambda: pr.search(d["tomo"], d["template"], mask, fine, batch=batch, ctx=ctx))
        ref_vals, ref_pos, ref_idx = tb.pick_peaks(ccf, idf, K, T / 2, ctx)
        ref_pos = ref_pos - 1
        del ccf, idf
        if args.pruned_ref_out:
            np.savez(args.pruned_ref_out, pos=ref_pos, idx=ref_idx, vals=ref_vals, t_exh=t_exh)
    torch.cuda.empty_cache()
    C = int(round(args.pruned_cands * K))
    tm = {}
    rpos, rcc, ridx = unet.learned_pruned_search(d["tomo"], d["template"], mask, fine, bins30, net, C,
                                                 args.unet_bins, args.pruned_radius, window=args.unet_window,
                                                 binning=nb, ctx=ctx, timings=tm)

    def recall(pos, idx=None):
        dd = np.linalg.norm(ref_pos[:, None, :].astype(float) - np.asarray(pos)[None].astype(float), axis=2)
        j = np.argmin(dd, axis=1)
        found = dd[np.arange(len(ref_pos)), j] <= 2
        if idx is None:
            return float(found.mean())
        return float(found.mean()), float((found & (np.asarray(idx)[j] == ref_idx)).mean())

    rc, ra = recall(rpos, ridx)
    # the network's candidates and bins alone, and the coarse 30 degree search's
    # peaks at the same count (positions; the nearest bin of the reference triplet)
    (cpos, _, cbins), t_prop = timed(lambda: unet.propose_host(net, d["tomo"], C, T / 2, args.unet_bins, nb))
    torch.cuda.empty_cache()
    ref_bin = pr.coarse_bin(np.asarray(fine)[ref_idx], bins30)
    dd = np.linalg.norm(ref_pos[:, None, :].astype(float) - np.asarray(cpos)[None].astype(float), axis=2)
    j = np.argmin(dd, axis=1)
    dmin = dd[np.arange(len(ref_pos)), j]
    near = dmin <= args.unet_window
    bin_hit = np.array([ref_bin[i] in set(cbins[j[i]]) for i in range(len(ref_pos))])
    net_by_radius = {str(r): float((dmin <= r).mean()) for r in (2, 4, 7, 12, 24)}
    (ccc, icc), t_c30 = timed(lambda: pr.search(d["tomo"], d["template"], mask, bins30, batch=batch, ctx=ctx))
    _, bpos, bidx = tb.pick_peaks(ccc, icc, C, T / 2, ctx)
    del ccc, icc
    okb = bidx >= 0
    bpos, bidx = bpos[okb] - 1, bidx[okb]
    dd = np.linalg.norm(ref_pos[:, None, :].astype(float) - bpos[None].astype(float), axis=2)
    jb = np.argmin(dd, axis=1)
    cmin = dd[np.arange(len(ref_pos)), jb]
    cnear = cmin <= args.unet_window
    coarse_by_radius = {str(r): float((cmin <= r).mean()) for r in (2, 4, 7, 12, 24)}
    cbin_hit = bidx[jb] == ref_bin
    # the network as a ranker of the coarse search's candidates: a coarse
    # sub-grid search, its --pruned-cands x K first peaks, and the fine search
    # (within --rerank-radius degrees of each candidate's coarse rotation, +-7
    # voxels) on the n best of them, ranked by the network (its centre
    # probability there) or, without the network, by their coarse CC
    fstart, finc, fend = cfg["angles"]
    cgrid = pr.coarse_grid(fstart, finc, fend, args.rerank_step // finc[0])
    (ccg, icg), t_cg = timed(lambda: pr.search(d["tomo"], d["template"], mask, cgrid, batch=batch, ctx=ctx))
    (pvals, ppos, pidx), t_pk = timed(lambda: tb.pick_peaks(ccg, icg, C, T / 2, ctx))
    del ccg, icg
    torch.cuda.empty_cache()
    okp = pidx >= 0
    ppos, pidx, pvals = ppos[okp] - 1, pidx[okp], pvals[okp]
    score, t_score = timed(lambda: unet.rerank_scores(net, d["tomo"], ppos, nb))
    near_sets = pr.neighbours(fine, np.asarray(cgrid)[pidx], args.rerank_radius)
    rerank = {}
    for n_keep in [int(round(f * K)) for f in (1.0, 1.1, 1.25, 1.5)]:
        out = {}
        for name, order in (("network_ranked", np.argsort(-score, kind="stable")),
                            ("coarse_cc_ranked", np.argsort(-pvals, kind="stable"))):
            keep = order[:n_keep]
            (rp, _, ri), t_ref = timed(lambda: pr.refine(d["tomo"], d["template"], mask, ppos[keep],
                                                         [(np.asarray(fine)[near_sets[i]], near_sets[i])
                                                          for i in keep], window=7, ctx=ctx))
            pc, pa = recall(rp, ri)
            out[name] = {"position": pc, "position_and_triplet": pa, "refine_s": t_ref,
                         "total_s": t_cg + t_pk + t_ref + (t_score if name == "network_ranked" else 0.0)}
        rerank[str(n_keep)] = out
    line = {"metric": "learned-pruned search speed-up over the exhaustive fine search (928x928x464, 48^3 template)",
            "value": t_exh / tm["total"], "unit": "x", "higher_is_better": True, "n_gpus": 1,
            "dtype": "bf16 network, f32 search", "data": "synthetic",
            "config": {"workload": "learned_928x928x464", "fine_angles": len(fine), "bins": len(bins30),
                       "candidates": tm["candidates_n"], "reference_peaks": K, "bins_per_candidate": args.unet_bins,
                       "refine_radius_deg": args.pruned_radius, "refine_window": args.unet_window,
                       "refine_triplets_per_candidate": tm["triplets_per_candidate"],
                       "train_tomograms": args.unet_train, "train_volume": [E, E, E], "binning": nb,
                       "pos_weight": args.unet_pos_weight, "target_radius": args.unet_target_radius,
                       "train_snr": [snr_lo, snr_hi],
                       "train_steps": args.unet_steps},
            "exhaustive_s": t_exh, "pruned_s": {k: tm[k] for k in ("total", "network", "triplet_sets", "refine")},
            "recall": {"position": rc, "position_and_triplet": ra},
            "network_alone": {"candidate_recall_within_window": float(near.mean()),
                              "candidate_recall_by_radius": net_by_radius,
                              "bin_in_top_bins": float((near & bin_hit).mean()), "propose_s": t_prop,
                              "training_tomogram_label_recall": train_recall},
            "rerank": {"coarse_step_deg": args.rerank_step, "coarse_angles": len(cgrid),
                       "pool": int(len(ppos)), "radius_deg": args.rerank_radius, "coarse_search_s": t_cg,
                       "peaks_s": t_pk, "network_s": t_score, "by_kept_candidates": rerank},
            "coarse_30deg_search_alone": {"candidate_recall_within_window": float(cnear.mean()),
                                          "candidate_recall_by_radius": coarse_by_radius,
                                          "bin_hit": float((cnear & cbin_hit).mean()), "search_s": t_c30},
            "training": {"flop_per_s": train_flops / t_train, "s_per_step": t_train / args.unet_steps,
                         "first_loss": losses[0], "last_loss": losses[-1], "data_s": t_data},
            "scaling": "weak", "vs_baseline": None}
    print(json.dumps(line), flush=True)


def run_unet(args):
    """The U-Net proposer's own kernels on a --unet-edge^3 volume: the forward
    pass (inference) and one training step (forward, backward, Adam, weight
    repacking), each timed with CUDA events over --steps iterations after
    --warmup; FLOP/s by the network's multiply-adds (forward 2 MAC per voxel,
    a training step 3x the forward), against the measured dense BF16 peak."""
    import torch
    import tom_b200 as tb
    from tom_b200 import unet
    world, rank, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    ctx = tb.default_context(local)
    n = args.unet_edge
    net = unet.UNetProposer(1008, ctx, seed=1)
    g = torch.Generator(device=net.dev).manual_seed(3)
    vol = torch.randn((n, n, n), device=net.dev, generator=g)
    tgt = (torch.rand((n, n, n), device=net.dev, generator=g) < 1e-4).float()
    idx = torch.randperm(n ** 3, device=net.dev, generator=g)[:64].contiguous()
    bins = torch.randint(0, 1008, (64,), device=net.dev, dtype=torch.int32, generator=g)
    st = torch.cuda.current_stream()

    def ev_time(fn, k):
        for _ in range(args.warmup):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(k):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    l0 = ctx.launches
    fwd_ms = ev_time(lambda: net.forward(vol, prob=True), args.steps)
    step_ms = ev_time(lambda: net.train_step(vol, tgt, idx, bins), args.steps)
    fl = net.flops_per_voxel() * n ** 3
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 1590.0, "fallback"
    if os.path.exists(path):
        with open(path) as f:
            peak, peak_src = float(json.load(f)["bf16_tflops"]), "measured"
    line = {"metric": "U-Net proposer TFLOP/s (BF16 tcgen05 3x3x3 convolutions, FP32 accumulation)",
            "value": fl / fwd_ms / 1e9, "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": "unet_%d" % n, "volume": [n, n, n], "channels": [16, 32, 64]},
            "forward_ms": fwd_ms, "train_step_ms": step_ms, "train_tflops": 3 * fl / step_ms / 1e9,
            "flop_per_voxel_forward": net.flops_per_voxel(),
            "roofline": {"bound": "tensor", "achieved": fl / fwd_ms / 1e9, "peak": peak, "unit": "TFLOP/s",
                         "frac": fl / fwd_ms / 1e9 / peak, "peak_source": peak_src},
            "gpu_launches": (ctx.launches - l0) // (2 * (args.warmup + args.steps)),
            "scaling": "weak", "vs_baseline": None}
    print(json.dumps(line), flush=True)


def run_align(args):
    """Batched uneven subtomogram alignment (2048 particles, edges 32-96, +-15 deg
    at 3 deg = 1331 triplets each, shifts <= 4): a stratified subset is timed and
    the full workload extrapolated by box size."""
    import torch
    import tom_b200 as tb
    from tom_b200 import synth
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    jobs, truth = synth.make_align_particles(args.align_particles, seed=77)
    ctx = tb.default_context(local)
    # warm-up: one particle of every box size (twiddle tables, first launches)
    first = {}
    for j in jobs:
        first.setdefault(j["ref"].shape, j)
    tb.av3_align_batch(list(first.values()), ctx, path=args.align_path, batch_bytes=args.align_batch_mb << 20)
    torch.cuda.synchronize()

    reps = 1 if len(jobs) > 200 else 3

    def timed(sub):
        """median and minimum wall time of `reps` calls on sub (all on the device at the end)"""
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t = time.perf_counter()
            out = tb.av3_align_batch(sub, ctx, path=args.align_path, batch_bytes=args.align_batch_mb << 20,
                                     timings=split)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t)
        return float(np.median(ts)), float(min(ts)), out

    split = {}

    l0 = ctx.launches
    clocks = ClockSampler(local)
    clocks.start()
    h0 = time.time()
    dt, dt_min, (angles, shifts, peaks) = timed(jobs)
    clocks.mark(h0, time.time())
    clk = clocks.stop()
    launches = (ctx.launches - l0) // reps
    split_all = dict(split)  # the last call on the whole batch: uploads and library call
    ok = [np.allclose(a, t[0]) for a, t in zip(angles, truth)]
    vox = [int(np.prod(j["ref"].shape)) for j in jobs]
    rv = 1331 * sum(vox)
    per_size = {}
    for j, v in zip(jobs, vox):
        per_size.setdefault(j["ref"].shape[0], 0)
        per_size[j["ref"].shape[0]] += 1
    # each box edge on its own: seconds per particle, and the 2048-particle
    # workload (edges drawn uniformly from the five) from them
    per_size_s = {}
    if len(jobs) <= 200:
        for n in sorted(per_size):
            sub = [j for j in jobs if j["ref"].shape[0] == n]
            per_size_s[n] = timed(sub)[0] / len(sub)
    sizes = (32, 48, 64, 80, 96)
    if len(jobs) == 2048:
        est_full = dt  # the whole workload, measured
    elif all(n in per_size_s for n in sizes):
        est_full = 2048 / len(sizes) * sum(per_size_s[n] for n in sizes)
    else:
        est_full = dt / sum(vox) * 2048 * np.mean([s ** 3 for s in sizes])
    # flops by the survey's count for this config: (5 log2 n^3 + 20) per rot*voxel
    flops = 1331 * sum(v * (5 * np.log2(v) + 20) for v in vox)
    line = {"metric": "subtomogram alignment rot*voxel/s (tom_av3_align, 1331 triplets per particle)",
            "flop_per_s": flops / dt,
            "flop_note": "(5 log2 n^3 + 20) flop per rot*voxel; FP32 CUDA-core nominal peak "
                         "148 SMs x 128 lanes x 2 x 1.965 GHz = 74.4 TFLOP/s",
            "value": rv / dt, "unit": "rot*voxel/s", "n_gpus": 1, "particles": len(jobs), "seconds": dt, "seconds_min": dt_min,
            "upload_s": split_all.get("upload_s"), "call_s": split_all.get("call_s"),
            "particles_per_s": len(jobs) / dt, "est_seconds_2048": est_full,
            "planted_angle_agreement": float(np.mean(ok)),
            "planted_angle_note": "fraction of particles whose scan maximum is the planted Euler triplet; "
                                  "not a pass mark: tom_av3_align's own objective (the FP64 oracle) also "
                                  "peaks at other grid triplets for noiseless 6-blob wedged phantoms",
            "per_size": per_size, "seconds_per_particle": per_size_s, "gpu_launches": launches,
            "align_path": args.align_path, "align_batch_mb": args.align_batch_mb, "clocks": clk,
            "dtype": "f32", "data": "synthetic"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "align_2048":
        return run_align(args)
    if args.workload == "pruned_928x928x464":
        return run_pruned(args)
    if args.workload == "learned_928x928x464":
        return run_learned_928(args)
    if args.workload == "unet":
        return run_unet(args)
    if args.workload == "learned_256":
        return run_learned(args)
    import torch
    import tom_b200 as tb
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    cfg, grid, d, mask = make_workload(args.workload)
    nvox = int(np.prod(cfg["N"]))
    ctx = tb.default_context(local)
    plan = tb.MatchPlan(cfg["N"], (cfg["T"],) * 3, batch=args.batch, ctx=ctx, path=args.path)
    plan.set_template(tb.to_device(d["template"], local), tb.to_device(mask, local))
    vol_dev = tb.to_device(d["tomo"], local)
    plan.set_volume(vol_dev)
    tune = None
    if args.batch == 0:
        e, _ = chunk(grid, 0, world, rank, 64)
        best, tune = plan.autotune(e, (8, 16, 32, 64))
        if dist:  # every rank runs the same batch: the smallest of the ranks' choices
            t = torch.tensor([best], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MIN)
            if int(t.item()) != best:
                best, _ = plan.autotune(e, (int(t.item()),))
        args.batch = best
    cc, idx = plan.new_results()
    # a step is a whole number of rotation batches, so every launch is full
    rps = -(-args.rot_per_step // args.batch) * args.batch

    def step(s):
        e, start = chunk(grid, s, world, rank, rps)
        plan.run(e, cc, idx, index_offset=start)

    for s in range(args.warmup):
        step(s)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ctx.profile(True)
    l0 = ctx.launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0 = time.time()
    ev0.record()
    for s in range(args.warmup, args.warmup + args.steps):
        step(s)
    ev1.record()
    torch.cuda.synchronize()
    clocks.mark(h0, time.time())
    ms = ev0.elapsed_time(ev1)
    launches = ctx.launches - l0
    kt = ctx.kernel_times()
    ctx.profile(False)
    clk = clocks.stop()
    if dist:
        dist.barrier()
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    units = args.steps * rps * nvox * world
    value = units / (ms / 1e3)

    # roofline of the dominant kernel class
    peak, peak_src = measured_peaks()
    dom = max(kt, key=lambda k: kt[k][0])
    dms, dn = kt[dom]
    avg_s = dms / max(dn, 1) / 1e3
    nb = args.batch
    ab = algorithmic_bytes(dom, cfg, nb)
    achieved = ab / avg_s / 1e9 if avg_s > 0 else 0.0
    traffic = TRAFFIC.get(args.workload, {}).get(dom, {}).get(args.batch)
    shares = {k: round(v[0] / max(sum(x[0] for x in kt.values()), 1e-9), 4) for k, v in kt.items()}
    # the same figure for every kernel class with algorithmic bytes
    rooflines = {}
    for kind, (kms, kn) in kt.items():
        kb = algorithmic_bytes(kind, cfg, nb)
        if kb and kn:
            ks = kms / kn / 1e3
            rooflines[kind] = {"avg_launch_ms": ks * 1e3, "achieved": kb / ks / 1e9, "frac": kb / ks / 1e9 / peak,
                               "traffic": TRAFFIC.get(args.workload, {}).get(kind, {}).get(args.batch)}

    # accuracy: top-K peaks of the max-CC map rescored in FP64 by direct sums
    rescore = None
    if args.rescore_k is None:
        args.rescore_k = 1000 if args.workload == "exhaustive_928x928x464" else 200
    if args.rescore_k > 0 and rank == 0:
        K = args.rescore_k
        vals, pos, aidx = tb.pick_peaks(cc, idx, K, cfg["T"] / 2, ctx)
        ok = aidx >= 0
        fp64 = plan.rescore_fp64(vol_dev, grid[aidx[ok]], pos[ok])
        err = np.abs(vals[ok].astype(np.float64) - fp64)
        rescore = {"k": int(ok.sum()), "max_abs_err": float(err.max()), "max_cc": float(np.abs(fp64).max()),
                   "max_rel_err": float(err.max() / np.abs(fp64).max()),
                   "note": "FP32 spectral max-CC at the top-K peaks vs FP64 direct-sum FLCF at the same angle"}

    # the device-resident plan is done: its batch buffers (up to ~100 GB at
    # 928^2 x 464) are released before the end-to-end call builds its own
    plan.close()
    del cc, idx, vol_dev
    torch.cuda.empty_cache()

    # end to end through the one-shot C-ABI call with pinned host buffers
    e2e = None
    if not args.no_e2e:
        pin = lambda shape, dt: torch.empty(int(np.prod(shape)), dtype=dt, pin_memory=True).numpy().reshape(
            shape, order="F")
        tomo_h = pin(cfg["N"], torch.float32)
        tomo_h[...] = d["tomo"]
        cc_h = pin(cfg["N"], torch.float32)
        idx_h = pin(cfg["N"], torch.int32)
        ectx = tb.Context(local)
        tb.match_host(tomo_h, d["template"], mask, grid[:8], batch=args.batch, ctx=ectx)  # warm-up
        if args.e2e_rot <= 0:
            # the whole grid, split across the ranks (angle partitioning)
            args.e2e_rot = -(-len(grid) // world) if len(grid) <= 25000 else 2048
        if args.e2e_steps <= 0:
            args.e2e_steps = 1 if args.e2e_rot * world >= len(grid) else 3
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for s in range(args.e2e_steps):
            e, _ = chunk(grid, s, world, rank, args.e2e_rot)
            from tom_b200 import _lib
            vol = tomo_h
            prm = _lib.MatchParams()
            prm.batch = args.batch
            prm.path = args.path
            ectx.check(_lib.lib().tomgpu_match(
                ectx.handle, vol.ctypes.data, tb.tom._cdims(cfg["N"]), d["template"].ctypes.data,
                tb.tom._cdims((cfg["T"],) * 3), mask.ctypes.data, None,
                np.ascontiguousarray(e, np.float32).ctypes.data_as(_lib.c_float_p), len(e),
                ctypes.byref(prm), cc_h.ctypes.data, idx_h.ctypes.data))
        te = time.perf_counter() - t0
        if dist:
            t = torch.tensor([te], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            te = float(t.item())
        tb_bytes = 4 * cfg["T"] ** 3
        e2e = {"value": args.e2e_steps * args.e2e_rot * nvox * world / te, "unit": UNIT,
               "h2d_bytes_per_step": 4 * nvox + 2 * tb_bytes + 12 * args.e2e_rot,
               "d2h_bytes_per_step": 8 * nvox,
               "rot_per_step": args.e2e_rot, "steps": args.e2e_steps}
        ectx.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(d, mask, grid, args.cpu_seconds)

    if rank == 0:
        metric = METRIC
        if args.workload != WORKLOAD:
            metric = "TM rot*voxel/s (exhaustive FLCF, %s tomogram, %d^3 template)" % (
                "x".join(str(v) for v in cfg["N"]), cfg["T"])
        line = {"metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": args.workload, "tomogram": list(cfg["N"]), "template": cfg["T"],
                           "angles": len(grid), "rot_per_step": rps, "rotation_batch": args.batch,
                           "kernel_path": args.path,
                           "batch_autotune_ms_per_rotation": tune,
                           "parallelism": f"angle-partitioned x{world}",
                           "l2": "inputs larger than L2 (tomogram spectrum %d MB, per-batch spectra %.1f GB)" % (
                               8 * (cfg["N"][0] // 2 + 1) * cfg["N"][1] * cfg["N"][2] // 10**6,
                               8 * (cfg["N"][0] // 2 + 1) * cfg["N"][1] * cfg["N"][2] * args.batch / 1e9)},
                "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                             "algorithmic_bytes_per_launch": ab, "avg_launch_ms": avg_s * 1e3},
                "kernel_share": shares, "rooflines": rooflines, "fp64_rescore": rescore,
                "seconds_per_search": {"device": len(grid) * nvox * world / value,
                                       "e2e": len(grid) * nvox * world / e2e["value"] if e2e else None,
                                       "note": "the whole angle grid at this rate, one template"},
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clk}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
