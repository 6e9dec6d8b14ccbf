"""Learned candidate proposer for the template search (no counterpart in TOM).

A small dilated 3-D convolutional network reads the max-CC map of a coarse
exhaustive search (the 30 degree grid) and proposes (1) candidate particle
centres and (2) coarse orientation bins; the fine angular search then runs
only in those bins, only around those centres.  The network is trained on
labels the search itself produces on synthetic tomograms: the peaks of the
fine exhaustive search (positions) and the coarse bin of their fine angle.

Every layer runs on the library's own kernels through the C ABI
(tomgpu_cnn_*: dilated 3x3x3 convolution forward / input gradient / weight
gradient, dense layers, ReLU, losses, Adam); torch only holds the buffers.

Network (receptive field 33 voxels): five 3x3x3 convolutions with ReLU,
channels 1-16-16-32-32-32, dilations 1, 2, 4, 8, 1; a dense centre head
32 -> 1 at every voxel (binary cross-entropy against the label heat map) and
a dense orientation head 32 -> n_bins at labelled centres (softmax
cross-entropy).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .tom import Context, MatchPlan, _cdims, _tptr, default_context, from_device, pick_peaks, to_device

LAYERS = ((1, 16, 1), (16, 16, 2), (16, 32, 4), (32, 32, 8), (32, 32, 1))
FEAT = LAYERS[-1][1]


def _lib_call(ctx, name, *args):
    ctx.check(getattr(_lib.lib(), name)(ctx.handle, *args))


class ProposerNet:
    """Parameters, Adam state and the forward / backward passes."""

    def __init__(self, n_bins: int, ctx: Context | None = None, seed: int = 0):
        import torch
        self.ctx = ctx or default_context()
        self.dev = f"cuda:{self.ctx.device}"
        self.n_bins = int(n_bins)
        g = torch.Generator().manual_seed(seed)
        self.params = []
        for ci, co, _ in LAYERS:
            std = np.sqrt(2.0 / (27 * ci))
            self.params.append((torch.randn((co, ci, 27), generator=g) * std).to(self.dev))
            self.params.append(torch.zeros(co).to(self.dev))
        self.params.append((torch.randn((1, FEAT), generator=g) * np.sqrt(1.0 / FEAT)).to(self.dev))
        self.params.append(torch.full((1,), -4.0).to(self.dev))  # rare positives: start near p = 0.02
        self.params.append((torch.randn((self.n_bins, FEAT), generator=g) * np.sqrt(1.0 / FEAT)).to(self.dev))
        self.params.append(torch.zeros(self.n_bins).to(self.dev))
        self.params = [p.contiguous() for p in self.params]
        self.grads = [torch.zeros_like(p) for p in self.params]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.step_count = 0

    # -------------------------------------------------------------- forward
    def forward(self, x):
        """x: torch [Z][Y][X] float on the device -> (activations, centre logits [Z][Y][X])."""
        import torch
        Z, Y, X = x.shape
        dims = _cdims((X, Y, Z))
        acts = [x.reshape(1, Z, Y, X).contiguous()]
        for li, (ci, co, dil) in enumerate(LAYERS):
            out = torch.empty((co, Z, Y, X), device=self.dev)
            _lib_call(self.ctx, "tomgpu_cnn_conv3d_fwd_dev", _tptr(acts[-1]), ci, dims, _tptr(self.params[2 * li]),
                      _tptr(self.params[2 * li + 1]), co, dil, 1, _tptr(out))
            acts.append(out)
        nv = X * Y * Z
        logit = torch.empty((1, Z, Y, X), device=self.dev)
        Wc, bc = self.params[2 * len(LAYERS)], self.params[2 * len(LAYERS) + 1]
        _lib_call(self.ctx, "tomgpu_cnn_dense_fwd_dev", _tptr(Wc), _tptr(bc), _tptr(acts[-1]), 1, FEAT, nv, 0,
                  _tptr(logit))
        return acts, logit[0]

    def orient_logits(self, feat, idx):
        """Orientation logits [n_bins][P] at the flat voxel indices idx (torch int64)."""
        import torch
        C, Z, Y, X = feat.shape
        P = int(idx.numel())
        fg = torch.empty((C, P), device=self.dev)
        _lib_call(self.ctx, "tomgpu_cnn_gather_dev", _tptr(feat), C, X * Y * Z, _tptr(idx), P, _tptr(fg))
        out = torch.empty((self.n_bins, P), device=self.dev)
        Wo, bo = self.params[-2], self.params[-1]
        _lib_call(self.ctx, "tomgpu_cnn_dense_fwd_dev", _tptr(Wo), _tptr(bo), _tptr(fg), self.n_bins, C, P, 0,
                  _tptr(out))
        return fg, out

    # -------------------------------------------------------------- training
    def train_step(self, x, target, pos_idx, pos_bins, pos_weight=50.0, lr=1e-3, w_orient=0.2):
        """One Adam step on one sample.  x, target: [Z][Y][X]; pos_idx: flat
        indices of the labelled centres (int64), pos_bins: their coarse bins
        (int32).  Returns (centre loss, orientation loss)."""
        import torch
        ctx = self.ctx
        Z, Y, X = x.shape
        nv = X * Y * Z
        dims = _cdims((X, Y, Z))
        for g in self.grads:
            g.zero_()
        acts, logit = self.forward(x)
        loss = torch.zeros(2, dtype=torch.float64, device=self.dev)
        g_logit = torch.empty((1, Z, Y, X), device=self.dev)
        _lib_call(ctx, "tomgpu_cnn_bce_dev", _tptr(logit), _tptr(target), nv, float(pos_weight), _tptr(g_logit),
                  _tptr(loss[0:1]))
        L = len(LAYERS)
        feat = acts[-1]
        g_feat = torch.empty_like(feat)
        _lib_call(ctx, "tomgpu_cnn_dense_bwd_dev", _tptr(self.params[2 * L]), _tptr(feat), _tptr(g_logit), 1, FEAT, nv,
                  _tptr(g_feat), _tptr(self.grads[2 * L]), _tptr(self.grads[2 * L + 1]))
        P = int(pos_idx.numel())
        if P > 0 and w_orient > 0:
            fg, ol = self.orient_logits(feat, pos_idx)
            g_ol = torch.empty_like(ol)
            _lib_call(ctx, "tomgpu_cnn_softmax_ce_dev", _tptr(ol), _tptr(pos_bins), self.n_bins, P, _tptr(g_ol),
                      _tptr(loss[1:2]))
            g_ol.mul_(w_orient)
            g_fg = torch.empty_like(fg)
            _lib_call(ctx, "tomgpu_cnn_dense_bwd_dev", _tptr(self.params[-2]), _tptr(fg), _tptr(g_ol), self.n_bins,
                      FEAT, P, _tptr(g_fg), _tptr(self.grads[-2]), _tptr(self.grads[-1]))
            _lib_call(ctx, "tomgpu_cnn_scatter_add_dev", _tptr(g_fg), FEAT, nv, _tptr(pos_idx), P, _tptr(g_feat))
        g = g_feat
        for li in range(L - 1, -1, -1):
            ci, co, dil = LAYERS[li]
            _lib_call(ctx, "tomgpu_cnn_relu_bwd_dev", _tptr(g), _tptr(acts[li + 1]), co * nv)
            _lib_call(ctx, "tomgpu_cnn_conv3d_bwd_weight_dev", _tptr(acts[li]), ci, dims, _tptr(g), co, dil,
                      _tptr(self.grads[2 * li]), _tptr(self.grads[2 * li + 1]))
            if li > 0:
                gin = torch.empty_like(acts[li])
                _lib_call(ctx, "tomgpu_cnn_conv3d_bwd_data_dev", _tptr(g), co, dims, _tptr(self.params[2 * li]), ci,
                          dil, _tptr(gin))
                g = gin
        self.step_count += 1
        for p, gr, m, v in zip(self.params, self.grads, self.m, self.v):
            _lib_call(ctx, "tomgpu_cnn_adam_dev", _tptr(p), _tptr(gr), _tptr(m), _tptr(v), p.numel(), float(lr),
                      0.9, 0.999, 1e-8, self.step_count)
        out = loss.cpu().numpy()
        return float(out[0]), float(out[1])

    def flops_per_voxel(self):
        """Multiply-adds x 2 of one forward pass per voxel (convolutions and the centre head)."""
        return 2 * (sum(27 * ci * co for ci, co, _ in LAYERS) + FEAT)


# ------------------------------------------------------------------ data

def normalise(a):
    a = np.asarray(a, np.float32)
    s = float(a.std())
    return (a - float(a.mean())) / (s if s > 0 else 1.0)


def coarse_bin(eulers_fine, coarse_grid):
    """Index in the coarse grid (tom_av3_angle_grid order) of the nearest coarse
    rotation to each fine Euler triplet (geodesic distance of the rotations)."""
    from .tom import euler_matrix
    Rc = np.stack([np.asarray(euler_matrix(e), np.float64).reshape(3, 3) for e in coarse_grid])
    out = []
    for e in np.asarray(eulers_fine).reshape(-1, 3):
        R = np.asarray(euler_matrix(e), np.float64).reshape(3, 3)
        tr = np.einsum("kij,ij->k", Rc, R)  # trace(Rc^T R)
        out.append(int(np.argmax(tr)))
    return np.array(out, np.int32)


def search(vol, template, mask, angles, batch=8, ctx=None):
    """Exhaustive FLCF search (the library's fast path) -> (maxcc, angle index) device tensors."""
    ctx = ctx or default_context()
    plan = MatchPlan(np.shape(vol), np.shape(template), batch=batch, ctx=ctx)
    plan.set_template(to_device(template, ctx.device), to_device(mask, ctx.device))
    plan.set_volume(to_device(vol, ctx.device))
    cc, idx = plan.new_results()
    plan.run(angles, cc, idx)
    plan.close()
    return cc, idx


def make_labels(cc_fine, idx_fine, n_peaks, radius, fine_grid, coarse_grid, ctx=None):
    """Label positions (0-based [x, y, z]) and coarse bins from the fine search."""
    vals, pos, aidx = pick_peaks(cc_fine, idx_fine, n_peaks, radius, ctx)
    ok = aidx >= 0
    pos = pos[ok] - 1
    bins = coarse_bin(np.asarray(fine_grid)[aidx[ok]], coarse_grid)
    return pos, bins, vals[ok]


def heat_target(shape_xyz, pos, dev):
    """1 at the label voxels and their 6 neighbours, 0 elsewhere; torch [Z][Y][X]."""
    import torch
    X, Y, Z = shape_xyz
    t = np.zeros((Z, Y, X), np.float32)
    for x, y, z in pos:
        for dx, dy, dz in ((0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
            t[(z + dz) % Z, (y + dy) % Y, (x + dx) % X] = 1.0
    return torch.from_numpy(t).to(dev)


def flat_index(pos, shape_xyz):
    X, Y, Z = shape_xyz
    p = np.asarray(pos, np.int64).reshape(-1, 3)
    return p[:, 0] + X * (p[:, 1] + Y * p[:, 2])


# ------------------------------------------------------------------ pruned search

def propose(net, cc_coarse, n_cand, radius, top_bins, ctx=None):
    """Candidates of the network from a coarse max-CC map: positions (0-based
    [x, y, z]), heat values and the top_bins orientation bins per candidate."""
    import torch
    ctx = ctx or net.ctx
    x = torch.from_numpy(np.ascontiguousarray(normalise(from_device(cc_coarse).transpose(2, 1, 0)))).to(net.dev)
    acts, logit = net.forward(x)
    Z, Y, X = logit.shape
    idx_dummy = torch.zeros((Z, Y, X), dtype=torch.int32, device=net.dev)
    # probabilities (>= 0), so the zeroed balls of the peak picking stay below every candidate
    vals, pos, _ = pick_peaks(torch.sigmoid(logit).contiguous(), idx_dummy, n_cand, radius, ctx)
    pos = pos - 1
    fi = torch.from_numpy(flat_index(pos, (X, Y, Z))).to(net.dev)
    _, ol = net.orient_logits(acts[-1], fi)
    bins = torch.topk(ol, k=min(top_bins, net.n_bins), dim=0).indices.t().cpu().numpy()
    return pos, vals, bins


def coarse_grid(fine_start, fine_incr, fine_end, factor):
    """The sub-grid of every factor-th step of a tom_av3_angle_grid (start,
    incr, end): the coarse grid of a pruned search."""
    from .tom import tom_av3_angle_grid
    inc = [i * factor for i in fine_incr]
    end = [s + ((e - s) // c) * c for s, c, e in zip(fine_start, inc, fine_end)]
    return tom_av3_angle_grid(fine_start, inc, end)


def pruned_search(vol, template, mask, fine, coarse, n_cand, radius_deg, window=2, peak_radius=None, batch=32,
                  ctx=None, timings=None):
    """A pruned FLCF search: the exhaustive search over the coarse grid, its
    n_cand first peaks (tom_peak rounds of radius peak_radius, default half
    the template edge), and around each the fine triplets within radius_deg
    (geodesic) of its coarse rotation searched on a crop (refine: the values
    equal the full search's there), the best within +-window voxels.
    timings: an optional dict that receives the seconds of the steps.
    Returns (positions 0-based [x, y, z], cc, fine triplet index) per candidate."""
    import time
    import torch
    ctx = ctx or default_context()
    T = np.shape(template)[0]
    clock = []

    def mark():
        torch.cuda.synchronize(ctx.device)
        clock.append(time.perf_counter())

    mark()
    cc, idx = search(vol, template, mask, coarse, batch=batch, ctx=ctx)
    mark()
    _, pos, cidx = pick_peaks(cc, idx, n_cand, T / 2 if peak_radius is None else peak_radius, ctx)
    del cc, idx
    ok = cidx >= 0
    pos, cidx = pos[ok] - 1, cidx[ok]
    mark()
    near = neighbours(fine, np.asarray(coarse)[cidx], radius_deg)
    mark()
    out = refine(vol, template, mask, pos, [(np.asarray(fine)[i], i) for i in near], window=window, ctx=ctx)
    mark()
    if timings is not None:
        for k, name in enumerate(("coarse", "candidates", "triplet_sets", "refine")):
            timings[name] = clock[k + 1] - clock[k]
        timings["total"] = clock[-1] - clock[0]
        timings["candidates_n"] = int(len(pos))
        timings["triplets_per_candidate"] = float(np.mean([len(x) for x in near])) if near else 0.0
    return out


def rerank(net, cc_coarse, idx_coarse, n_cand, n_pool, radius, ctx=None):
    """Candidates of the coarse map re-ranked by the network: the n_pool first
    coarse peaks (tom_peak rounds of radius `radius`), each scored by the
    network's centre probability at its voxel, the n_cand best kept.
    Returns (positions 0-based [x, y, z], coarse angle index, score)."""
    import torch
    ctx = ctx or net.ctx
    x = torch.from_numpy(np.ascontiguousarray(normalise(from_device(cc_coarse).transpose(2, 1, 0)))).to(net.dev)
    _, logit = net.forward(x)
    heat = torch.sigmoid(logit)
    _, pos, aidx = pick_peaks(cc_coarse, idx_coarse, n_pool, radius, ctx)
    ok = aidx >= 0
    pos, aidx = pos[ok] - 1, aidx[ok]
    p = torch.as_tensor(pos, device=net.dev)
    score = heat[p[:, 2], p[:, 1], p[:, 0]].cpu().numpy()
    order = np.argsort(-score, kind="stable")[:n_cand]
    return pos[order], aidx[order], score[order]


def refine(vol, template, mask, centres, angle_sets, window=2, batch=8, ctx=None):
    """The fine search around each centre only: the FLCF on a periodic crop of
    edge L >= T + 2 window + 1 (an FFT length), with the centre's own angle
    list; the best CC within +-window voxels of the centre.  The crop holds
    every voxel the FLCF at those positions reads, so the values equal the
    full-volume search's there.  The tomogram stays on the device; crops,
    results and the window maxima are device tensors on the context's stream
    (one result buffer pair for all centres), read back once at the end.
    Returns (positions, cc, fine angle index)."""
    import torch
    ctx = ctx or default_context()
    dev = f"cuda:{ctx.device}"
    vol = np.asarray(vol, np.float32)
    shape = vol.shape
    T = np.shape(template)[0]
    need = T + 2 * window + 1
    L = next(n for n in (16, 24, 32, 40, 48, 64, 80, 96, 128) if n >= need)
    half = L // 2
    centres = np.asarray(centres, np.int64).reshape(-1, 3)
    n = len(centres)
    plan = MatchPlan((L, L, L), np.shape(template), batch=batch, ctx=ctx)
    try:
        plan.set_template(to_device(template, ctx.device), to_device(mask, ctx.device))
        vt = torch.from_numpy(np.ascontiguousarray(vol.transpose(2, 1, 0))).to(dev)  # [z][y][x]
        ar = torch.arange(L, device=dev)
        cc, idx = plan.new_results()
        crop = torch.empty((L, L, L), dtype=torch.float32, device=dev)
        w0, w1 = half - window, half + window + 1
        best_v = torch.empty(n, dtype=torch.float32, device=dev)
        best_k = torch.empty(n, dtype=torch.int64, device=dev)
        best_i = torch.empty(n, dtype=torch.int32, device=dev)
        for q, (c, angs) in enumerate(zip(centres, angle_sets)):
            zi, yi, xi = [(ar + int(c[d] - half)) % shape[d] for d in (2, 1, 0)]
            crop.copy_(vt.index_select(0, zi).index_select(1, yi).index_select(2, xi))
            plan.set_volume(crop)
            plan.init_results(cc, idx)
            grid, _ = angs
            plan.run(grid, cc, idx)
            # window maxima, flattened x-slowest (the order of an [x][y][z] array)
            wv = cc[w0:w1, w0:w1, w0:w1].permute(2, 1, 0).reshape(-1)
            wi = idx[w0:w1, w0:w1, w0:w1].permute(2, 1, 0).reshape(-1)
            k = torch.argmax(wv)
            best_v[q] = wv[k]
            best_k[q] = k
            best_i[q] = wi[k]
        torch.cuda.synchronize(ctx.device)
        vals, ks, locs = best_v.cpu().numpy(), best_k.cpu().numpy(), best_i.cpu().numpy()
    finally:
        plan.close()
    w = 2 * window + 1
    out_pos, out_idx = [], []
    for q, (c, angs) in enumerate(zip(centres, angle_sets)):
        kx, ky, kz = np.unravel_index(int(ks[q]), (w, w, w))
        out_pos.append([(c[0] + kx - window) % shape[0], (c[1] + ky - window) % shape[1],
                        (c[2] + kz - window) % shape[2]])
        ids = angs[1]
        out_idx.append(int(ids[locs[q]]) if locs[q] >= 0 else -1)
    return np.array(out_pos), np.asarray(vals, np.float64), np.array(out_idx)


def rotation_matrices(eulers):
    """The rot3d matrices of ZXZ Euler triplets [phi, psi, theta] in degrees,
    (n, 3, 3) float64 (Sptrans/tom_rotatec.c:164-288, vectorised)."""
    e = np.deg2rad(np.asarray(eulers, np.float64).reshape(-1, 3))
    cf, sf = np.cos(e[:, 0]), np.sin(e[:, 0])
    cp, sp = np.cos(e[:, 1]), np.sin(e[:, 1])
    ct, st = np.cos(e[:, 2]), np.sin(e[:, 2])
    R = np.empty((len(e), 3, 3))
    R[:, 0, 0] = cp * cf - ct * sp * sf
    R[:, 1, 0] = sp * cf + ct * cp * sf
    R[:, 2, 0] = st * sf
    R[:, 0, 1] = -cp * sf - ct * sp * cf
    R[:, 1, 1] = -sp * sf + ct * cp * cf
    R[:, 2, 1] = st * cf
    R[:, 0, 2] = st * sp
    R[:, 1, 2] = -st * cp
    R[:, 2, 2] = ct
    return R


def neighbours(fine_grid, centres, max_deg):
    """For each centre triplet, the indices of the fine-grid triplets whose
    rotation lies within max_deg of it (geodesic angle of R_f R_c^T)."""
    Rf = rotation_matrices(fine_grid).reshape(-1, 9)
    Rc = rotation_matrices(centres).reshape(-1, 9)
    lim = 1.0 + 2.0 * np.cos(np.deg2rad(max_deg))  # trace of a rotation by max_deg
    out = []
    for c in Rc:
        out.append(np.nonzero(Rf @ c >= lim - 1e-9)[0])
    return out


def bin_members(fine_grid, coarse_grid):
    """Fine-grid indices of each coarse bin (nearest-rotation partition)."""
    b = coarse_bin(fine_grid, coarse_grid)
    return [np.nonzero(b == k)[0] for k in range(len(coarse_grid))]
