"""U-Net candidate proposer (no counterpart in TOM).

A 3-level 3-D U-Net (16 / 32 / 64 channels, 3x3x3 convolutions, 2x2x2
average pooling, nearest 2x upsampling with channel concatenation) reads a
normalised tomogram and predicts, per voxel, the probability of a particle
centre (a 1x1 head) and, at candidate voxels, one of the coarse orientation
bins (a dense head over the 16 features).  Labels come from the search itself
(the peaks of an exhaustive search and the coarse bin of their angle); the
pruned search then refines only around the proposals
(search/tom_os3_findTemplate.m:255-307 is the loop it replaces there).

Every layer runs on the library's own kernels through the C ABI
(tomgpu_unet_*): the 3x3x3 convolutions, their input gradients and weight
gradients as tcgen05 BF16 contractions with FP32 accumulation in tensor
memory; the first layer (one input channel), the heads, pooling and
upsampling as CUDA-core kernels; the losses, the dense orientation head and
Adam from tomgpu_cnn_*.  Activations and activation gradients are BF16
(channels-last), master weights, weight gradients and Adam state FP32; the
BF16 packed weights are re-derived after every update.  torch holds the
buffers only.

Layers (name: Cin -> Cout at level): first 1 -> 16, e1b 16 -> 16 (L1);
pool; e2a 16 -> 32, e2b 32 -> 32 (L2); pool; e3a 32 -> 64, e3b 64 -> 64 (L3);
up, concat with e2: d2a 96 -> 32, d2b 32 -> 32 (L2); up, concat with e1:
d1a 48 -> 16, d1b 16 -> 16 (L1); heads.  Every convolution is followed by a
ReLU.  The volume edges must be multiples of 4.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .tom import Context, _cdims, _tptr, default_context

CONVS = (("e1b", 16, 16), ("e2a", 16, 32), ("e2b", 32, 32), ("e3a", 32, 64), ("e3b", 64, 64),
         ("d2a", 96, 32), ("d2b", 32, 32), ("d1a", 48, 16), ("d1b", 16, 16))
FEAT = 16


def _call(ctx, name, *args):
    ctx.check(getattr(_lib.lib(), name)(ctx.handle, *args))


class UNetProposer:
    """Parameters, Adam state, packed weights, activation buffers and the
    forward / backward passes of the U-Net."""

    def __init__(self, n_bins: int, ctx: Context | None = None, seed: int = 0, params: dict | None = None):
        import torch
        self.ctx = ctx or default_context()
        self.dev = f"cuda:{self.ctx.device}"
        self.n_bins = int(n_bins)
        if params is None:
            params = init_params(self.n_bins, seed)
        self.p = {k: torch.from_numpy(np.ascontiguousarray(v, np.float32)).to(self.dev) for k, v in params.items()}
        self.g = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.m = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.pf = {n: torch.empty(27 * ci * co, dtype=torch.int16, device=self.dev) for n, ci, co in CONVS}
        self.pb = {n: torch.empty(27 * ci * co, dtype=torch.int16, device=self.dev) for n, ci, co in CONVS}
        self.step_count = 0
        self._shape = None
        self._train_bufs = False
        self.repack()

    # ------------------------------------------------------------ weights
    def repack(self):
        """The BF16 packed forms of every 3x3x3 convolution's weights."""
        for n, ci, co in CONVS:
            _call(self.ctx, "tomgpu_unet_pack_weights_dev", _tptr(self.p["w_" + n]), co, ci, 0, _tptr(self.pf[n]))
            _call(self.ctx, "tomgpu_unet_pack_weights_dev", _tptr(self.p["w_" + n]), co, ci, 1, _tptr(self.pb[n]))

    def params_numpy(self):
        return {k: v.cpu().numpy() for k, v in self.p.items()}

    # ------------------------------------------------------------ buffers
    def _alloc(self, shape_zyx, train):
        import torch
        if self._shape == tuple(shape_zyx) and (self._train_bufs or not train):
            return
        Z, Y, X = shape_zyx
        if Z % 4 or Y % 4 or X % 4:
            raise ValueError("volume edges must be multiples of 4")
        L1, L2, L3 = (Z, Y, X), (Z // 2, Y // 2, X // 2), (Z // 4, Y // 4, X // 4)
        self.a = self.ga = self.logit = None  # release the previous shape's buffers first

        def buf(L, c):
            return torch.zeros(L + (c,), dtype=torch.int16, device=self.dev)

        self.a = {"e1a": buf(L1, 16), "D1": buf(L1, 48), "p1": buf(L2, 16), "e2a": buf(L2, 32), "D2": buf(L2, 96),
                  "p2": buf(L3, 32), "e3a": buf(L3, 64), "e3": buf(L3, 64), "d2a": buf(L2, 32), "d2": buf(L2, 32),
                  "d1a": buf(L1, 16), "f": buf(L1, 16)}
        self.logit = torch.empty(L1, dtype=torch.float32, device=self.dev)
        if train:
            self.ga = {"f": buf(L1, 16), "d1a": buf(L1, 16), "D1": buf(L1, 48), "d2": buf(L2, 32),
                       "d2a": buf(L2, 32), "D2": buf(L2, 96), "e3": buf(L3, 64), "e3a": buf(L3, 64),
                       "p2": buf(L3, 32), "e2a": buf(L2, 32), "p1": buf(L2, 16), "e1a": buf(L1, 16)}
        self._shape = tuple(shape_zyx)
        self._train_bufs = train
        self.dims = [_cdims((X, Y, Z)), _cdims((X // 2, Y // 2, Z // 2)), _cdims((X // 4, Y // 4, Z // 4))]

    def _conv(self, name, src, cs, off, cin, lvl, cout, dst, dcs, doff):
        _call(self.ctx, "tomgpu_unet_conv3_dev", _tptr(src), cs, off, cin, self.dims[lvl], _tptr(self.pf[name]), cout,
              _tptr(self.p["b_" + name]), 1, None, 0, 0, _tptr(dst), dcs, doff)

    # ------------------------------------------------------------ forward
    def forward(self, vol, train=False, prob=False):
        """vol: torch float32 [Z][Y][X] on the device (normalised).  Returns the
        candidate logits [Z][Y][X] (prob: their sigmoid, the centre
        probabilities; a buffer reused by the next call)."""
        ctx = self.ctx
        self._alloc(tuple(vol.shape), train)
        a = self.a
        self.vol = vol
        _call(ctx, "tomgpu_unet_conv_first_dev", _tptr(vol), self.dims[0], _tptr(self.p["w0"]), _tptr(self.p["b0"]),
              _tptr(a["e1a"]))
        self._conv("e1b", a["e1a"], 16, 0, 16, 0, 16, a["D1"], 48, 32)
        _call(ctx, "tomgpu_unet_pool_dev", _tptr(a["D1"]), 48, 32, 16, self.dims[0], _tptr(a["p1"]))
        self._conv("e2a", a["p1"], 16, 0, 16, 1, 32, a["e2a"], 32, 0)
        self._conv("e2b", a["e2a"], 32, 0, 32, 1, 32, a["D2"], 96, 64)
        _call(ctx, "tomgpu_unet_pool_dev", _tptr(a["D2"]), 96, 64, 32, self.dims[1], _tptr(a["p2"]))
        self._conv("e3a", a["p2"], 32, 0, 32, 2, 64, a["e3a"], 64, 0)
        self._conv("e3b", a["e3a"], 64, 0, 64, 2, 64, a["e3"], 64, 0)
        _call(ctx, "tomgpu_unet_upsample_dev", _tptr(a["e3"]), 64, self.dims[1], _tptr(a["D2"]), 96, 0)
        self._conv("d2a", a["D2"], 96, 0, 96, 1, 32, a["d2a"], 32, 0)
        self._conv("d2b", a["d2a"], 32, 0, 32, 1, 32, a["d2"], 32, 0)
        _call(ctx, "tomgpu_unet_upsample_dev", _tptr(a["d2"]), 32, self.dims[0], _tptr(a["D1"]), 48, 0)
        self._conv("d1a", a["D1"], 48, 0, 48, 0, 16, a["d1a"], 16, 0)
        self._conv("d1b", a["d1a"], 16, 0, 16, 0, 16, a["f"], 16, 0)
        _call(ctx, "tomgpu_unet_head_dev", _tptr(a["f"]), self.logit.numel(), _tptr(self.p["head"]),
              1 if prob else 0, _tptr(self.logit))
        return self.logit

    def orient_logits(self, idx):
        """Orientation logits [n_bins][P] at flat voxel indices idx (int64 tensor)
        of the last forward pass; also returns the gathered features [16][P]."""
        import torch
        P = int(idx.numel())
        fg = torch.empty((FEAT, P), device=self.dev)
        _call(self.ctx, "tomgpu_unet_gather_dev", _tptr(self.a["f"]), FEAT, _tptr(idx), P, _tptr(fg))
        out = torch.empty((self.n_bins, P), device=self.dev)
        _call(self.ctx, "tomgpu_cnn_dense_fwd_dev", _tptr(self.p["Wo"]), _tptr(self.p["bo"]), _tptr(fg), self.n_bins,
              FEAT, P, 0, _tptr(out))
        return fg, out

    # ------------------------------------------------------------ backward
    def _bwd_conv(self, name, x, xcs, xoff, cin, lvl, g, gcs, goff, cout, gin, mask, mcs, moff, n_vox):
        """Weight, bias and (when gin is given) input gradients of one convolution."""
        ctx = self.ctx
        _call(ctx, "tomgpu_unet_channel_sum_dev", _tptr(g), gcs, goff, cout, n_vox, _tptr(self.g["b_" + name]))
        _call(ctx, "tomgpu_unet_conv3_wgrad_dev", _tptr(x), xcs, xoff, cin, self.dims[lvl], _tptr(g), gcs, goff, cout,
              _tptr(self.g["w_" + name]))
        if gin is not None:
            _call(ctx, "tomgpu_unet_conv3_dev", _tptr(g), gcs, goff, cout, self.dims[lvl], _tptr(self.pb[name]), cin,
                  None, 0, None if mask is None else _tptr(mask), mcs, moff, _tptr(gin), cin if mask is None else mcs,
                  0 if mask is None else moff)

    def backward(self, g_logit, orient=None):
        """Accumulate the parameter gradients (zero them first) for the
        gradient g_logit [Z][Y][X] of the candidate logits and, optionally,
        orient = (idx, fg, g_orient_logits [n_bins][P]) of the orientation head."""
        import torch
        ctx, a, ga = self.ctx, self.a, self.ga
        Z, Y, X = self._shape
        n1 = X * Y * Z
        n2, n3 = n1 // 8, n1 // 64
        _call(ctx, "tomgpu_unet_head_bwd_dev", _tptr(a["f"]), n1, _tptr(self.p["head"]), _tptr(g_logit),
              _tptr(ga["f"]), _tptr(self.g["head"]))
        if orient is not None:
            idx, fg, g_ol = orient
            P = int(idx.numel())
            g_fg = torch.empty_like(fg)
            _call(ctx, "tomgpu_cnn_dense_bwd_dev", _tptr(self.p["Wo"]), _tptr(fg), _tptr(g_ol), self.n_bins, FEAT, P,
                  _tptr(g_fg), _tptr(self.g["Wo"]), _tptr(self.g["bo"]))
            _call(ctx, "tomgpu_unet_scatter_add_dev", _tptr(g_fg), FEAT, _tptr(idx), P, _tptr(a["f"]), _tptr(ga["f"]))
        self._bwd_conv("d1b", a["d1a"], 16, 0, 16, 0, ga["f"], 16, 0, 16, ga["d1a"], a["d1a"], 16, 0, n1)
        self._bwd_conv("d1a", a["D1"], 48, 0, 48, 0, ga["d1a"], 16, 0, 16, ga["D1"], a["D1"], 48, 0, n1)
        _call(ctx, "tomgpu_unet_upsample_bwd_dev", _tptr(ga["D1"]), 48, 0, 32, self.dims[0], _tptr(ga["d2"]))
        self._bwd_conv("d2b", a["d2a"], 32, 0, 32, 1, ga["d2"], 32, 0, 32, ga["d2a"], a["d2a"], 32, 0, n2)
        self._bwd_conv("d2a", a["D2"], 96, 0, 96, 1, ga["d2a"], 32, 0, 32, ga["D2"], a["D2"], 96, 0, n2)
        _call(ctx, "tomgpu_unet_upsample_bwd_dev", _tptr(ga["D2"]), 96, 0, 64, self.dims[1], _tptr(ga["e3"]))
        self._bwd_conv("e3b", a["e3a"], 64, 0, 64, 2, ga["e3"], 64, 0, 64, ga["e3a"], a["e3a"], 64, 0, n3)
        self._bwd_conv("e3a", a["p2"], 32, 0, 32, 2, ga["e3a"], 64, 0, 64, ga["p2"], None, 0, 0, n3)
        _call(ctx, "tomgpu_unet_pool_bwd_dev", _tptr(ga["p2"]), 32, self.dims[1], _tptr(a["D2"]), 96, 64,
              _tptr(ga["D2"]), 1)
        self._bwd_conv("e2b", a["e2a"], 32, 0, 32, 1, ga["D2"], 96, 64, 32, ga["e2a"], a["e2a"], 32, 0, n2)
        self._bwd_conv("e2a", a["p1"], 16, 0, 16, 1, ga["e2a"], 32, 0, 32, ga["p1"], None, 0, 0, n2)
        _call(ctx, "tomgpu_unet_pool_bwd_dev", _tptr(ga["p1"]), 16, self.dims[0], _tptr(a["D1"]), 48, 32,
              _tptr(ga["D1"]), 1)
        self._bwd_conv("e1b", a["e1a"], 16, 0, 16, 0, ga["D1"], 48, 32, 16, ga["e1a"], a["e1a"], 16, 0, n1)
        _call(ctx, "tomgpu_unet_conv_first_wgrad_dev", _tptr(self.vol), self.dims[0], _tptr(ga["e1a"]),
              _tptr(self.g["w0"]), _tptr(self.g["b0"]))

    # ------------------------------------------------------------ training
    def zero_grad(self):
        for t in self.g.values():
            t.zero_()

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        for k in self.p:
            _call(self.ctx, "tomgpu_cnn_adam_dev", _tptr(self.p[k]), _tptr(self.g[k]), _tptr(self.m[k]),
                  _tptr(self.v[k]), self.p[k].numel(), float(lr), float(beta1), float(beta2), float(eps),
                  self.step_count)
        self.repack()

    def train_step(self, vol, target, pos_idx, pos_bins, pos_weight=50.0, lr=1e-3, w_orient=0.2):
        """One Adam step on one sample.  vol, target: torch [Z][Y][X] on the
        device; pos_idx: flat indices of the labelled centres (int64), pos_bins:
        their coarse bins (int32).  Returns (centre loss, orientation loss)."""
        import torch
        ctx = self.ctx
        self.zero_grad()
        logit = self.forward(vol, train=True)
        n = logit.numel()
        loss = torch.zeros(2, dtype=torch.float64, device=self.dev)
        g_logit = torch.empty_like(logit)
        _call(ctx, "tomgpu_cnn_bce_dev", _tptr(logit), _tptr(target), n, float(pos_weight), _tptr(g_logit),
              _tptr(loss[0:1]))
        orient = None
        P = int(pos_idx.numel())
        if P > 0 and w_orient > 0:
            fg, ol = self.orient_logits(pos_idx)
            g_ol = torch.empty_like(ol)
            _call(ctx, "tomgpu_cnn_softmax_ce_dev", _tptr(ol), _tptr(pos_bins), self.n_bins, P, _tptr(g_ol),
                  _tptr(loss[1:2]))
            g_ol.mul_(w_orient)
            orient = (pos_idx, fg, g_ol)
        self.backward(g_logit, orient)
        self.adam(lr)
        out = loss.cpu().numpy()
        return float(out[0]), float(out[1])

    def flops_per_voxel(self):
        """Multiply-adds x 2 of one forward pass per full-resolution voxel."""
        lv = {"e1b": 1, "e2a": 8, "e2b": 8, "e3a": 64, "e3b": 64, "d2a": 8, "d2b": 8, "d1a": 1, "d1b": 1}
        macs = 27 * 16 + 16 + sum(27 * ci * co / lv[n] for n, ci, co in CONVS)
        return 2 * macs


def init_params(n_bins, seed=0):
    """He-initialised FP32 parameters: w0 [16, 1, 27], b0 [16], per convolution
    w_<name> [Cout, Cin, 27] and b_<name> [Cout], the candidate head
    head [17] (16 weights, bias -4: rare positives start near p = 0.02) and
    the orientation head Wo [n_bins, 16], bo [n_bins]."""
    r = np.random.default_rng(seed)
    p = {"w0": (r.standard_normal((16, 1, 27)) * np.sqrt(2.0 / 27)).astype(np.float32),
         "b0": np.zeros(16, np.float32)}
    for name, ci, co in CONVS:
        p["w_" + name] = (r.standard_normal((co, ci, 27)) * np.sqrt(2.0 / (27 * ci))).astype(np.float32)
        p["b_" + name] = np.zeros(co, np.float32)
    p["head"] = np.concatenate([r.standard_normal(16) * 0.25, [-4.0]]).astype(np.float32)
    p["Wo"] = (r.standard_normal((n_bins, 16)) * 0.25).astype(np.float32)
    p["bo"] = np.zeros(n_bins, np.float32)
    return p


# ------------------------------------------------------------------ inference


def normalise(vol, ctx=None, out=None):
    """(vol - mean) / std of a device volume (moments in FP64 on the device)."""
    import torch
    ctx = ctx or default_context()
    out = torch.empty_like(vol) if out is None else out
    _call(ctx, "tomgpu_unet_normalise_dev", _tptr(vol), vol.numel(), _tptr(out))
    return out


def bin2(vol, ctx=None):
    """2x2x2 mean of a device volume [Z][Y][X] (even edges)."""
    import torch
    ctx = ctx or default_context()
    Z, Y, X = vol.shape
    out = torch.empty((Z // 2, Y // 2, X // 2), dtype=torch.float32, device=vol.device)
    _call(ctx, "tomgpu_unet_bin2_dev", _tptr(vol), _cdims((X, Y, Z)), _tptr(out))
    return out


def prepare(vol_host, binning, ctx, dev):
    """A host tomogram [x][y][z] on the device as the network's input:
    [Z][Y][X], binned by 2 when binning == 2, normalised."""
    import torch
    v = torch.from_numpy(np.ascontiguousarray(np.asarray(vol_host, np.float32).transpose(2, 1, 0))).to(dev)
    if binning == 2:
        v = bin2(v, ctx)
    elif binning != 1:
        raise ValueError("binning is 1 or 2")
    return normalise(v, ctx, out=v)


def infer(net, vol, slab=128, halo=32, prob=True):
    """Centre probabilities (prob=False: logits) [Z][Y][X] and the features
    [Z][Y][X][16] (BF16 bits) of a whole normalised volume, in z slabs of
    `slab` planes each run with `halo` more planes on either side (zero beyond
    the volume), which bounds the activation memory.  An output voxel reads
    the input within 23 voxels of it (the ten convolutions at their levels
    through the pooling and upsampling), and the slabs start on multiples of
    4, so the pooling grids stay aligned: with halo >= 24 every voxel's
    outputs are those of the whole-volume pass.  slab and halo are multiples
    of 4."""
    import torch
    Z, Y, X = vol.shape
    if slab % 4 or halo % 4 or Z % 4:
        raise ValueError("slab, halo and the z edge must be multiples of 4")
    out = torch.empty((Z, Y, X), dtype=torch.float32, device=net.dev)
    feat = torch.empty((Z, Y, X, FEAT), dtype=torch.int16, device=net.dev)
    for z0 in range(0, Z, slab):
        z1 = min(Z, z0 + slab)
        lo, hi = max(0, z0 - halo), min(Z, z1 + halo)
        lg = net.forward(vol[lo:hi], prob=prob)
        out[z0:z1].copy_(lg[z0 - lo:z1 - lo])
        feat[z0:z1].copy_(net.a["f"][z0 - lo:z1 - lo])
    return out, feat


def orient_logits_at(net, feat, idx):
    """Orientation logits [n_bins][P] at flat voxel indices idx (int64 tensor)
    of a feature volume from infer()."""
    import torch
    P = int(idx.numel())
    fg = torch.empty((FEAT, P), device=net.dev)
    _call(net.ctx, "tomgpu_unet_gather_dev", _tptr(feat), FEAT, _tptr(idx), P, _tptr(fg))
    out = torch.empty((net.n_bins, P), device=net.dev)
    _call(net.ctx, "tomgpu_cnn_dense_fwd_dev", _tptr(net.p["Wo"]), _tptr(net.p["bo"]), _tptr(fg), net.n_bins, FEAT,
          P, 0, _tptr(out))
    return out


def propose(net, vol, n_cand, radius, top_bins, slab=128, halo=32, border=16):
    """Candidates of the network on a normalised device volume [Z][Y][X]: the
    n_cand first maxima of the centre probability (tom_peak rounds with a ball
    of `radius`), 0-based [x, y, z], their probabilities and the top_bins
    orientation bins of each (most probable first).  Voxels within `border`
    of a face are not proposed: the network sees the zero padding there."""
    import torch
    from .tom import pick_peaks
    prob, feat = infer(net, vol, slab, halo, prob=True)
    Z, Y, X = prob.shape
    if border > 0:
        b = int(border)
        prob[:b].zero_()
        prob[Z - b:].zero_()
        prob[:, :b].zero_()
        prob[:, Y - b:].zero_()
        prob[:, :, :b].zero_()
        prob[:, :, X - b:].zero_()
    dummy = torch.zeros((Z, Y, X), dtype=torch.int32, device=net.dev)
    vals, pos, _ = pick_peaks(prob, dummy, n_cand, radius, net.ctx)
    del dummy
    ok = pos[:, 0] > 0
    pos, vals = pos[ok] - 1, vals[ok]
    fi = torch.from_numpy((pos[:, 0] + X * (pos[:, 1] + Y * pos[:, 2])).astype(np.int64)).to(net.dev)
    ol = orient_logits_at(net, feat, fi)
    bins = torch.topk(ol, k=min(top_bins, net.n_bins), dim=0).indices.t().cpu().numpy()
    return pos, vals, bins


def propose_host(net, vol, n_cand, radius, top_bins, binning=1, slab=128, halo=32):
    """propose() on a host tomogram [x][y][z] (binned by 2 first when binning
    == 2); radius in tomogram voxels; positions returned in tomogram voxels
    (a binned candidate at the centre of its 2^3 block)."""
    v = prepare(vol, binning, net.ctx, net.dev)
    pos, vals, bins = propose(net, v, n_cand, radius / binning, top_bins, slab, halo, border=16 // binning)
    del v
    return unbin_positions(pos, binning, np.shape(vol)), vals, bins


def unbin_positions(pos, binning, shape_xyz):
    """Tomogram voxels (0-based [x, y, z]) of positions on a volume binned by
    `binning`: the voxel at the upper centre of each binned voxel's block,
    inside the tomogram."""
    pos = np.asarray(pos, np.int64).reshape(-1, 3)
    if binning == 1:
        return pos
    return np.minimum(binning * pos + binning // 2, np.asarray(shape_xyz, np.int64) - 1)


def rerank_scores(net, vol, pos, binning=1, slab=128, halo=32):
    """The network's centre probability at each candidate (0-based [x, y, z]
    tomogram voxels) of a host tomogram [x][y][z]: the maximum over the
    candidate's (binned) voxel and its 26 neighbours."""
    import torch
    v = prepare(vol, binning, net.ctx, net.dev)
    prob, _ = infer(net, v, slab, halo, prob=True)
    del v
    Z, Y, X = prob.shape
    p = torch.as_tensor(np.asarray(pos, np.int64) // binning, device=net.dev)
    best = torch.full((p.shape[0],), -1.0, device=net.dev)
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                best = torch.maximum(best, prob[(p[:, 2] + dz).clamp(0, Z - 1), (p[:, 1] + dy).clamp(0, Y - 1),
                                                (p[:, 0] + dx).clamp(0, X - 1)])
    return best.cpu().numpy()


def learned_pruned_search(vol, template, mask, fine, coarse, net, n_cand, top_bins, radius_deg, window=2,
                          peak_radius=None, slab=128, halo=32, binning=1, ctx=None, timings=None):
    """The pruned search with the network in place of the coarse search: the
    network's n_cand candidates on the tomogram, and around each the fine
    triplets within radius_deg (geodesic) of its top_bins coarse orientation
    bins searched on a crop (proposer.refine: the values equal the full
    search's there), the best within +-window voxels.  vol: the tomogram as a
    host array [x][y][z]; binning 2 runs the network on the 2x2x2-binned
    tomogram (twice the receptive field in tomogram voxels) and maps its
    candidates back to the centres of their 2^3 blocks.  Returns (positions 0-based [x, y, z], cc, fine
    triplet index) per candidate; timings receives the seconds per step."""
    import time
    import torch
    from . import proposer as pr
    ctx = ctx or net.ctx
    T = np.shape(template)[0]
    clock = []

    def mark():
        torch.cuda.synchronize(ctx.device)
        clock.append(time.perf_counter())

    mark()
    pos, _, bins = propose_host(net, vol, n_cand, T / 2 if peak_radius is None else peak_radius, top_bins,
                                binning, slab, halo)
    mark()
    coarse = np.asarray(coarse)
    ub = np.unique(np.asarray(bins).reshape(-1))
    per_bin = dict(zip(ub.tolist(), pr.neighbours(fine, coarse[ub], radius_deg)))
    sets = []
    for b in bins:
        ids = np.unique(np.concatenate([per_bin[int(k)] for k in b]))
        sets.append((np.asarray(fine)[ids], ids))
    mark()
    out = pr.refine(vol, template, mask, pos, sets, window=window, ctx=ctx)
    mark()
    if timings is not None:
        for k, name in enumerate(("network", "triplet_sets", "refine")):
            timings[name] = clock[k + 1] - clock[k]
        timings["total"] = clock[-1] - clock[0]
        timings["candidates_n"] = int(len(pos))
        timings["triplets_per_candidate"] = float(np.mean([len(s[1]) for s in sets])) if sets else 0.0
    return out


# ------------------------------------------------------------------ training data


def training_sample(N, T, n_copies, n_blobs, rho, snr, max_tilt, seed, phantom, mask, coarse, fine=None, ctx=None,
                    binning=1):
    """A seeded synthetic tomogram and its labels from the search itself: the
    n_copies first peaks of the exhaustive search (tom_peak rounds of radius
    T/2) over the fine grid when given, else over the coarse grid, their
    positions and the coarse bins of their angles.  binning 2: the volume
    2x2x2-binned and the positions halved.  Returns (normalised volume
    [Z][Y][X] float32, positions 0-based [x, y, z], bins)."""
    from . import proposer as pr
    from . import synth
    from .tom import pick_peaks
    ctx = ctx or default_context()
    d = synth.make_tomogram(N, T, n_copies, n_blobs, rho, snr, max_tilt, seed=seed, mask_radius=T // 2 - 1,
                            phantom=phantom)
    grid = coarse if fine is None else fine
    cc, idx = pr.search(d["tomo"], d["template"], mask, grid, batch=16, ctx=ctx)
    _, pos, aidx = pick_peaks(cc, idx, n_copies, T / 2, ctx)
    del cc, idx
    ok = aidx >= 0
    bins = aidx[ok] if fine is None else pr.coarse_bin(np.asarray(fine)[aidx[ok]], coarse)
    v = prepare(d["tomo"], binning, ctx, f"cuda:{ctx.device}")
    return v, (pos[ok] - 1) // binning, np.asarray(bins, np.int32)


def ball_target(shape_zyx, pos, radius, dev):
    """1 within `radius` voxels of each label position, 0 elsewhere; [Z][Y][X]."""
    import torch
    Z, Y, X = shape_zyx
    t = np.zeros((Z, Y, X), np.float32)
    r = int(np.floor(radius))
    off = [(dx, dy, dz) for dz in range(-r, r + 1) for dy in range(-r, r + 1) for dx in range(-r, r + 1)
           if dx * dx + dy * dy + dz * dz <= radius * radius]
    for x, y, z in np.asarray(pos, np.int64).reshape(-1, 3):
        for dx, dy, dz in off:
            t[(z + dz) % Z, (y + dy) % Y, (x + dx) % X] = 1.0
    return torch.from_numpy(t).to(dev)


def train(net, samples, steps, pos_weight=300.0, lr=1e-3, w_orient=0.2, start=0, target_radius=3.0):
    """steps Adam steps cycling over samples [(volume, positions, bins)]:
    binary cross-entropy of the centre probability against balls of
    target_radius around the labels (positives weighted by pos_weight: a
    particle is a few hundred voxels of millions) and softmax cross-entropy
    of the orientation bin at the labels.  Returns the (centre loss,
    orientation loss) of every step."""
    import torch
    prep = []
    for v, pos, bins in samples:
        Z, Y, X = v.shape
        p = np.asarray(pos, np.int64).reshape(-1, 3)
        fi = torch.from_numpy(p[:, 0] + X * (p[:, 1] + Y * p[:, 2])).to(net.dev)
        prep.append((v, ball_target((Z, Y, X), p, target_radius, net.dev), fi,
                     torch.from_numpy(np.asarray(bins, np.int32)).to(net.dev)))
    out = []
    for i in range(start, start + steps):
        v, t, fi, b = prep[i % len(prep)]
        out.append(net.train_step(v, t, fi, b, pos_weight=pos_weight, lr=lr, w_orient=w_orient))
    return out
