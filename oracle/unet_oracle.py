"""CPU oracle of the U-Net candidate proposer (test infrastructure only).

A plain numpy restatement, in FP64, of the network that tom_b200/unet.py runs
on the tensor cores: 3x3x3 "same" cross-correlations on channels-last volumes
([Z][Y][X][C]), 2x2x2 average pooling, nearest 2x upsampling, channel
concatenation, ReLU, a 1x1 candidate head and, for the gradients, the
hand-written backward pass of each.  The proposer has no counterpart in TOM;
its data come from the search (search/tom_os3_findTemplate.m:255-307 is the
loop it prunes).  The product never imports this module: the tests compare
the library's kernels with it and check its gradients against central
differences.

Quantisation points: with bf16=True the forward pass rounds every stored
activation, the packed weights and the gradients between layers to BF16
(round to nearest even) exactly where the library stores BF16, so the
remaining difference to the GPU is FP32 versus FP64 accumulation.
"""
from __future__ import annotations

import numpy as np

# (name, cin, cout) of the 3x3x3 convolutions after the first layer; the
# concatenations are D2 = [up(e3) (64), e2 (32)] and D1 = [up(d2) (32), e1 (16)]
CONVS = (("e1b", 16, 16), ("e2a", 16, 32), ("e2b", 32, 32), ("e3a", 32, 64), ("e3b", 64, 64),
         ("d2a", 96, 32), ("d2b", 32, 32), ("d1a", 48, 16), ("d1b", 16, 16))


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(a, np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _q(a, on):
    return bf16(a) if on else np.asarray(a, np.float64)


def conv3(x, w, b=None):
    """out[z,y,x,co] = b[co] + sum_t sum_ci w[co,ci,t] x[z+dz-1, y+dy-1, x+dx-1, ci]
    (t = 9 dz + 3 dy + dx, zero outside)."""
    Z, Y, X, _ = x.shape
    xp = np.pad(np.asarray(x, np.float64), ((1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((Z, Y, X, w.shape[0]))
    for t in range(27):
        dz, dy, dx = t // 9, t // 3 % 3, t % 3
        out += xp[dz:dz + Z, dy:dy + Y, dx:dx + X, :] @ np.asarray(w[:, :, t], np.float64).T
    if b is not None:
        out += np.asarray(b, np.float64)
    return out


def conv3_grads(x, w, g):
    """(input gradient, weight gradient [co, ci, 27], bias gradient) of conv3."""
    Z, Y, X, _ = x.shape
    xp = np.pad(np.asarray(x, np.float64), ((1, 1), (1, 1), (1, 1), (0, 0)))
    gxp = np.zeros_like(xp)
    gw = np.zeros(w.shape)
    g = np.asarray(g, np.float64)
    for t in range(27):
        dz, dy, dx = t // 9, t // 3 % 3, t % 3
        win = xp[dz:dz + Z, dy:dy + Y, dx:dx + X, :]
        gw[:, :, t] = np.einsum("zyxo,zyxi->oi", g, win)
        gxp[dz:dz + Z, dy:dy + Y, dx:dx + X, :] += g @ np.asarray(w[:, :, t], np.float64)
    return gxp[1:-1, 1:-1, 1:-1, :], gw, g.sum(axis=(0, 1, 2))


def pool(x):
    Z, Y, X, C = x.shape
    return x.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C).mean(axis=(1, 3, 5))


def pool_bwd(g):
    return up(g) / 8.0


def up(x):
    return x.repeat(2, axis=0).repeat(2, axis=1).repeat(2, axis=2)


def up_bwd(g):
    Z, Y, X, C = g.shape
    return g.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C).sum(axis=(1, 3, 5))


def relu(a):
    return np.maximum(a, 0.0)


def init_params(n_bins, seed=0):
    """He-initialised FP32 parameters: w0 [16, 1, 27], b0, then per CONVS entry
    w [cout, cin, 27], b [cout], the candidate head wh [16], bh [1] and the
    orientation head Wo [n_bins, 16], bo [n_bins]."""
    r = np.random.default_rng(seed)
    p = {"w0": (r.standard_normal((16, 1, 27)) * np.sqrt(2.0 / 27)).astype(np.float32),
         "b0": np.zeros(16, np.float32)}
    for name, ci, co in CONVS:
        p["w_" + name] = (r.standard_normal((co, ci, 27)) * np.sqrt(2.0 / (27 * ci))).astype(np.float32)
        p["b_" + name] = np.zeros(co, np.float32)
    p["wh"] = (r.standard_normal(16) * 0.25).astype(np.float32)
    p["bh"] = np.full(1, -4.0, np.float32)
    p["Wo"] = (r.standard_normal((n_bins, 16)) * 0.25).astype(np.float32)
    p["bo"] = np.zeros(n_bins, np.float32)
    return p


def forward(p, vol, bf=False):
    """vol [Z][Y][X] (normalised) -> dict of the activations and 'logit' [Z][Y][X]."""
    a = {}
    x = np.asarray(vol, np.float64)[..., None]
    w = lambda k: _q(p[k], bf)  # noqa: E731  (the packed BF16 weights)
    a["e1a"] = _q(relu(conv3(x, np.asarray(p["w0"], np.float64), p["b0"])), bf)
    a["e1"] = _q(relu(conv3(a["e1a"], w("w_e1b"), p["b_e1b"])), bf)
    a["p1"] = _q(pool(a["e1"]), bf)
    a["e2a"] = _q(relu(conv3(a["p1"], w("w_e2a"), p["b_e2a"])), bf)
    a["e2"] = _q(relu(conv3(a["e2a"], w("w_e2b"), p["b_e2b"])), bf)
    a["p2"] = _q(pool(a["e2"]), bf)
    a["e3a"] = _q(relu(conv3(a["p2"], w("w_e3a"), p["b_e3a"])), bf)
    a["e3"] = _q(relu(conv3(a["e3a"], w("w_e3b"), p["b_e3b"])), bf)
    a["D2"] = np.concatenate([up(a["e3"]), a["e2"]], axis=3)
    a["d2a"] = _q(relu(conv3(a["D2"], w("w_d2a"), p["b_d2a"])), bf)
    a["d2"] = _q(relu(conv3(a["d2a"], w("w_d2b"), p["b_d2b"])), bf)
    a["D1"] = np.concatenate([up(a["d2"]), a["e1"]], axis=3)
    a["d1a"] = _q(relu(conv3(a["D1"], w("w_d1a"), p["b_d1a"])), bf)
    a["f"] = _q(relu(conv3(a["d1a"], w("w_d1b"), p["b_d1b"])), bf)
    a["logit"] = a["f"] @ np.asarray(p["wh"], np.float64) + float(p["bh"][0])
    return a


def backward(p, vol, a, g_logit, g_f_extra=None, bf=False, inter=None):
    """Gradients of every parameter for the upstream gradient g_logit [Z][Y][X]
    of the candidate logits (plus g_f_extra [Z][Y][X][16] on the features,
    e.g. from the orientation head).  Returns a dict keyed like the params;
    inter, a dict, receives the activation gradients between the layers."""
    gr = {}
    keep = inter if inter is not None else {}
    w = lambda k: _q(p[k], bf)  # noqa: E731
    mask = lambda g, act: g * (act > 0)  # noqa: E731
    g_logit = np.asarray(g_logit, np.float64)
    gr["wh"] = np.einsum("zyx,zyxc->c", g_logit, a["f"])
    gr["bh"] = np.array([g_logit.sum()])
    g = g_logit[..., None] * np.asarray(p["wh"], np.float64)
    if g_f_extra is not None:
        g = g + g_f_extra
    g = _q(mask(g, a["f"]), bf)
    keep["f"] = g

    def layer(name, x, g_out, act_in=None):
        gx, gw_, gb_ = conv3_grads(x, w("w_" + name), g_out)
        gr["w_" + name], gr["b_" + name] = gw_, gb_
        return gx if act_in is None else mask(gx, act_in)

    g = keep["d1a"] = _q(layer("d1b", a["d1a"], g, a["d1a"]), bf)
    gD1 = keep["D1"] = _q(layer("d1a", a["D1"], g, a["D1"]), bf)
    g = keep["d2"] = _q(up_bwd(gD1[..., :32]), bf)
    g = keep["d2a"] = _q(layer("d2b", a["d2a"], g, a["d2a"]), bf)
    gD2 = keep["D2"] = _q(layer("d2a", a["D2"], g, a["D2"]), bf)
    g = keep["e3"] = _q(up_bwd(gD2[..., :64]), bf)
    g = keep["e3a"] = _q(layer("e3b", a["e3a"], g, a["e3a"]), bf)
    g_p2 = keep["p2"] = _q(layer("e3a", a["p2"], g), bf)
    g_e2 = keep["e2"] = _q(gD2[..., 64:] + mask(pool_bwd(g_p2), a["e2"]), bf)
    g = keep["e2a"] = _q(layer("e2b", a["e2a"], g_e2, a["e2a"]), bf)
    g_p1 = keep["p1"] = _q(layer("e2a", a["p1"], g), bf)
    g_e1 = keep["e1"] = _q(gD1[..., 32:] + mask(pool_bwd(g_p1), a["e1"]), bf)
    g = keep["e1a"] = _q(layer("e1b", a["e1a"], g_e1, a["e1a"]), bf)
    _, gr["w0"], gr["b0"] = conv3_grads(np.asarray(vol, np.float64)[..., None], np.asarray(p["w0"], np.float64), g)
    return gr

