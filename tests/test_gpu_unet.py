"""The U-Net proposer's kernels against the FP64 oracle (oracle/unet_oracle.py).

Tolerances.  A BF16 output (convolutions, pooling, gradients between layers)
is compared with the oracle's FP64 value rounded to BF16: they differ by at
most one BF16 unit (2^-7 relative) where the FP32 and FP64 sums fall on the
two sides of a rounding boundary.  FP32 outputs (weight gradients, heads) are
sums of exact BF16 products: within 1e-4 of the largest value.  The whole
network (10 layers, BF16 between them, the oracle rounding at the same
points): activations and logits within 2e-2 in relative norm, and every
parameter gradient, given the same activations, within 2e-2."""
import ctypes

import numpy as np
import pytest

import unet_oracle as uo

pytestmark = pytest.mark.gpu


def _bf(a, dev):
    """BF16 bit patterns (torch int16) of a float array, channels-last as given."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32))).to(dev)
    return t.to(torch.bfloat16).view(torch.int16).contiguous()


def _from_bf(t):
    import torch
    return t.view(torch.bfloat16).float().cpu().numpy().astype(np.float64)


def _f32(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32))).to(dev)


def _bf_close(got, ref):
    r = uo.bf16(ref)
    assert np.all(np.abs(got - r) <= 2 ** -7 * np.abs(r) + 1e-6 * max(np.abs(r).max(), 1e-30))


def _close(got, ref, rel=1e-4):
    assert np.abs(np.asarray(got, np.float64) - ref).max() <= rel * max(np.abs(ref).max(), 1e-12)


def _call(ctx, name, *args):
    from tom_b200 import _lib
    ctx.check(getattr(_lib.lib(), name)(ctx.handle, *args))


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("cin,cout,masked,Y", [(16, 16, False, 21), (32, 64, False, 21), (96, 32, False, 21),
                                               (48, 16, True, 21), (64, 64, True, 21), (16, 96, True, 21),
                                               (32, 48, False, 21), (16, 16, False, 45), (48, 32, True, 45),
                                               (96, 96, False, 45), (64, 64, True, 70)])
def test_conv3_tensor_cores_vs_oracle(gpu, cin, cout, masked, Y):
    import torch
    ctx = gpu.default_context()
    dev = f"cuda:{ctx.device}"
    rng = np.random.default_rng(cin * 7 + cout + Y)
    # partial tiles in x (8) and y (16; blocks of two tiles where Y >= 34)
    Z, X = 5, 26
    # the input as a channel slice of a wider buffer, the output likewise
    ics, ioff, ocs, ooff = cin + 16, 8, cout + 8, 8
    xin = uo.bf16(rng.standard_normal((Z, Y, X, ics)))
    w = uo.bf16(rng.standard_normal((cout, cin, 27)) * 0.2)
    b = rng.standard_normal(cout).astype(np.float32)
    m = uo.bf16(rng.standard_normal((Z, Y, X, ocs)))
    tin, tm = _bf(xin, dev), _bf(m, dev)
    tw, tb_ = _f32(w, dev), _f32(b, dev)
    pk = torch.empty(27 * cin * cout, dtype=torch.int16, device=dev)
    _call(ctx, "tomgpu_unet_pack_weights_dev", _p(tw), cout, cin, 0, _p(pk))
    out = torch.full((Z, Y, X, ocs), 7, dtype=torch.int16, device=dev)
    dims = (ctypes.c_int * 3)(X, Y, Z)
    _call(ctx, "tomgpu_unet_conv3_dev", _p(tin), ics, ioff, cin, dims, _p(pk), cout, _p(tb_), 0 if masked else 1,
          _p(tm) if masked else None, ocs, ooff, _p(out), ocs, ooff)
    ctx.synchronize()
    ref = uo.conv3(xin[..., ioff:ioff + cin], w, b)
    ref = ref * (m[..., ooff:ooff + cout] > 0) if masked else np.maximum(ref, 0)
    got = _from_bf(out)
    _bf_close(got[..., ooff:ooff + cout], ref)
    # the channels outside the slice are untouched
    assert np.all(out[..., :ooff].cpu().numpy() == 7)


@pytest.mark.parametrize("cin,cout", [(16, 16), (48, 16), (96, 32), (64, 64), (32, 64)])
def test_conv3_input_gradient_and_weight_gradient(gpu, cin, cout):
    import torch
    ctx = gpu.default_context()
    dev = f"cuda:{ctx.device}"
    rng = np.random.default_rng(cin + 13 * cout)
    Z, Y, X = 4, 18, 19
    x = uo.bf16(rng.standard_normal((Z, Y, X, cin)))
    g = uo.bf16(rng.standard_normal((Z, Y, X, cout)))
    w = uo.bf16(rng.standard_normal((cout, cin, 27)) * 0.2)
    gx_ref, gw_ref, _ = uo.conv3_grads(x, w, g)
    tx, tg, tw = _bf(x, dev), _bf(g, dev), _f32(w, dev)
    dims = (ctypes.c_int * 3)(X, Y, Z)
    pk = torch.empty(27 * cin * cout, dtype=torch.int16, device=dev)
    _call(ctx, "tomgpu_unet_pack_weights_dev", _p(tw), cout, cin, 1, _p(pk))
    gx = torch.empty((Z, Y, X, cin), dtype=torch.int16, device=dev)
    _call(ctx, "tomgpu_unet_conv3_dev", _p(tg), cout, 0, cout, dims, _p(pk), cin, None, 0, None, 0, 0, _p(gx), cin, 0)
    gw = torch.zeros((cout, cin, 27), dtype=torch.float32, device=dev)
    _call(ctx, "tomgpu_unet_conv3_wgrad_dev", _p(tx), cin, 0, cin, dims, _p(tg), cout, 0, cout, _p(gw))
    ctx.synchronize()
    _bf_close(_from_bf(gx), gx_ref)
    _close(gw.cpu().numpy(), gw_ref)


def test_first_layer_head_pool_upsample_and_sums(gpu):
    import torch
    ctx = gpu.default_context()
    dev = f"cuda:{ctx.device}"
    rng = np.random.default_rng(5)
    Z, Y, X = 6, 10, 12
    n = X * Y * Z
    dims = (ctypes.c_int * 3)(X, Y, Z)
    vol = rng.standard_normal((Z, Y, X)).astype(np.float32)
    w0 = (rng.standard_normal((16, 1, 27)) * 0.3).astype(np.float32)
    b0 = rng.standard_normal(16).astype(np.float32)
    # (every buffer a kernel reads is held in a variable until the stream has
    # synchronised: a temporary's memory could be reused by the next upload)
    e = torch.empty((Z, Y, X, 16), dtype=torch.int16, device=dev)
    tv, tw0, tb0 = _f32(vol, dev), _f32(w0, dev), _f32(b0, dev)
    _call(ctx, "tomgpu_unet_conv_first_dev", _p(tv), dims, _p(tw0), _p(tb0), _p(e))
    ctx.synchronize()
    _bf_close(_from_bf(e), np.maximum(uo.conv3(vol[..., None], w0, b0), 0))
    g = uo.bf16(rng.standard_normal((Z, Y, X, 16)))
    gw = torch.zeros(16 * 27, device=dev)
    gb = torch.zeros(16, device=dev)
    tg = _bf(g, dev)
    _call(ctx, "tomgpu_unet_conv_first_wgrad_dev", _p(tv), dims, _p(tg), _p(gw), _p(gb))
    _, gw_ref, gb_ref = uo.conv3_grads(vol[..., None], w0, g)
    ctx.synchronize()
    _close(gw.cpu().numpy().reshape(16, 1, 27), gw_ref)
    _close(gb.cpu().numpy(), gb_ref)
    # head and its backward
    f = uo.bf16(np.maximum(rng.standard_normal((Z, Y, X, 16)), 0))
    hw = rng.standard_normal(17).astype(np.float32)
    tf = _bf(f, dev)
    logit = torch.empty((Z, Y, X), device=dev)
    thw = _f32(hw, dev)
    _call(ctx, "tomgpu_unet_head_dev", _p(tf), n, _p(thw), 0, _p(logit))
    prob = torch.empty((Z, Y, X), device=dev)
    _call(ctx, "tomgpu_unet_head_dev", _p(tf), n, _p(thw), 1, _p(prob))
    ctx.synchronize()
    lref = f @ hw[:16].astype(np.float64) + hw[16]
    _close(logit.cpu().numpy(), lref, 1e-5)
    _close(prob.cpu().numpy(), 1 / (1 + np.exp(-lref)), 1e-5)
    gl = rng.standard_normal((Z, Y, X)).astype(np.float32)
    gf = torch.empty((Z, Y, X, 16), dtype=torch.int16, device=dev)
    ghw = torch.zeros(17, device=dev)
    tgl = _f32(gl, dev)
    _call(ctx, "tomgpu_unet_head_bwd_dev", _p(tf), n, _p(thw), _p(tgl), _p(gf), _p(ghw))
    ctx.synchronize()
    _bf_close(_from_bf(gf), gl[..., None] * hw[:16] * (f > 0))
    _close(ghw.cpu().numpy()[:16], np.einsum("zyx,zyxc->c", gl, f))
    _close(ghw.cpu().numpy()[16:], np.array([gl.astype(np.float64).sum()]))
    # pooling of a channel slice, its backward with mask and accumulation
    C, cs, off = 32, 48, 16
    a = uo.bf16(rng.standard_normal((Z, Y, X, cs)))
    pooled = torch.empty((Z // 2, Y // 2, X // 2, C), dtype=torch.int16, device=dev)
    ta = _bf(a, dev)
    _call(ctx, "tomgpu_unet_pool_dev", _p(ta), cs, off, C, dims, _p(pooled))
    ctx.synchronize()
    _bf_close(_from_bf(pooled), uo.pool(a[..., off:off + C]))
    gp = uo.bf16(rng.standard_normal((Z // 2, Y // 2, X // 2, C)))
    base = uo.bf16(rng.standard_normal((Z, Y, X, cs)))
    tbase = _bf(base, dev)
    tgp = _bf(gp, dev)
    _call(ctx, "tomgpu_unet_pool_bwd_dev", _p(tgp), C, dims, _p(ta), cs, off, _p(tbase), 1)
    ctx.synchronize()
    _bf_close(_from_bf(tbase)[..., off:off + C],
              base[..., off:off + C] + uo.pool_bwd(gp) * (a[..., off:off + C] > 0))
    # upsampling into a slice and its backward
    u = torch.zeros((Z, Y, X, cs), dtype=torch.int16, device=dev)
    _call(ctx, "tomgpu_unet_upsample_dev", _p(tgp), C, dims, _p(u), cs, off)
    ctx.synchronize()
    assert np.array_equal(_from_bf(u)[..., off:off + C], uo.up(gp))
    ub = torch.empty((Z // 2, Y // 2, X // 2, C), dtype=torch.int16, device=dev)
    _call(ctx, "tomgpu_unet_upsample_bwd_dev", _p(ta), cs, off, C, dims, _p(ub))
    ctx.synchronize()
    _bf_close(_from_bf(ub), uo.up_bwd(a[..., off:off + C]))
    # channel sums of a slice
    s = torch.zeros(C, device=dev)
    _call(ctx, "tomgpu_unet_channel_sum_dev", _p(ta), cs, off, C, n, _p(s))
    ctx.synchronize()
    _close(s.cpu().numpy(), a[..., off:off + C].reshape(-1, C).sum(axis=0))


def test_unet_forward_and_gradients_vs_oracle(gpu):
    import torch
    from tom_b200 import unet
    ctx = gpu.default_context()
    rng = np.random.default_rng(11)
    n_bins = 7
    po = uo.init_params(n_bins, seed=4)
    for k in po:
        if k.startswith("b_") or k == "b0":
            po[k] = (np.abs(rng.standard_normal(po[k].shape)) * 0.05).astype(np.float32)
    pp = {k: v for k, v in po.items() if k not in ("wh", "bh")}
    pp["head"] = np.concatenate([po["wh"], po["bh"]]).astype(np.float32)
    net = unet.UNetProposer(n_bins, ctx, params=pp)
    Z, Y, X = 16, 72, 40
    vol = rng.standard_normal((Z, Y, X)).astype(np.float32)
    tv = torch.from_numpy(vol).to(net.dev)
    logit = net.forward(tv, train=True)
    a = uo.forward(po, vol, bf=True)
    got = logit.cpu().numpy()
    assert np.linalg.norm(got - a["logit"]) <= 2e-2 * np.linalg.norm(a["logit"])
    # the backward pass on the GPU's own activations: a ReLU output that FP32
    # and FP64 sums put on the two sides of zero (about 1e-3 of the features
    # here) would otherwise pass or block a full-size gradient
    ag = {k: _from_bf(v) for k, v in net.a.items()}
    ag["e1"], ag["e2"] = ag["D1"][..., 32:], ag["D2"][..., 64:]
    for k in ("e1a", "p1", "e2a", "e3a", "e3", "d2a", "d1a", "f"):
        assert np.linalg.norm(ag[k] - a[k]) <= 2e-2 * np.linalg.norm(a[k]), k
    gl = (rng.standard_normal((Z, Y, X)) * 0.1).astype(np.float32)
    idx = np.array([5, 700, 2222, 40000], np.int64)
    ti = torch.from_numpy(idx).to(net.dev)
    fg, ol = net.orient_logits(ti)
    g_ol = torch.from_numpy(rng.standard_normal((n_bins, len(idx))).astype(np.float32)).to(net.dev)
    net.zero_grad()
    net.backward(torch.from_numpy(gl).to(net.dev), (ti, fg, g_ol))
    ctx.synchronize()
    # the oracle: the orientation head's gradient on the gathered features
    Wo = po["Wo"].astype(np.float64)
    extra = np.zeros((Z * Y * X, 16))
    extra[idx] = (Wo.T @ g_ol.cpu().numpy().astype(np.float64)).T
    gr = uo.backward(po, vol, ag, gl, extra.reshape(Z, Y, X, 16), bf=True)
    gr["head"] = np.concatenate([gr["wh"], gr["bh"]])
    errs = {}
    for k, v in net.g.items():
        if k in ("Wo", "bo"):
            continue
        ref = gr[k].reshape(v.shape)
        errs[k] = float(np.linalg.norm(v.cpu().numpy() - ref) / max(np.linalg.norm(ref), 1e-30))
    print("relative gradient errors", errs)
    assert all(e <= 2e-2 for e in errs.values()), errs


def test_unet_training_lowers_the_loss(gpu):
    import torch
    from tom_b200 import unet
    ctx = gpu.default_context()
    rng = np.random.default_rng(2)
    net = unet.UNetProposer(4, ctx, seed=3)
    Z, Y, X = 16, 72, 40
    vol = rng.standard_normal((Z, Y, X)).astype(np.float32)
    tgt = np.zeros((Z, Y, X), np.float32)
    pos = np.column_stack([rng.integers(3, X - 3, 6), rng.integers(3, Y - 3, 6), rng.integers(3, Z - 3, 6)])
    for x, y, z in pos:
        vol[z - 2:z + 3, y - 2:y + 3, x - 2:x + 3] += 2.0
        tgt[z, y, x] = 1.0
    tv, tt = torch.from_numpy(vol).to(net.dev), torch.from_numpy(tgt).to(net.dev)
    idx = torch.from_numpy((pos[:, 0] + X * (pos[:, 1] + Y * pos[:, 2])).astype(np.int64)).to(net.dev)
    bins = torch.from_numpy((np.arange(6) % 4).astype(np.int32)).to(net.dev)
    first = net.train_step(tv, tt, idx, bins, pos_weight=20.0, lr=3e-3)
    for _ in range(60):
        last = net.train_step(tv, tt, idx, bins, pos_weight=20.0, lr=3e-3)
    assert last[0] < 0.5 * first[0] and last[1] < first[1]


def test_normalise_bin_and_slabbed_inference(gpu):
    import torch
    from tom_b200 import unet
    ctx = gpu.default_context()
    net = unet.UNetProposer(5, ctx, seed=8)
    rng = np.random.default_rng(4)
    vol = torch.from_numpy(rng.standard_normal((56, 72, 40)).astype(np.float32)).to(net.dev)
    v = unet.normalise(vol, ctx)
    m = vol.double().mean().item()
    s = vol.double().std(unbiased=False).item()
    assert np.allclose(v.cpu().numpy(), (vol.cpu().numpy() - m) / s, atol=1e-5)
    b = unet.bin2(vol, ctx)
    ref = vol.cpu().numpy().astype(np.float64).reshape(28, 2, 36, 2, 20, 2).mean(axis=(1, 3, 5))
    assert np.allclose(b.cpu().numpy(), ref, rtol=1e-6, atol=1e-6)
    whole, fw = unet.infer(net, v, slab=56, halo=24)
    slabbed, fs = unet.infer(net, v, slab=16, halo=24)
    ctx.synchronize()
    assert torch.equal(whole, slabbed) and torch.equal(fw, fs)
