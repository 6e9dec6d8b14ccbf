"""The learned proposer's kernels against the FP64 oracle (forward and both
gradients of the dilated convolution, the dense layers, the losses), and its
training on the search's own labels.

Tolerance: FP32 kernels against FP64 sums, |d| <= 1e-4 x the largest value."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _close(got, ref, rel=1e-4):
    assert np.abs(np.asarray(got, np.float64) - ref).max() <= rel * max(np.abs(ref).max(), 1e-12)


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


@pytest.mark.parametrize("ci,co,dil", [(1, 16, 1), (16, 32, 4), (32, 32, 8), (32, 16, 2)])
def test_conv3d_kernels_vs_oracle(gpu, oracle, ci, co, dil):
    import ctypes
    import torch
    from tom_b200 import proposer as pr
    ctx = gpu.default_context()
    dev = f"cuda:{ctx.device}"
    rng = np.random.default_rng(ci * 100 + co + dil)
    Z, Y, X = 11, 13, 18
    x = rng.standard_normal((ci, Z, Y, X)).astype(np.float32)
    w = (rng.standard_normal((co, ci, 27)) * 0.2).astype(np.float32)
    b = rng.standard_normal(co).astype(np.float32)
    g = rng.standard_normal((co, Z, Y, X)).astype(np.float32)
    dims = (ctypes.c_int * 3)(X, Y, Z)
    tx, tw, tb_, tg = _t(x, dev), _t(w, dev), _t(b, dev), _t(g, dev)
    out = torch.empty((co, Z, Y, X), device=dev)
    pr._lib_call(ctx, "tomgpu_cnn_conv3d_fwd_dev", tx.data_ptr(), ci, dims, tw.data_ptr(), tb_.data_ptr(), co, dil, 0,
                 out.data_ptr())
    ref = oracle.cnn_conv3d(x, w, b, dil)
    _close(out.cpu().numpy(), ref)
    gx_ref, gw_ref, gb_ref = oracle.cnn_conv3d_grads(x, w, dil, g)
    gw = torch.zeros_like(tw)
    gb = torch.zeros_like(tb_)
    pr._lib_call(ctx, "tomgpu_cnn_conv3d_bwd_weight_dev", tx.data_ptr(), ci, dims, tg.data_ptr(), co, dil,
                 gw.data_ptr(), gb.data_ptr())
    _close(gw.cpu().numpy(), gw_ref)
    _close(gb.cpu().numpy(), gb_ref)
    if ci in (1, 8, 16, 32, 64):
        gx = torch.empty_like(tx)
        pr._lib_call(ctx, "tomgpu_cnn_conv3d_bwd_data_dev", tg.data_ptr(), co, dims, tw.data_ptr(), ci, dil,
                     gx.data_ptr())
        _close(gx.cpu().numpy(), gx_ref)


def test_dense_and_losses_vs_oracle(gpu, oracle):
    import torch
    from tom_b200 import proposer as pr
    ctx = gpu.default_context()
    dev = f"cuda:{ctx.device}"
    rng = np.random.default_rng(3)
    K, C, P = 40, 32, 77
    W = rng.standard_normal((K, C)).astype(np.float32)
    b = rng.standard_normal(K).astype(np.float32)
    F = rng.standard_normal((C, P)).astype(np.float32)
    g = rng.standard_normal((K, P)).astype(np.float32)
    tW, tb_, tF, tg = _t(W, dev), _t(b, dev), _t(F, dev), _t(g, dev)
    out = torch.empty((K, P), device=dev)
    pr._lib_call(ctx, "tomgpu_cnn_dense_fwd_dev", tW.data_ptr(), tb_.data_ptr(), tF.data_ptr(), K, C, P, 0,
                 out.data_ptr())
    _close(out.cpu().numpy(), W.astype(np.float64) @ F + b[:, None])
    gF = torch.empty_like(tF)
    gW = torch.zeros_like(tW)
    gb = torch.zeros_like(tb_)
    pr._lib_call(ctx, "tomgpu_cnn_dense_bwd_dev", tW.data_ptr(), tF.data_ptr(), tg.data_ptr(), K, C, P,
                 gF.data_ptr(), gW.data_ptr(), gb.data_ptr())
    _close(gF.cpu().numpy(), W.T.astype(np.float64) @ g)
    _close(gW.cpu().numpy(), g.astype(np.float64) @ F.T)
    _close(gb.cpu().numpy(), g.sum(axis=1))
    # losses
    z = rng.standard_normal(500).astype(np.float32)
    y = (rng.random(500) > 0.9).astype(np.float32)
    loss = torch.zeros(1, dtype=torch.float64, device=dev)
    gz = torch.empty(500, device=dev)
    tz, ty = _t(z, dev), _t(y, dev)  # held: the launch is asynchronous
    pr._lib_call(ctx, "tomgpu_cnn_bce_dev", tz.data_ptr(), ty.data_ptr(), 500, 7.0, gz.data_ptr(), loss.data_ptr())
    lref, gref = oracle.cnn_bce(z, y, 7.0)
    assert abs(loss.item() - lref) <= 1e-5 * abs(lref)
    _close(gz.cpu().numpy(), gref)
    lg = rng.standard_normal((K, P)).astype(np.float32)
    lab = rng.integers(0, K, P).astype(np.int32)
    loss.zero_()
    glg = torch.empty((K, P), device=dev)
    tlg, tlab = _t(lg, dev), _t(lab, dev)
    pr._lib_call(ctx, "tomgpu_cnn_softmax_ce_dev", tlg.data_ptr(), tlab.data_ptr(), K, P, glg.data_ptr(),
                 loss.data_ptr())
    lref, gref = oracle.cnn_softmax_ce(lg, lab)
    assert abs(loss.item() - lref) <= 1e-5 * abs(lref)
    _close(glg.cpu().numpy(), gref)


def test_refine_equals_exhaustive(gpu, oracle):
    """The fine search on periodic crops around candidates gives the full
    volume's FLCF at those voxels and angles."""
    from tom_b200 import proposer as pr
    import torch
    rng = np.random.default_rng(4)
    N, T = (64, 48, 40), 16
    vol = rng.standard_normal(N).astype(np.float32)
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    grid = np.column_stack([rng.uniform(0, 360, 40), rng.uniform(0, 360, 40), rng.uniform(5, 175, 40)])
    cc, idx = pr.search(vol, tmpl, mask, grid)
    torch.cuda.synchronize()
    ccn, idn = gpu.from_device(cc), gpu.from_device(idx)
    centres = np.array([[3, 5, 7], [60, 40, 30], [31, 20, 19], [0, 47, 39]])
    sets = [(grid, np.arange(len(grid)))] * len(centres)
    pos, rcc, ridx = pr.refine(vol, tmpl, mask, centres, sets, window=0)
    assert np.array_equal(pos, centres)
    ref = ccn[tuple(centres.T)]
    assert np.abs(rcc - ref).max() <= 1e-5 * np.abs(ccn).max()
    assert np.array_equal(ridx, idn[tuple(centres.T)])


def test_training_reduces_loss(gpu):
    """A few Adam steps of the network on the search's own labels (our kernels
    end to end) lower the centre loss and fit the orientation labels."""
    import torch
    from tom_b200 import proposer as pr
    from tom_b200 import synth
    ctx = gpu.default_context()
    N, T = (64, 64, 64), 16
    coarse = gpu.tom_av3_angle_grid((0, 0, 0), (45, 45, 45), (315, 315, 180))
    d = synth.make_tomogram(N, T, 6, 6, 6, 0.3, 60, seed=11, euler_pool=coarse, mask_radius=T // 2 - 1)
    mask = synth.sphere_mask(T, T // 2 - 1)
    cc, idx = pr.search(d["tomo"], d["template"], mask, coarse, ctx=ctx)
    pos, bins, _ = pr.make_labels(cc, idx, 6, T / 2, coarse, coarse, ctx)
    net = pr.ProposerNet(len(coarse), ctx, seed=3)
    x = torch.from_numpy(np.ascontiguousarray(pr.normalise(gpu.from_device(cc).transpose(2, 1, 0)))).to(net.dev)
    tgt = pr.heat_target(N, pos, net.dev)
    fi = torch.from_numpy(pr.flat_index(pos, N)).to(net.dev)
    tb_ = torch.from_numpy(bins.astype(np.int32)).to(net.dev)
    first = net.train_step(x, tgt, fi, tb_, pos_weight=50.0, lr=1e-3)
    for _ in range(120):
        last = net.train_step(x, tgt, fi, tb_, pos_weight=50.0, lr=1e-3)
    assert np.isfinite(last[0]) and last[0] < 0.5 * first[0]
    assert last[1] < 0.5 * first[1]


def test_pruned_search_recalls_exhaustive_peaks(gpu):
    """The pruned search (coarse sub-grid, its top peaks, the fine triplets
    within a geodesic radius of each candidate's coarse rotation refined on
    crops within +-3 voxels) finds the exhaustive fine search's peaks: every
    exhaustive peak that sits on a particle by position, nearly all with the
    same triplet, on a 128^3 tomogram with 12 particles whose orientations
    lie on the fine grid."""
    from tom_b200 import proposer as pr
    from tom_b200 import synth
    ctx = gpu.default_context()
    N, T, K = (128, 128, 128), 32, 12
    fine = gpu.tom_av3_angle_grid((0, 0, 0), (10, 10, 10), (350, 350, 170))
    coarse = gpu.tom_av3_angle_grid((0, 0, 0), (30, 30, 30), (330, 330, 150))
    d = synth.make_tomogram(N, T, K, 6, 10, 1.0, 60, seed=21, euler_pool=fine, mask_radius=T // 2 - 2)
    mask = synth.sphere_mask(T, T // 2 - 2)
    ccf, idf = pr.search(d["tomo"], d["template"], mask, fine, batch=16, ctx=ctx)
    _, ref_pos, ref_idx = gpu.pick_peaks(ccf, idf, K, T / 2, ctx)
    ref_pos = ref_pos - 1
    # the exhaustive peaks on a particle (within 2 voxels of a placed centre)
    truth = np.asarray(d["positions"], float)
    on = np.linalg.norm(ref_pos[:, None, :] - truth[None], axis=2).min(axis=1) <= 2
    assert on.sum() >= K - 1
    assert np.array_equal(coarse, pr.coarse_grid((0, 0, 0), (10, 10, 10), (350, 350, 170), 3))
    tm = {}
    rpos, rcc, ridx = pr.pruned_search(d["tomo"], d["template"], mask, fine, coarse, 2 * K, 30.0, window=3,
                                       batch=16, ctx=ctx, timings=tm)
    assert tm["candidates_n"] == 2 * K and 0 < tm["triplets_per_candidate"] < len(fine)
    dd = np.linalg.norm(ref_pos[:, None, :].astype(float) - rpos[None].astype(float), axis=2)
    j = np.argmin(dd, axis=1)
    found = dd[np.arange(K), j] <= 2
    same = ridx[j] == ref_idx
    assert found[on].all(), dd.min(axis=1)
    assert (found & same)[on].mean() >= 0.9, (ridx[j], ref_idx)
