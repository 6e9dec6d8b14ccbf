"""The U-Net oracle's hand-written backward pass against central differences
(FP64, no rounding), and its BF16 rounding helper.  CPU only."""
import numpy as np

import unet_oracle as uo


def test_bf16_rounding_is_nearest_even():
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties to the even (1.0)
    assert uo.bf16(np.float32(1 + 2 ** -8)) == 1.0
    assert uo.bf16(np.float32(1 + 3 * 2 ** -8)) == 1 + 2 ** -6
    assert uo.bf16(np.float32(-2.7)) == -2.703125
    x = np.random.default_rng(0).standard_normal(1000).astype(np.float32)
    r = uo.bf16(x)
    assert np.all(np.abs(r - x) <= 2 ** -8 * np.abs(x) + 1e-30)


def _loss(p, vol, wl, wf, idx):
    a = uo.forward(p, vol)
    return float((a["logit"] * wl).sum() + (a["f"].reshape(-1, 16)[idx] * wf).sum()), a


def test_backward_matches_central_differences():
    rng = np.random.default_rng(3)
    p = uo.init_params(5, seed=2)
    # small positive biases keep most ReLUs active, so the check sees every layer
    for k in p:
        if k.startswith("b_") or k == "b0":
            p[k] = (np.abs(rng.standard_normal(p[k].shape)) * 0.1).astype(np.float32)
    p = {k: v.astype(np.float64) for k, v in p.items()}
    Z, Y, X = 8, 8, 8
    vol = rng.standard_normal((Z, Y, X))
    wl = rng.standard_normal((Z, Y, X))
    idx = np.array([3, 77, 300])
    wf = rng.standard_normal((3, 16))
    _, a = _loss(p, vol, wl, wf, idx)
    extra = np.zeros((Z * Y * X, 16))
    extra[idx] = wf
    gr = uo.backward(p, vol, a, wl, extra.reshape(Z, Y, X, 16))
    eps = 1e-6
    for k in ["w0", "b0"] + [f"{w}_{n}" for n, _, _ in uo.CONVS for w in ("w", "b")]:
        flat = p[k].reshape(-1)
        for j in rng.choice(flat.size, size=min(4, flat.size), replace=False):
            old = flat[j]
            flat[j] = old + eps
            lp, _ = _loss(p, vol, wl, wf, idx)
            flat[j] = old - eps
            lm, _ = _loss(p, vol, wl, wf, idx)
            flat[j] = old
            num = (lp - lm) / (2 * eps)
            ana = gr[k].reshape(-1)[j]
            assert abs(num - ana) <= 1e-5 * max(1.0, abs(num)), (k, j, num, ana)
    gh = np.concatenate([gr["wh"], gr["bh"]])
    assert np.allclose(gh[:16], np.einsum("zyx,zyxc->c", wl, a["f"]))
    assert np.isclose(gh[16], wl.sum())


def test_network_definition_matches_the_oracle():
    from tom_b200 import unet
    assert tuple(unet.CONVS) == tuple(uo.CONVS)
    p = unet.init_params(11, seed=0)
    for name, ci, co in unet.CONVS:
        assert p["w_" + name].shape == (co, ci, 27) and p["b_" + name].shape == (co,)
    assert p["w0"].shape == (16, 1, 27) and p["head"].shape == (17,) and p["head"][16] == -4.0
    assert p["Wo"].shape == (11, 16) and p["bo"].shape == (11,)
    # 2 x multiply-adds per full-resolution voxel: the first layer, the head,
    # and each convolution at its level (1/8 per pooling)
    macs = 27 * 16 + 16 + sum(27 * ci * co / {"e1b": 1, "d1a": 1, "d1b": 1, "e3a": 64, "e3b": 64}.get(n, 8)
                             for n, ci, co in uo.CONVS)
    assert unet.UNetProposer.flops_per_voxel(None) == 2 * macs == 113216


def test_ball_targets():
    from tom_b200 import unet
    t = unet.ball_target((20, 24, 28), [[5, 6, 7], [0, 23, 19]], 3.0, "cpu").numpy()
    assert t.shape == (20, 24, 28)
    per_ball = sum(1 for dz in range(-3, 4) for dy in range(-3, 4) for dx in range(-3, 4)
                   if dx * dx + dy * dy + dz * dz <= 9)
    assert per_ball == 123 and t.sum() == 2 * per_ball
    # positions are [x, y, z]; the second ball wraps around the x and y faces
    assert t[7, 6, 5] == 1 and t[19, 23, 0] == 1 and t[19, 0, 27] == 1 and t[19, 20, 0] == 1


def test_binned_positions_map_to_their_block_centres():
    from tom_b200 import unet
    p = unet.unbin_positions([[0, 0, 0], [3, 5, 231], [463, 463, 231]], 2, (928, 928, 463))
    assert p.tolist() == [[1, 1, 1], [7, 11, 462], [927, 927, 462]]
    assert unet.unbin_positions([[4, 5, 6]], 1, (8, 8, 8)).tolist() == [[4, 5, 6]]
