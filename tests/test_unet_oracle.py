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
