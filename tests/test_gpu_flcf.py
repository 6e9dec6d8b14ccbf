"""FLCF matching parity on the GPU against the FP64 oracle.

Tolerance (the parity bar): |cc_gpu - cc_oracle| <= 1e-4 * max|cc_oracle|
over every voxel, and identical angle indices wherever the oracle's best CC
beats its runner-up by more than that tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REL = 1e-4


def _compare(cc, idx, ref_cc, ref_idx, ref_second):
    scale = np.abs(ref_cc).max()
    err = np.abs(cc.astype(np.float64) - ref_cc).max()
    assert err <= REL * scale, f"max |dcc| {err:.3e} > {REL * scale:.3e}"
    sep = (ref_cc - ref_second) > 2 * REL * scale
    assert np.array_equal(idx[sep], ref_idx[sep]), f"{(idx[sep] != ref_idx[sep]).sum()} index mismatches"
    return err / scale


def test_local_stats(gpu, oracle):
    rng = np.random.default_rng(21)
    vol = (rng.standard_normal((64, 48, 40)) * 2 + 5).astype(np.float32)
    T = 16
    t = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    plan = gpu.MatchPlan(vol.shape, t.shape)
    plan.set_template(gpu.to_device(t), gpu.to_device(mask))
    plan.set_volume(gpu.to_device(vol))
    m, s = plan.stats()
    mean, std, _ = oracle.local_stats(vol.astype(np.float64), mask)
    assert np.abs(gpu.from_device(m) - mean).max() < 1e-5 * np.abs(mean).max()
    assert np.abs(gpu.from_device(s) - std).max() < 1e-5 * std.max()


@pytest.mark.parametrize("with_psf", [False, True])
def test_os3_corr_single_map(gpu, oracle, with_psf):
    rng = np.random.default_rng(22)
    vol = rng.standard_normal((64, 64, 32)).astype(np.float32)
    T = 16
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    psf = oracle.tom_wedge((T, T, T), 30).astype(np.float32) if with_psf else None
    # template statistics of the preprocessed template (findTemplate:157,233-234)
    tn, tmean, tstd = oracle.prepare_template(tmpl, mask, psf)
    rot = oracle.rotate(tn.astype(np.float32), (30, 45, 60)) * mask
    if psf is not None:
        rot = oracle.apply_weight_function(rot, psf)
    rot = rot.astype(np.float32)
    st = oracle.FLCF(vol.astype(np.float64), mask)
    ref = st.corr(rot.astype(np.float64), tmean, tstd)
    opts = {"mask": mask, "template": tmpl, "psf": psf}
    got, _ = gpu.tom_os3_corr(vol, rot, opts)
    assert np.abs(got - ref).max() <= REL * np.abs(ref).max()


@pytest.mark.parametrize("with_psf", [False, True])
def test_find_template_small(gpu, oracle, with_psf):
    rng = np.random.default_rng(23)
    N, T = (64, 48, 40), 16
    vol = rng.standard_normal(N).astype(np.float32)
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    psf = oracle.tom_wedge((T, T, T), 30).astype(np.float32) if with_psf else None
    angles = oracle.av3_angle_grid((0, 0, 0), (45, 45, 60), (315, 90, 120))[:37]
    ref_cc, ref_idx, ref_2 = oracle.find_template(vol, tmpl, mask, angles, psf=psf, keep_second=True)
    ccc, ang = gpu.tom_os3_findTemplate(vol, tmpl, angles, mask=mask, psf=psf, batch=5)
    idx = np.where(ang > 0, ang - 1, -1).astype(np.int64)
    _compare(ccc, idx, ref_cc, ref_idx, ref_2)


def test_exhaustive_128_angle_subset(gpu, oracle):
    """The 128^3 / 32^3 exhaustive workload (6 blobs, 10 copies, SNR 0.1, +-60 wedge,
    mask radius 14) on the first 24 angles of its 30-degree grid."""
    from tom_b200 import synth
    cfg = synth.CONFIGS["exhaustive_128"]
    grid = oracle.av3_angle_grid(*cfg["angles"])
    d = synth.make_tomogram(cfg["N"], cfg["T"], cfg["n_copies"], cfg["n_blobs"], cfg["rho"], cfg["snr"],
                            cfg["max_tilt"], seed=100, euler_pool=grid[:24])
    mask = synth.sphere_mask(cfg["T"], cfg["mask_radius"])
    ref_cc, ref_idx, ref_2 = oracle.find_template(d["tomo"], d["template"], mask, grid[:24], keep_second=True)
    ccc, ang = gpu.tom_os3_findTemplate(d["tomo"], d["template"], grid[:24], mask=mask, batch=8)
    idx = np.where(ang > 0, ang - 1, -1).astype(np.int64)
    _compare(ccc, idx, ref_cc, ref_idx, ref_2)


@pytest.mark.parametrize("N", [(928, 48, 40), (64, 464, 40), (64, 48, 464)])
def test_radix29_sizes(gpu, oracle, N):
    """The 928/464 edges of the full-size workload (radix 16/8/4 x 29), each axis in turn."""
    rng = np.random.default_rng(sum(N))
    vol = rng.standard_normal(N).astype(np.float32)
    T = 16
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (90, 90, 90), (90, 90, 90))
    ref_cc, ref_idx, ref_2 = oracle.find_template(vol, tmpl, mask, angles, keep_second=True)
    ccc, ang = gpu.tom_os3_findTemplate(vol, tmpl, angles, mask=mask, batch=3)
    idx = np.where(ang > 0, ang - 1, -1).astype(np.int64)
    _compare(ccc, idx, ref_cc, ref_idx, ref_2)


def test_match_host_reuses_context_state(gpu, oracle):
    """tomgpu_match keeps its plan and device buffers in the context between
    calls with the same sizes: a second call (other template, other angles),
    a call with other sizes and a call after tomgpu_ctx_trim all equal calls
    on fresh contexts."""
    rng = np.random.default_rng(21)
    T = 16
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    vol_a = rng.standard_normal((48, 40, 32)).astype(np.float32)
    vol_b = rng.standard_normal((40, 48, 32)).astype(np.float32)
    t1 = rng.standard_normal((T, T, T)).astype(np.float32)
    t2 = rng.standard_normal((T, T, T)).astype(np.float32)
    grid = oracle.av3_angle_grid((0, 0, 0), (60, 60, 60), (300, 300, 180))
    calls = [(vol_a, t1, grid[:12]), (vol_a, t2, grid[12:30]), (vol_b, t1, grid[:7]), (vol_b, t2, grid[30:41])]
    ctx = gpu.Context(0)
    try:
        for i, (v, t, e) in enumerate(calls):
            if i == 3:
                ctx.check(gpu._lib.lib().tomgpu_ctx_trim(ctx.handle))
            got_cc, got_idx = gpu.match_host(v, t, mask, e, batch=4, ctx=ctx)
            fresh = gpu.Context(0)
            try:
                ref_cc, ref_idx = gpu.match_host(v, t, mask, e, batch=4, ctx=fresh)
            finally:
                fresh.close()
            assert np.array_equal(got_cc, ref_cc), i
            assert np.array_equal(got_idx, ref_idx), i
    finally:
        ctx.close()


def test_default_batch_is_sized_from_free_memory(gpu, oracle):
    """With batch 0 a plan takes the largest of 64 / 32 / 16 rotations whose
    buffers fit in half the free device memory: for a small volume that is
    64 (the plan holds what an explicit batch of 64 holds), and its search
    finds the maxima of a search with batch 8 (the batches group the running
    maximum differently, so near-ties may round apart: the autotune test's
    bars)."""
    import torch
    rng = np.random.default_rng(17)
    T = 16
    vol = rng.standard_normal((48, 40, 32)).astype(np.float32)
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (60, 60, 60), (300, 300, 180))[:70]
    p64 = gpu.MatchPlan(vol.shape, tmpl.shape, batch=64)
    b64 = p64.bytes
    p64.close()
    out = {}
    for batch in (0, 8):
        plan = gpu.MatchPlan(vol.shape, tmpl.shape, batch=batch)
        if batch == 0:
            assert plan.bytes == b64
        plan.set_template(gpu.to_device(tmpl), gpu.to_device(mask))
        plan.set_volume(gpu.to_device(vol))
        cc, idx = plan.new_results()
        plan.run(angles, cc, idx)
        torch.cuda.synchronize()
        out[batch] = gpu.from_device(cc).copy(), gpu.from_device(idx).copy()
        plan.close()
    assert np.abs(out[0][0] - out[8][0]).max() <= 1e-6 * np.abs(out[8][0]).max()
    assert (out[0][1] != out[8][1]).mean() < 1e-3
