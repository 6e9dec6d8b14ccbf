"""Host-side paths on a device: a checkpointed device search that is
interrupted between chunks and resumed (tools/tom_os3_secureSave.m's
save-and-resume of tom_os3_findTemplate's job lists), the zero-std template
rule (search/tom_os3_corr.m:169-176: CC 0 where the denominator vanishes, so
bestPeak keeps the first angle, search/tom_os3_bestPeak.m:94-96), and the
ordering of a context's stream switch."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _job(oracle, N=(64, 48, 40), T=16, n=23, seed=41):
    rng = np.random.default_rng(seed)
    vol = rng.standard_normal(N).astype(np.float32)
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), T // 2 - 1).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (30, 30, 30), (330, 330, 180))[:n].astype(np.float32)
    return vol, tmpl, mask, angles


def _plan(gpu, vol, tmpl, mask, batch=4, ctx=None):
    plan = gpu.MatchPlan(vol.shape, tmpl.shape, batch=batch, ctx=ctx)
    plan.set_template(gpu.to_device(tmpl), gpu.to_device(mask))
    plan.set_volume(gpu.to_device(vol))
    return plan


def test_checkpointed_device_search_resumes_bit_identical(gpu, oracle, tmp_path):
    """A device search (MatchPlanEngine) that fails on the host after its third
    chunk resumes from the checkpoint of the chunks before and ends equal, bit
    for bit, to the uninterrupted search with the same chunking; the
    end-to-end find_template_checkpointed gives the same volumes and meets
    the oracle's parity bar."""
    from tom_b200.checkpoint import MatchPlanEngine, SearchCheckpoint, find_template_checkpointed, run_checkpointed
    vol, tmpl, mask, angles = _job(oracle)
    chunk = 5

    class Failing(MatchPlanEngine):
        def __init__(self, plan, fail_after):
            super().__init__(plan)
            self.left = fail_after

        def run(self, eulers, index_offset):
            if self.left == 0:
                raise RuntimeError("host failure between chunks")
            self.left -= 1
            super().run(eulers, index_offset)

    plan = _plan(gpu, vol, tmpl, mask)
    try:
        ref_cc, ref_idx, info = run_checkpointed(MatchPlanEngine(plan), angles, chunk, str(tmp_path / "ref.npz"))
        assert info["chunks_run"] == 5 and info["resumed_at"] == 0
        path = str(tmp_path / "ck.npz")
        with pytest.raises(RuntimeError, match="host failure"):
            run_checkpointed(Failing(plan, 3), angles, chunk, path)
        meta, _, _ = SearchCheckpoint(path).load()
        assert meta["cursor"] == 3 * chunk
    finally:
        plan.close()
    plan = _plan(gpu, vol, tmpl, mask)  # a new plan, as after a restart
    try:
        cc, idx, info = run_checkpointed(MatchPlanEngine(plan), angles, chunk, path)
    finally:
        plan.close()
    assert info["resumed_at"] == 3 * chunk and info["chunks_run"] == 2
    assert np.array_equal(cc, ref_cc) and np.array_equal(idx, ref_idx)
    ccc, ang, info = find_template_checkpointed(vol, tmpl, angles, str(tmp_path / "e2e.npz"), mask=mask, batch=4,
                                                chunk=chunk)
    assert info["chunks_run"] == 5
    assert np.array_equal(ccc, ref_cc) and np.array_equal(ang, np.where(ref_idx >= 0, ref_idx + 1, -1000))
    o_cc, o_idx, o_2 = oracle.find_template(vol, tmpl, mask, angles, keep_second=True)
    scale = np.abs(o_cc).max()
    assert np.abs(ccc - o_cc).max() <= 1e-4 * scale
    sep = (o_cc - o_2) > 2e-4 * scale
    assert np.array_equal(ref_idx[sep], o_idx[sep])


@pytest.mark.parametrize("N", [(128, 128, 128), (45, 38, 27)])
def test_zero_std_template_gives_cc_zero_and_the_first_angle(gpu, oracle, N):
    """A constant template has zero std under the mask: every CC is 0 and the
    first angle is kept everywhere, on the dedicated kernels (128^3) and on the
    run-time ones (odd edges), as the oracle's rule."""
    T = 16
    vol = np.random.default_rng(3).standard_normal(N).astype(np.float32)
    tmpl = np.full((T, T, T), 2.5, np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (30, 30, 30), (330, 330, 180))[:11]
    ccc, ang = gpu.tom_os3_findTemplate(vol, tmpl, angles, mask=mask, batch=4)
    ref_cc, ref_idx = oracle.find_template(vol, tmpl, mask, angles[:3])
    assert (ref_cc == 0).all() and (ref_idx == 0).all()
    assert (ccc == 0).all() and (ang == 1).all()


def test_stream_switch_waits_for_queued_work(gpu, oracle):
    """A search queued on stream A, then the context switched to stream B and
    a peak search of the result volume issued there at once: B waits for A's
    queued work on the device, so the peak equals the peak of the finished
    search."""
    import torch
    from tom_b200 import _lib
    from tom_b200.tom import _cdims, _tptr
    N, T = (512, 512, 128), 32
    rng = np.random.default_rng(8)
    vol = rng.standard_normal(N).astype(np.float32)
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 14).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (10, 10, 10), (350, 350, 180))[:128]
    ctx = gpu.Context(0)
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    try:
        ctx.set_stream(sa.cuda_stream)
        plan = _plan(gpu, vol, tmpl, mask, batch=32, ctx=ctx)
        cc, idx = plan.new_results()
        ctx.synchronize()
        torch.cuda.synchronize()
        plan.run(angles, cc, idx)           # queued on A
        ctx.set_stream(sb.cuda_stream)      # B waits for A's queued work
        val = ctypes.c_float()
        pos = (ctypes.c_int * 3)()
        ctx.check(_lib.lib().tomgpu_peak_dev(ctx.handle, _tptr(cc), _cdims(N), ctypes.byref(val), pos))
        torch.cuda.synchronize()
        final = gpu.from_device(cc)
        rv, rp = oracle.find_max(np.asfortranarray(final))
        assert float(val.value) == float(rv) and tuple(pos[:]) == tuple(p + 1 for p in rp)
        assert float(val.value) > -1000
        plan.close()
    finally:
        ctx.close()
