"""Error paths of the matching entry points on a device.  Unsupported sizes,
bad arguments and a wrong call order come back as status codes with a message
(the cases the reference gateways end with mexErrMsgTxt), and the context
stays usable afterwards.  Every invalid input here is rejected by the host-side
checks of the library before anything is launched."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(oracle, shape=(48, 40, 32), T=16, seed=3):
    rng = np.random.default_rng(seed)
    vol = rng.standard_normal(shape).astype(np.float32)
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), T // 2 - 1).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (60, 60, 60), (300, 300, 180))[:6]
    return vol, tmpl, mask, angles


def _search(gpu, ctx, vol, tmpl, mask, angles):
    import torch
    plan = gpu.MatchPlan(vol.shape, tmpl.shape, batch=4, ctx=ctx)
    try:
        plan.set_template(gpu.to_device(tmpl), gpu.to_device(mask))
        plan.set_volume(gpu.to_device(vol))
        cc, idx = plan.new_results()
        plan.run(angles, cc, idx)
        torch.cuda.synchronize()
        return gpu.from_device(cc).copy(), gpu.from_device(idx).copy()
    finally:
        plan.close()


def test_unsupported_sizes_and_bad_batch(gpu, oracle):
    L = gpu._lib
    cases = [
        ((3637, 64, 64), (16, 16, 16), 4, L.TOMGPU_ERR_UNSUPPORTED, "not supported"),  # beyond the line limits
        ((32, 32, 32), (48, 48, 48), 4, L.TOMGPU_ERR_UNSUPPORTED, "not supported"),  # template > volume
        ((48, 40, 32), (17, 16, 49), 4, L.TOMGPU_ERR_UNSUPPORTED, "not supported"),  # template > volume in z
        ((48, 40, 32), (16, 16, 16), 5000, L.TOMGPU_ERR_ARG, "batch"),
    ]
    vol, tmpl, mask, angles = _inputs(oracle)
    ctx = gpu.Context(0)
    try:
        for vol_shape, t_shape, batch, status, words in cases:
            with pytest.raises(gpu.TomGpuError) as e:
                gpu.MatchPlan(vol_shape, t_shape, batch=batch, ctx=ctx)
            assert e.value.status == status and words in str(e.value), (vol_shape, t_shape, batch)
        # the same context then runs a search as a fresh one does
        got = _search(gpu, ctx, vol, tmpl, mask, angles)
    finally:
        ctx.close()
    fresh = gpu.Context(0)
    try:
        ref = _search(gpu, fresh, vol, tmpl, mask, angles)
    finally:
        fresh.close()
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


def test_call_order_result_buffers_and_empty_angle_list(gpu, oracle):
    import torch
    L = gpu._lib
    vol, tmpl, mask, angles = _inputs(oracle)
    ctx = gpu.Context(0)
    try:
        plan = gpu.MatchPlan(vol.shape, tmpl.shape, batch=4, ctx=ctx)
        cc, idx = plan.new_results()
        with pytest.raises(gpu.TomGpuError) as e:
            plan.run(angles, cc, idx)  # before the template and the volume
        assert e.value.status == L.TOMGPU_ERR_STATE
        plan.set_template(gpu.to_device(tmpl), gpu.to_device(mask))
        plan.set_volume(gpu.to_device(vol))
        # result buffers off the 8-byte alignment of the x-line kernels' paired accesses
        off = torch.empty(cc.numel() + 1, dtype=torch.float32, device=cc.device)[1:]
        with pytest.raises(gpu.TomGpuError) as e:
            plan.run(angles, off, idx)
        assert e.value.status == L.TOMGPU_ERR_ARG and "aligned" in str(e.value)
        with pytest.raises(gpu.TomGpuError) as e:
            plan.run(angles, cc, idx, index_offset=-1)
        assert e.value.status == L.TOMGPU_ERR_ARG
        # no rotations: the results keep their initial values
        plan.run(np.zeros((0, 3), np.float32), cc, idx)
        torch.cuda.synchronize()
        assert (gpu.from_device(cc) == -1000).all() and (gpu.from_device(idx) == -1).all()
        # and the plan still searches
        plan.run(angles, cc, idx)
        torch.cuda.synchronize()
        got = gpu.from_device(cc).copy(), gpu.from_device(idx).copy()
        plan.close()
    finally:
        ctx.close()
    fresh = gpu.Context(0)
    try:
        ref = _search(gpu, fresh, vol, tmpl, mask, angles)
    finally:
        fresh.close()
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


def test_match_host_errors_and_empty_angle_list(gpu, oracle):
    """tomgpu_match with sizes it cannot run reports them and keeps no state;
    with no rotations it returns the initial values; the next valid call in the
    same context equals one in a fresh context."""
    L = gpu._lib
    vol, tmpl, mask, angles = _inputs(oracle)
    ctx = gpu.Context(0)
    try:
        bad = np.zeros((3637, 8, 8), np.float32)  # an edge beyond the FFT line limits
        with pytest.raises(gpu.TomGpuError) as e:
            gpu.match_host(bad, tmpl, mask, angles, batch=4, ctx=ctx)
        assert e.value.status == L.TOMGPU_ERR_UNSUPPORTED
        cc0, idx0 = gpu.match_host(vol, tmpl, mask, np.zeros((0, 3), np.float32), batch=4, ctx=ctx)
        assert (cc0 == -1000).all() and (idx0 == -1).all()
        got = gpu.match_host(vol, tmpl, mask, angles, batch=4, ctx=ctx)
    finally:
        ctx.close()
    fresh = gpu.Context(0)
    try:
        ref = gpu.match_host(vol, tmpl, mask, angles, batch=4, ctx=fresh)
    finally:
        fresh.close()
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


def test_template_change_after_the_volume(gpu, oracle):
    """The volume's local statistics are made with the mask and its FLCF
    denominators with the template's std.  A new template with the same mask
    keeps the volume (the denominators follow the template): the search equals
    a fresh plan's.  A new mask unsets the volume: a run reports
    TOMGPU_ERR_STATE before launching anything, and with the volume set again
    the search equals a fresh plan's."""
    import torch
    L = gpu._lib
    vol, tmpl, mask, angles = _inputs(oracle)
    tmpl2 = np.random.default_rng(9).standard_normal(tmpl.shape).astype(np.float32)
    mask2 = oracle.sphere_mask(tmpl.shape, tmpl.shape[0] // 2 - 2).astype(np.float32)

    def results(plan, cc, idx):
        plan.init_results(cc, idx)
        plan.run(angles, cc, idx)
        torch.cuda.synchronize()
        return gpu.from_device(cc).copy(), gpu.from_device(idx).copy()

    ctx = gpu.Context(0)
    try:
        plan = gpu.MatchPlan(vol.shape, tmpl.shape, batch=4, ctx=ctx)
        plan.set_template(gpu.to_device(tmpl), gpu.to_device(mask))
        vd = gpu.to_device(vol)
        plan.set_volume(vd)
        cc, idx = plan.new_results()
        plan.set_template(gpu.to_device(tmpl2), gpu.to_device(mask))  # same mask
        same_mask = results(plan, cc, idx)
        plan.set_template(gpu.to_device(tmpl), gpu.to_device(mask2))  # another mask
        with pytest.raises(gpu.TomGpuError) as e:
            plan.run(angles, cc, idx)
        assert e.value.status == L.TOMGPU_ERR_STATE
        plan.set_volume(vd)
        new_mask = results(plan, cc, idx)
        plan.close()
    finally:
        ctx.close()
    fresh = gpu.Context(0)
    try:
        ref1 = _search(gpu, fresh, vol, tmpl2, mask, angles)
        ref2 = _search(gpu, fresh, vol, tmpl, mask2, angles)
    finally:
        fresh.close()
    for got, ref in ((same_mask, ref1), (new_mask, ref2)):
        assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
