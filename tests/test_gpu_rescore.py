"""FP64 rescoring of candidate peaks (tomgpu_match_rescore_fp64_dev) against the
oracle's FP64 direct sums, and the FP32 search map against the rescored values."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("with_psf", [False, True])
def test_rescore_matches_direct_fp64(gpu, oracle, with_psf):
    import torch
    rng = np.random.default_rng(41)
    N, T = (64, 48, 40), 16
    vol = (rng.standard_normal(N) + 3.0).astype(np.float32)
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    psf = oracle.tom_wedge((T, T, T), 30).astype(np.float32) if with_psf else None
    angles = oracle.av3_angle_grid((0, 0, 0), (60, 60, 90), (300, 60, 90))
    plan = gpu.MatchPlan(N, (T, T, T))
    vd = gpu.to_device(vol)
    plan.set_template(gpu.to_device(tmpl), gpu.to_device(mask), gpu.to_device(psf) if with_psf else None)
    plan.set_volume(vd)
    cc, idx = plan.new_results()
    plan.run(angles, cc, idx)
    torch.cuda.synchronize()
    vals, pos, aidx = gpu.pick_peaks(cc, idx, 12, 4.0)
    got = plan.rescore_fp64(vd, angles[aidx], pos)
    t, tmean, tstd = oracle.prepare_template(tmpl, mask, psf)
    for k in range(12):
        tr = oracle.rotate(t.astype(np.float32), angles[aidx[k]]).astype(np.float64) * mask
        if psf is not None:
            tr = oracle.apply_weight_function(tr, psf)
        ref = oracle.flcf_direct_at(vol, tr, mask, tmean, tstd, [pos[k] - 1])[0]
        # both FP64; the float template normalisation may round a few voxels differently
        assert abs(got[k] - ref) <= 2e-8 * max(1.0, abs(ref)), (k, got[k], ref)
    # the FP32 spectral search agrees with the FP64 rescoring at its own peaks
    assert np.abs(vals - got).max() <= 1e-4 * np.abs(got).max()
    plan.close()
