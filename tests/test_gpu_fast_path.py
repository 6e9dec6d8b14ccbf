"""The register-resident hot kernels (power-of-two sizes and the 928 / 464
edges) against the generic kernels and against FP64 direct sums at sampled
voxels, at the benchmark sizes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REL = 1e-4


def _run(gpu, vol, tmpl, mask, angles, generic, batch):
    import torch
    plan = gpu.MatchPlan(vol.shape, tmpl.shape, batch=batch, generic=generic)
    plan.set_template(gpu.to_device(tmpl), gpu.to_device(mask))
    plan.set_volume(gpu.to_device(vol))
    cc, idx = plan.new_results()
    plan.run(angles, cc, idx)
    torch.cuda.synchronize()
    out = gpu.from_device(cc).copy(), gpu.from_device(idx).copy()
    plan.close()
    return out


@pytest.mark.parametrize("workload,n_ang", [("exhaustive_128", 24), ("profile_256x256x128", 12),
                                            ("exhaustive_512x512x256", 10), ("exhaustive_928x928x464", 6)])
def test_fast_equals_generic_and_direct_sums(gpu, oracle, workload, n_ang):
    from tom_b200 import synth
    cfg = synth.CONFIGS[workload]
    grid = oracle.av3_angle_grid(*cfg["angles"])
    sel = np.linspace(0, len(grid) - 1, n_ang).astype(int)
    d = synth.make_tomogram(cfg["N"], cfg["T"], cfg["n_copies"], cfg["n_blobs"], cfg["rho"], cfg["snr"],
                            cfg["max_tilt"], seed=7, euler_pool=grid[sel], mask_radius=cfg["mask_radius"])
    mask = synth.sphere_mask(cfg["T"], cfg["mask_radius"])
    angles = grid[sel]
    fcc, fidx = _run(gpu, d["tomo"], d["template"], mask, angles, False, 4)
    gcc, gidx = _run(gpu, d["tomo"], d["template"], mask, angles, True, 3)
    scale = np.abs(gcc).max()
    assert np.abs(fcc - gcc).max() <= 1e-5 * scale
    rng = np.random.default_rng(8)
    vox = np.vstack([d["positions"].astype(int),
                     np.column_stack([rng.integers(0, n, 40) for n in cfg["N"]])])
    best, ridx, second = oracle.find_template_direct_at(d["tomo"], d["template"], mask, angles, vox)
    got = fcc[tuple(vox.T)]
    assert np.abs(got - best).max() <= REL * np.abs(best).max()
    sep = best - second > 2 * REL * np.abs(best).max()
    assert np.array_equal(fidx[tuple(vox.T)][sep], ridx[sep])
    # planted copies are found at their own orientation
    hits = fidx[tuple(d["positions"].astype(int).T)]
    assert (hits == d["euler_index"]).mean() >= 0.8


@pytest.mark.parametrize("shape", [(928, 928, 48), (64, 64, 464), (928, 48, 464)])
def test_928_464_kernels_equal_generic(gpu, oracle, shape):
    """Each 928 / 464 kernel on its own (the other axes on the generic kernels)."""
    rng = np.random.default_rng(9)
    vol = rng.standard_normal(shape).astype(np.float32)
    T = 48
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 23).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (40, 40, 40), (320, 320, 160))[::97][:5]
    fcc, fidx = _run(gpu, vol, tmpl, mask, angles, False, 3)
    gcc, gidx = _run(gpu, vol, tmpl, mask, angles, True, 2)
    scale = np.abs(gcc).max()
    assert np.abs(fcc - gcc).max() <= 1e-5 * scale
    assert (fidx != gidx).mean() < 1e-3


@pytest.mark.parametrize("ny", [128, 256, 512])
@pytest.mark.parametrize("T", [8, 12, 20, 32, 48, 64])
def test_y_column_kernels_every_template_height(gpu, oracle, ny, T):
    """The y-edge 256 / 512 column kernels sum the template's forward y-DFT
    from its nonzeros, ceil(Ty / 8) terms per residue (the y-edge 128 kernel
    transforms the template column in full): every term count a template
    edge (an FFT length) reaches, against the generic kernels (x and z edges
    on the generic kernels)."""
    rng = np.random.default_rng(11 + T)
    vol = rng.standard_normal((64, ny, 80)).astype(np.float32)
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), T // 2 - 1).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (40, 40, 40), (320, 320, 160))[::89][:5]
    fcc, fidx = _run(gpu, vol, tmpl, mask, angles, False, 3)
    gcc, gidx = _run(gpu, vol, tmpl, mask, angles, True, 2)
    scale = np.abs(gcc).max()
    assert np.abs(fcc - gcc).max() <= 1e-5 * scale
    assert (fidx != gidx).mean() < 1e-3


@pytest.mark.parametrize("nz", [256, 464])
@pytest.mark.parametrize("T", [8, 12, 20, 32, 48, 64])
def test_z_spectrum_kernel_every_template_depth(gpu, oracle, nz, T):
    """The z-edge 256 / 464 template-spectrum kernels sum each line's z-DFT
    from its ceil(Tz / 8) terms per residue: every term count against the
    generic kernels (x and y edges on the generic kernels)."""
    rng = np.random.default_rng(31 + T)
    vol = rng.standard_normal((64, 80, nz)).astype(np.float32)
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), T // 2 - 1).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (40, 40, 40), (320, 320, 160))[::83][:5]
    fcc, fidx = _run(gpu, vol, tmpl, mask, angles, False, 3)
    gcc, gidx = _run(gpu, vol, tmpl, mask, angles, True, 2)
    scale = np.abs(gcc).max()
    assert np.abs(fcc - gcc).max() <= 1e-5 * scale
    assert (fidx != gidx).mean() < 1e-3


def test_autotune_keeps_results(gpu, oracle):
    """The batch autotuner picks a candidate and the plan still finds the same maxima."""
    import torch
    rng = np.random.default_rng(10)
    vol = rng.standard_normal((64, 48, 40)).astype(np.float32)
    T = 16
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (60, 60, 60), (300, 300, 180))[:20]
    ref_cc, ref_idx = _run(gpu, vol, tmpl, mask, angles, False, 4)
    plan = gpu.MatchPlan(vol.shape, tmpl.shape, batch=4)
    plan.set_template(gpu.to_device(tmpl), gpu.to_device(mask))
    plan.set_volume(gpu.to_device(vol))
    best, ms = plan.autotune(angles, (2, 5, 8))
    assert best in (2, 5, 8) and set(ms) == {2, 5, 8}
    cc, idx = plan.new_results()
    plan.run(angles, cc, idx)
    torch.cuda.synchronize()
    assert np.abs(gpu.from_device(cc) - ref_cc).max() <= 1e-6 * np.abs(ref_cc).max()
    assert (gpu.from_device(idx) != ref_idx).mean() < 1e-3
    plan.close()


@pytest.mark.parametrize("shape,batch", [((512, 40, 24), 5), ((512, 64, 32), 16), ((512, 512, 16), 3),
                                         ((928, 40, 24), 5), ((928, 30, 16), 3)])
def test_tma_x_lines_equal_cp_async_x_lines(gpu, oracle, shape, batch):
    """The x-line kernels of the 512 and 928 x edges with TMA tile loads and
    the 512 y-column kernel with its F_I values and twiddles in tensor memory
    (the default, path 0) give the results of the kernels without them
    (path 2: cp.async tiles, shared-memory constants) bit for bit (the same
    arithmetic; a y edge that is not a multiple of the tile's 16 or 8 lines
    exercises the TMA's zero fill), and meet the oracle's parity bar."""
    import torch
    rng = np.random.default_rng(shape[1])
    vol = rng.standard_normal(shape).astype(np.float32)
    T = 16
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (30, 30, 30), (330, 330, 180))[:11]
    out = {}
    for path in (0, 2):
        plan = gpu.MatchPlan(vol.shape, tmpl.shape, batch=batch, path=path)
        plan.set_template(gpu.to_device(tmpl), gpu.to_device(mask))
        plan.set_volume(gpu.to_device(vol))
        cc, idx = plan.new_results()
        plan.run(angles, cc, idx)
        plan.ctx.synchronize()
        torch.cuda.synchronize()
        out[path] = gpu.from_device(cc).copy(), gpu.from_device(idx).copy()
        plan.close()
    assert np.array_equal(out[0][0], out[2][0]) and np.array_equal(out[0][1], out[2][1])
    if shape[1] <= 64:
        ref_cc, ref_idx, ref_2 = oracle.find_template(vol, tmpl, mask, angles, keep_second=True)
        scale = np.abs(ref_cc).max()
        assert np.abs(out[0][0] - ref_cc).max() <= REL * scale
        sep = (ref_cc - ref_2) > 2 * REL * scale
        assert np.array_equal(out[0][1][sep], ref_idx[sep])


@pytest.mark.parametrize("shape", [(48, 40, 256), (64, 64, 256), (512, 24, 256)])
def test_tcgen05_inverse_z_dft(gpu, oracle, shape):
    """The inverse z-DFT of the 256 z edge with its radix-16 stages as tcgen05
    tensor-core contractions (path 3, split TF32 with FP32 accumulation) against
    the FP32 CUDA-core kernel (path 0) and the FP64 oracle's parity bar; the
    device error word stays clear (no MMA wait ran out)."""
    import torch
    rng = np.random.default_rng(shape[0] + shape[1])
    vol = rng.standard_normal(shape).astype(np.float32)
    T = 16
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 7).astype(np.float32)
    angles = oracle.av3_angle_grid((0, 0, 0), (30, 30, 30), (330, 330, 180))[:9]
    out = {}
    for path in (0, 3):
        plan = gpu.MatchPlan(vol.shape, tmpl.shape, batch=4, path=path)
        plan.set_template(gpu.to_device(tmpl), gpu.to_device(mask))
        plan.set_volume(gpu.to_device(vol))
        cc, idx = plan.new_results()
        plan.run(angles, cc, idx)
        plan.ctx.synchronize()
        torch.cuda.synchronize()
        out[path] = gpu.from_device(cc).copy(), gpu.from_device(idx).copy()
        plan.close()
    ref_cc, ref_idx, ref_2 = oracle.find_template(vol, tmpl, mask, angles, keep_second=True)
    scale = np.abs(ref_cc).max()
    assert np.abs(out[3][0] - out[0][0]).max() <= 1e-5 * scale
    assert np.abs(out[3][0] - ref_cc).max() <= REL * scale
    sep = (ref_cc - ref_2) > 2 * REL * scale
    assert np.array_equal(out[3][1][sep], ref_idx[sep])
