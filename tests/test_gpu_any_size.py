"""Tomograms and templates of any size, as MATLAB's fftn takes them
(search/tom_os3_corr.m:151-153, search/tom_os3_findTemplate.m:245,
Filtrans/tom_fourier.m:44-50): odd edges, edges with prime factors 7, 11 and
13 (mixed radix), edges with other prime factors (Bluestein), and 1024.

Parity bar as in test_gpu_flcf.py: |cc_gpu - cc_oracle| <= 1e-4 max|cc_oracle|
over every voxel, identical angle indices wherever the oracle's best CC beats
its runner-up by more than twice that; FFTs within 1e-11 (FP64) and 2e-6
(FP32) of the maximum."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REL = 1e-4


def _compare(cc, idx, ref_cc, ref_idx, ref_second):
    scale = np.abs(ref_cc).max()
    err = np.abs(cc.astype(np.float64) - ref_cc).max()
    assert err <= REL * scale, f"max |dcc| {err:.3e} > {REL * scale:.3e}"
    sep = (ref_cc - ref_second) > 2 * REL * scale
    assert sep.mean() > 0.5
    assert np.array_equal(idx[sep], ref_idx[sep]), f"{(idx[sep] != ref_idx[sep]).sum()} index mismatches"


def _search(gpu, oracle, N, T, seed, n_angles=7, psf=False):
    rng = np.random.default_rng(seed)
    T = (T, T, T) if np.isscalar(T) else tuple(T)
    vol = rng.standard_normal(N).astype(np.float32)
    tmpl = rng.standard_normal(T).astype(np.float32)
    mask = oracle.sphere_mask(T, min(T) // 2 - 1).astype(np.float32)
    w = oracle.tom_wedge(T, 30).astype(np.float32) if psf else None
    angles = oracle.av3_angle_grid((0, 0, 0), (45, 45, 60), (315, 90, 120))[:n_angles]
    ref_cc, ref_idx, ref_2 = oracle.find_template(vol, tmpl, mask, angles, psf=w, keep_second=True)
    ccc, ang = gpu.tom_os3_findTemplate(vol, tmpl, angles, mask=mask, psf=w, batch=3)
    idx = np.where(ang > 0, ang - 1, -1).astype(np.int64)
    _compare(ccc, idx, ref_cc, ref_idx, ref_2)


@pytest.mark.parametrize("N,T", [((100, 90, 77), 17), ((100, 90, 77), 33), ((77, 64, 45), (17, 20, 13)),
                                 ((37, 41, 29), 9), ((121, 26, 39), (11, 13, 7))])
def test_find_template_any_size(gpu, oracle, N, T):
    """Odd and prime edges on every axis (77 = 7 x 11, 37/41/29/17 through
    Bluestein), odd and non-cubic templates."""
    _search(gpu, oracle, N, T, seed=sum(N))


def test_find_template_any_size_with_psf(gpu, oracle):
    """The weight filter of an odd template (tom_apply_weight_function on 17^3)."""
    _search(gpu, oracle, (60, 45, 33), 17, seed=5, psf=True)


def test_find_template_1024(gpu, oracle):
    """A 1024 x 1024 x 64 tomogram (the 1024 edge runs compiled kernels), the
    whole map against the oracle."""
    _search(gpu, oracle, (1024, 1024, 64), 16, seed=1024, n_angles=3)


def test_os3_corr_single_map_odd(gpu, oracle):
    """tom_os3_corr's single map (the c2r map kernel at an odd x edge)."""
    rng = np.random.default_rng(31)
    vol = rng.standard_normal((45, 38, 27)).astype(np.float32)
    T = 13
    tmpl = rng.standard_normal((T, T, T)).astype(np.float32)
    mask = oracle.sphere_mask((T, T, T), 5).astype(np.float32)
    tn, tmean, tstd = oracle.prepare_template(tmpl, mask, None)
    rot = (oracle.rotate(tn.astype(np.float32), (30, 45, 60)) * mask).astype(np.float32)
    ref = oracle.FLCF(vol.astype(np.float64), mask).corr(rot.astype(np.float64), tmean, tstd)
    got, _ = gpu.tom_os3_corr(vol, rot, {"mask": mask, "template": tmpl, "psf": None})
    assert np.abs(got - ref).max() <= REL * np.abs(ref).max()


@pytest.mark.parametrize("L", [1, 2, 3, 5, 7, 9, 11, 13, 17, 22, 29, 33, 37, 77, 90, 100, 121, 127, 169, 200,
                               300, 720, 1000, 1024, 2003])
def test_fft_any_length(gpu, L):
    rng = np.random.default_rng(L)
    for shape in [(L, 8, 6), (6, L, 8), (8, 6, L)]:
        a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        f = gpu.tom_fourier(a)
        ref = np.fft.fftn(a)
        assert np.abs(f - ref).max() <= 1e-11 * np.abs(ref).max(), shape
        b = gpu.tom_ifourier(f)
        assert np.abs(b - a).max() <= 1e-11 * np.abs(a).max(), shape


@pytest.mark.parametrize("shape", [(33, 17, 25), (100, 90, 77), (127, 3, 2), (1, 40, 9)])
@pytest.mark.parametrize("prec", [32, 64])
def test_fft_r2c_c2r_any_size(gpu, shape, prec):
    import torch
    from tom_b200 import _lib
    from tom_b200.tom import _cdims, _tptr
    ctx = gpu.default_context()
    rng = np.random.default_rng(sum(shape))
    a = rng.standard_normal(shape)
    dt = torch.float32 if prec == 32 else torch.float64
    x = torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).to("cuda", dt)
    nh = shape[0] // 2 + 1
    half = torch.empty((shape[2], shape[1], nh, 2), dtype=dt, device="cuda")
    ctx.check(_lib.lib().tomgpu_fft3d_r2c_dev(ctx.handle, _tptr(x), _tptr(half), _cdims(shape), prec))
    torch.cuda.synchronize()
    got = torch.view_as_complex(half).cpu().numpy().transpose(2, 1, 0)
    ref = np.fft.rfftn(a, axes=(2, 1, 0))
    tol = 2e-6 if prec == 32 else 1e-13
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
    back = torch.empty_like(x)
    ctx.check(_lib.lib().tomgpu_fft3d_c2r_dev(ctx.handle, _tptr(half), _tptr(back), _cdims(shape), prec))
    torch.cuda.synchronize()
    assert np.abs(back.cpu().numpy().transpose(2, 1, 0) - a).max() <= tol * 10 * np.abs(a).max()


def test_edges_beyond_the_line_limits(gpu, oracle):
    """Edges the line engines cannot hold in one block are refused before any
    work: a prime edge above 3528 (Bluestein would need a 7290-point line) and
    a smooth edge above 7150."""
    L = gpu._lib
    T = (4, 4, 4)
    for shape in [(3637, 8, 8), (8, 8000, 8)]:
        with pytest.raises(gpu.TomGpuError) as e:
            gpu.MatchPlan(shape, T, batch=2)
        assert e.value.status == L.TOMGPU_ERR_UNSUPPORTED, shape
