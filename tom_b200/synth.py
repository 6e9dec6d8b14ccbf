"""Seeded synthetic tomograms for the template-matching workloads.

The reference names no public dataset; its phantom helpers
(av3_new/tom_build_phantom_volume.m, av3_new/tom_av3_build_phantom_particle.m,
Oscar3/matlabPicker/noise/tom_os3_generateNoise.m:66) paste rotated copies of
a template into noise at a given SNR and apply a missing wedge.  This module
does the same with an analytic phantom: a sum of isotropic Gaussian blobs, so a
rotated copy is the same blobs at rotated centres (no interpolation).

Conventions: arrays are [x, y, z] float32 in Fortran order (x fastest).  A copy
"at Euler e" is what tom_rotate(template, e) produces: output voxel x samples
the template at c + M (x - c) with M the rot3d matrix, so blob b of the
template sits at M^T b in the copy.
"""
from __future__ import annotations

import numpy as np


def rot3d_matrix(euler_deg):
    """3x3 M with r = c + M (x - c) for tom_rotatec's ZXZ convention (double)."""
    ph, ps, th = np.deg2rad(np.asarray(euler_deg, np.float64))
    cf, sf, cp, sp, ct, st = np.cos(ph), np.sin(ph), np.cos(ps), np.sin(ps), np.cos(th), np.sin(th)
    rm00 = cp * cf - ct * sp * sf
    rm10 = sp * cf + ct * cp * sf
    rm20 = st * sf
    rm01 = -cp * sf - ct * sp * cf
    rm11 = -sp * sf + ct * cp * cf
    rm21 = st * cf
    rm02 = st * sp
    rm12 = -st * cp
    rm22 = ct
    return np.array([[rm00, rm10, rm20], [rm01, rm11, rm21], [rm02, rm12, rm22]])


class BlobPhantom:
    """k Gaussian blobs with centres inside radius rho around the box centre."""

    def __init__(self, rng, n_blobs, rho, sigma=(2.0, 4.0), amp=(1.0, 3.0)):
        c = []
        while len(c) < n_blobs:
            p = rng.uniform(-rho, rho, 3)
            if np.linalg.norm(p) <= rho:
                c.append(p)
        self.centers = np.array(c)
        self.sigmas = rng.uniform(*sigma, n_blobs)
        self.amps = rng.uniform(*amp, n_blobs)

    def render(self, shape, origin, euler=None, out=None, radius=None):
        """Add the phantom (optionally at Euler `euler`) centred at `origin`
        (0-based voxel coordinates) into `out` (or a new zero array)."""
        shape = tuple(int(s) for s in shape)
        if out is None:
            out = np.zeros(shape, np.float32, order="F")
        cen = self.centers if euler is None else self.centers @ rot3d_matrix(euler)  # rows: M^T b
        ext = int(np.ceil(np.abs(self.centers).max() + 3 * self.sigmas.max())) + 1
        lo = [max(0, int(np.floor(o)) - ext) for o in origin]
        hi = [min(s, int(np.ceil(o)) + ext + 1) for o, s in zip(origin, shape)]
        if any(h <= l for l, h in zip(lo, hi)):
            return out
        gx, gy, gz = [np.arange(l, h, dtype=np.float64) for l, h in zip(lo, hi)]
        X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
        acc = np.zeros(X.shape)
        for b, s, a in zip(cen, self.sigmas, self.amps):
            d2 = (X - origin[0] - b[0]) ** 2 + (Y - origin[1] - b[1]) ** 2 + (Z - origin[2] - b[2]) ** 2
            acc += a * np.exp(-d2 / (2 * s * s))
        if radius is not None:
            r2 = (X - origin[0]) ** 2 + (Y - origin[1]) ** 2 + (Z - origin[2]) ** 2
            acc[r2 > radius * radius] = 0
        out[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] += acc.astype(np.float32)
        return out

    def template(self, T):
        """The template box T^3 with the phantom at its rotation centre ceil(T/2)."""
        c = [np.ceil(t / 2) for t in (T, T, T)]
        return self.render((T, T, T), c)


def wedge_fourier(vol, max_tilt_deg):
    """Apply a +-max_tilt missing wedge about Y in Fourier space: zero where
    |kx| / |kz| < tan(90 - max_tilt) (tom_wedge(., 90 - max_tilt) on the spectrum)."""
    import scipy.fft as sfft
    n = vol.shape
    f = sfft.rfftn(np.asarray(vol, np.float32), axes=(0, 1, 2)[::-1], workers=-1)
    # rfftn over axes (2,1,0) makes axis 0 (x) the half axis
    kx = np.fft.rfftfreq(n[0])[:, None, None] * n[0]
    kz = np.fft.fftfreq(n[2])[None, None, :] * n[2]
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.abs(kx) / np.abs(kz)
    keep = ~(np.tan(np.deg2rad(90.0 - max_tilt_deg)) > r)
    f *= keep
    return np.asfortranarray(sfft.irfftn(f, s=n[::-1], axes=(2, 1, 0), workers=-1).astype(np.float32))


def place_copies(rng, N, T, n_copies, min_dist=None, max_tries=100000):
    """Seeded non-overlapping centres (0-based) at least T/2 from the borders."""
    min_dist = T if min_dist is None else min_dist
    pos = []
    tries = 0
    while len(pos) < n_copies and tries < max_tries:
        tries += 1
        p = np.array([rng.uniform(T / 2, n - T / 2) for n in N]).round()
        if all(np.linalg.norm(p - q) >= min_dist for q in pos):
            pos.append(p)
    return np.array(pos)


def make_tomogram(N, T, n_copies, n_blobs, rho, snr, max_tilt, seed, euler_pool=None, mask_radius=None,
                  phantom=None):
    """A seeded tomogram of shape N with n_copies of a blob phantom.

    Returns dict(tomo, template, positions (0-based), eulers, euler_index (into
    euler_pool, or -1), phantom).  SNR = var(signal under the mask) / var(noise)
    with unit-variance Gaussian noise (tom_os3_generateNoise.m:66)."""
    rng = np.random.default_rng(seed)
    ph = phantom or BlobPhantom(rng, n_blobs, rho)
    tmpl = ph.template(T)
    pos = place_copies(rng, N, T, n_copies)
    if euler_pool is not None:
        ids = rng.integers(0, len(euler_pool), len(pos))
        eul = np.asarray(euler_pool)[ids]
    else:
        ids = np.full(len(pos), -1)
        eul = np.column_stack([rng.uniform(0, 360, len(pos)), rng.uniform(0, 360, len(pos)),
                               rng.uniform(0, 180, len(pos))])
    sig = np.zeros(N, np.float32, order="F")
    rad = mask_radius if mask_radius is not None else T / 2 - 1
    for p, e in zip(pos, eul):
        ph.render(N, p, e, out=sig, radius=rad)
    # signal variance under the template's mask
    c = np.ceil(T / 2)
    g = np.meshgrid(*[np.arange(T) - c] * 3, indexing="ij")
    m = (g[0] ** 2 + g[1] ** 2 + g[2] ** 2) < rad * rad
    var_s = float(np.var(tmpl[m]))
    scale = np.sqrt(snr / var_s) if var_s > 0 else 1.0
    noise = rng.standard_normal(N, dtype=np.float32)
    tomo = np.asfortranarray(noise) + sig * np.float32(scale)
    if max_tilt is not None and max_tilt < 90:
        tomo = wedge_fourier(tomo, max_tilt)
    return dict(tomo=np.asfortranarray(tomo, np.float32), template=tmpl.astype(np.float32), positions=pos,
                eulers=eul, euler_index=ids, phantom=ph, signal_scale=scale)


def sphere_mask(T, radius):
    """Mask with the os3 convention (1 where distance from floor(T/2) < radius)."""
    c = T // 2
    g = np.meshgrid(*[np.arange(T) - c] * 3, indexing="ij")
    return np.asfortranarray(((g[0] ** 2 + g[1] ** 2 + g[2] ** 2) < radius * radius).astype(np.float32))


# The workloads of the benchmark configurations (shapes, counts, value ranges).
CONFIGS = {
    "exhaustive_128": dict(N=(128, 128, 128), T=32, n_copies=10, n_blobs=6, rho=12, snr=0.1, max_tilt=60,
                           mask_radius=14, angles=((0, 0, 0), (30, 30, 30), (330, 330, 180))),
    # a reduced volume with the 512x512x256 workload's template, for profiler captures
    "profile_256x256x128": dict(N=(256, 256, 128), T=40, n_copies=10, n_blobs=8, rho=16, snr=0.1,
                                max_tilt=55, mask_radius=16, angles=((0, 0, 0), (10, 10, 10), (350, 350, 180))),
    # x edge of the benchmark (the same x-line kernel) on a small y-z plane, for
    # profiler captures at the benchmark's rotation batch
    "profile_512x128x64": dict(N=(512, 128, 64), T=40, n_copies=4, n_blobs=8, rho=16, snr=0.1,
                               max_tilt=55, mask_radius=16, angles=((0, 0, 0), (10, 10, 10), (350, 350, 180))),
    # the y-column (512) and x-line (512) kernels of the benchmark on a thin z slab
    "profile_512x512x48": dict(N=(512, 512, 48), T=40, n_copies=4, n_blobs=8, rho=16, snr=0.1,
                               max_tilt=55, mask_radius=16, angles=((0, 0, 0), (10, 10, 10), (350, 350, 180))),
    # the z edge 256 (the inverse z pass) and x edge 512 on a thin y slab, for profiler captures
    "profile_512x64x256": dict(N=(512, 64, 256), T=40, n_copies=4, n_blobs=8, rho=16, snr=0.1,
                               max_tilt=55, mask_radius=16, angles=((0, 0, 0), (10, 10, 10), (350, 350, 180))),
    "exhaustive_512x512x256": dict(N=(512, 512, 256), T=40, n_copies=40, n_blobs=8, rho=16, snr=0.1,
                                   max_tilt=55, mask_radius=16, angles=((0, 0, 0), (10, 10, 10), (350, 350, 180))),
    # the 928 / 464 kernels on small volumes, for profiler captures
    "profile_928x928x48": dict(N=(928, 928, 48), T=48, n_copies=20, n_blobs=10, rho=20, snr=0.05,
                               max_tilt=60, mask_radius=23, angles=((0, 0, 0), (7, 7, 7), (357, 357, 175))),
    "profile_928x96x464": dict(N=(928, 96, 464), T=48, n_copies=20, n_blobs=10, rho=20, snr=0.05,
                               max_tilt=60, mask_radius=23, angles=((0, 0, 0), (7, 7, 7), (357, 357, 175))),
    # the full-size tomogram with one of its 48^3 species (52 x 52 x 26 = 70,304 triplets)
    "exhaustive_928x928x464": dict(N=(928, 928, 464), T=48, n_copies=200, n_blobs=10, rho=20, snr=0.05,
                                   max_tilt=60, mask_radius=23, angles=((0, 0, 0), (7, 7, 7), (357, 357, 175))),
}


def make_align_particles(n_particles, seed, sizes=(32, 48, 64, 80, 96), snr=0.05, tilt=(45.0, 65.0),
                         search_half=15.0, search_step=3.0, max_shift=4):
    """Subtomogram-alignment workload: each particle a copy of a 6-blob phantom
    (rendered at its box size) at a seeded Euler, shifted by up to max_shift
    voxels, plus Gaussian noise at the given SNR, with its own +-tilt missing
    wedge; the scan covers +-search_half degrees around a seeded start
    orientation near the truth.  Returns a list of job dicts for
    tom_b200.av3_align_batch plus the true Eulers and shifts."""
    rng = np.random.default_rng(seed)
    jobs, truth = [], []
    phantoms, shared = {}, {}
    for p in range(n_particles):
        n = int(rng.choice(sizes))
        if n not in phantoms:
            phantoms[n] = BlobPhantom(np.random.default_rng(seed * 1000 + n), 6, n / 4)
            # one reference, mask and ccf mask per box size, shared by its particles
            # (an alignment run aligns every particle against the same reference)
            shared[n] = (phantoms[n].template(n), sphere_mask(n, n / 2 - 2), sphere_mask(n, max_shift + 1))
        ph = phantoms[n]
        ref, mask, mccf = shared[n]
        # true orientation on the scan grid around a seeded start
        start = np.array([rng.uniform(30, 300), rng.uniform(30, 300), rng.uniform(30, 150)]).round()
        k = rng.integers(-int(search_half // search_step), int(search_half // search_step) + 1, 3)
        true_e = start + k * search_step
        sh = rng.integers(-max_shift, max_shift + 1, 3)
        part = np.zeros((n, n, n), np.float32, order="F")
        c = [np.ceil(n / 2) + d for d in sh]
        ph.render((n, n, n), c, true_e, out=part)
        var_s = float(np.var(ref[ref > 0.05 * ref.max()])) if ref.max() > 0 else 1.0
        part = part * np.float32(np.sqrt(snr / var_s)) + rng.standard_normal((n, n, n)).astype(np.float32)
        a = rng.uniform(*tilt)
        g = np.meshgrid(*[np.arange(-(n // 2), n - n // 2)] * 3, indexing="ij")
        with np.errstate(divide="ignore", invalid="ignore"):
            r = np.abs(g[0]) / np.abs(g[2])
        w = np.ones((n, n, n), np.float32, order="F")
        w[np.tan(np.deg2rad(90 - a)) > r] = 0
        part = np.real(np.fft.ifftn(np.fft.fftn(part) * np.fft.ifftshift(w))).astype(np.float32)
        rngs = [(float(s0 - search_half), float(search_step), float(s0 + search_half)) for s0 in start]
        jobs.append(dict(ref=ref, part=np.asfortranarray(part), mask=mask, mask_ccf=mccf, wedge_ref=w,
                         wedge_part=w, phi=rngs[0], psi=rngs[1], theta=rngs[2]))
        truth.append((true_e, sh))
    return jobs, truth
