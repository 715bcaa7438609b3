"""Seeded synthetic microscopy volumes (phantom, PSF, noisy observation).

No public dataset is named for this path, so seeded synthetic inputs with the
benchmark configurations' shapes and value distributions stand in:

* phantom: spheres with centres uniform in the volume, radii uniform in
  [1.5, 4] voxels and intensities uniform in [200, 1000], added onto a
  background of 10;
* PSF: a separable Gaussian of the same size as the image, centred at n/2
  (the reference shifts kernels by -n/2, src/MaximumLikelihoodDeconvolve.cxx
  :287), normalised to unit sum, optionally mixed with a wide halo Gaussian;
* observation: the phantom circularly convolved with the PSF at image size
  (float64 FFT), then Poisson noise.

All arrays are numpy float32 in (z, y, x) order, x fastest, which is the
reference's memory layout (src/ImageClip.cxx:41-42).
"""
from __future__ import annotations

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def phantom(shape_zyx, n_spheres, r: np.random.Generator, background=10.0,
            radius=(1.5, 4.0), intensity=(200.0, 1000.0)) -> np.ndarray:
    nz, ny, nx = shape_zyx
    vol = np.full(shape_zyx, background, dtype=np.float64)
    cz = r.uniform(0, nz, n_spheres)
    cy = r.uniform(0, ny, n_spheres)
    cx = r.uniform(0, nx, n_spheres)
    rad = r.uniform(radius[0], radius[1], n_spheres)
    amp = r.uniform(intensity[0], intensity[1], n_spheres)
    for z0, y0, x0, rr, a in zip(cz, cy, cx, rad, amp):
        lo = [max(0, int(np.floor(c - rr))) for c in (z0, y0, x0)]
        hi = [min(n, int(np.ceil(c + rr)) + 1) for c, n in zip((z0, y0, x0), shape_zyx)]
        zz, yy, xx = np.meshgrid(np.arange(lo[0], hi[0]), np.arange(lo[1], hi[1]),
                                 np.arange(lo[2], hi[2]), indexing="ij")
        inside = (zz - z0) ** 2 + (yy - y0) ** 2 + (xx - x0) ** 2 <= rr * rr
        vol[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] += a * inside
    return vol.astype(np.float32)


def gaussian_psf(shape_zyx, sigma_xy, sigma_z) -> np.ndarray:
    """Separable Gaussian centred at n/2 on each axis, unit sum (float64)."""
    nz, ny, nx = shape_zyx
    g = []
    for n, s in ((nz, sigma_z), (ny, sigma_xy), (nx, sigma_xy)):
        t = np.arange(n, dtype=np.float64) - n // 2
        g.append(np.exp(-0.5 * (t / s) ** 2))
    psf = g[0][:, None, None] * g[1][None, :, None] * g[2][None, None, :]
    return psf / psf.sum()


def halo_psf(shape_zyx, core=(2.0, 5.0), halo=(6.0, 12.0), halo_weight=0.1,
             scale=1.0) -> np.ndarray:
    """0.9 * G(core) + 0.1 * G(halo), each normalised first; float32."""
    a = gaussian_psf(shape_zyx, core[0] * scale, core[1] * scale)
    b = gaussian_psf(shape_zyx, halo[0] * scale, halo[1] * scale)
    p = (1.0 - halo_weight) * a + halo_weight * b
    return (p / p.sum()).astype(np.float32)


def blur_circular(img, psf) -> np.ndarray:
    """Circular convolution at image size with the PSF centred at n/2."""
    kern = np.fft.ifftshift(psf.astype(np.float64))
    out = np.fft.irfftn(np.fft.rfftn(img.astype(np.float64)) * np.fft.rfftn(kern),
                        s=img.shape)
    return out


def observe(img, psf, r: np.random.Generator) -> np.ndarray:
    b = np.clip(blur_circular(img, psf), 0, None)
    return r.poisson(b).astype(np.float32)


def make_case(shape_zyx, n_spheres, sigma_xy=None, sigma_z=None, seed=0,
              halo=False, psf_scale=1.0):
    """Returns (observed image, PSF, ground-truth phantom) as float32."""
    r = rng(seed)
    truth = phantom(shape_zyx, n_spheres, r)
    if halo:
        psf = halo_psf(shape_zyx, scale=psf_scale)
    else:
        psf = gaussian_psf(shape_zyx, sigma_xy, sigma_z).astype(np.float32)
    obs = observe(truth, psf, r)
    return obs, psf, truth


# Named workloads (image sizes are (z, y, x)).
def cfg0(seed=0):
    """64x64x32 (x,y,z), 40 spheres, sigma_xy 1.5, sigma_z 3.0."""
    return make_case((32, 64, 64), 40, 1.5, 3.0, seed=seed)


def cfg1(seed=1):
    """256x256x64 (x,y,z), 600 spheres, 0.9 G(2,5) + 0.1 G(6,12) PSF."""
    return make_case((64, 256, 256), 600, seed=seed, halo=True)


def cfg2_volume(i: int, seed0: int = 2000):
    """Volume i of the batched workload: x, y uniform in 16*{6..20}, z in
    8*{2..12}, one sphere per 8000 voxels, its own Gaussian PSF (sigma_xy in
    [1.2, 2.5], sigma_z in [2.5, 6])."""
    r = rng(seed0 + i)
    x, y = 16 * int(r.integers(6, 21)), 16 * int(r.integers(6, 21))
    z = 8 * int(r.integers(2, 13))
    n = max(1, (x * y * z) // 8000)
    return make_case((z, y, x), n, float(r.uniform(1.2, 2.5)), float(r.uniform(2.5, 6.0)),
                     seed=seed0 + 10_000 + i)


def cfg3(seed=3):
    """512x512x128 (x,y,z), one sphere per 4000 voxels, the cfg1 halo PSF."""
    return make_case((128, 512, 512), (512 * 512 * 128) // 4000, seed=seed, halo=True)
