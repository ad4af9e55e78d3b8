"""Seeded synthetic fixed/moving pairs for the SyN-CC workloads.

There is no public dataset for this path; every workload uses generated images whose shape,
spacing and intensity statistics follow the benchmark configurations:

* ``blobs_2d``: sum of isotropic Gaussian blobs (sigma U[4,20] px, amplitude U[0.2,1]) plus
  N(0, 0.01) noise (2-D 256^2 workload, CC radius 2).
* ``ellipsoid_phantom_3d``: nested ellipsoids with class intensities 0.1/0.4/0.7/1.0, a smooth
  multiplicative bias 1+b (b a cubic tensor-product spline on 4^3 control values in
  [-0.15, 0.15]), noise sigma 0.02 and a 2-voxel Gaussian blur (3-D 182x218x182 workload).
* ``smooth_field``: i.i.d. N(0,1) per component, Gaussian-smoothed, scaled to a maximum
  displacement norm; the moving image is the fixed image warped (linear) by it.

All randomness comes from ``numpy.random.default_rng(seed)``; the default seeds are
``0x5EED0000 + pair_index``.
"""
from __future__ import annotations

import numpy as np
from scipy import ndimage

SEED_BASE = 0x5EED0000


def smooth_field(shape: tuple, sigma: float, max_norm: float, rng: np.random.Generator) -> np.ndarray:
    """Random smooth displacement (voxel units), shape + (dim,), max ||u|| = max_norm."""
    d = len(shape)
    comps = []
    for _ in range(d):
        n = rng.standard_normal(shape)
        comps.append(ndimage.gaussian_filter(n, sigma, mode="nearest"))
    u = np.stack(comps[::-1], axis=-1)  # component order x, y, z (numpy axes are reversed)
    nrm = np.sqrt((u ** 2).sum(-1)).max()
    return u * (max_norm / nrm)


def warp_linear(img: np.ndarray, u: np.ndarray) -> np.ndarray:
    """img(x + u(x)) with linear interpolation, clamped at the edges (u in voxels, x,y,z order)."""
    d = img.ndim
    grids = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in img.shape], indexing="ij")
    coords = [grids[a] + u[..., d - 1 - a] for a in range(d)]
    return ndimage.map_coordinates(img, coords, order=1, mode="nearest")


def blobs_2d(size=(256, 256), n_blobs=40, noise=0.01, seed=SEED_BASE) -> np.ndarray:
    rng = np.random.default_rng(seed)
    ny, nx = size[1], size[0]
    y, x = np.mgrid[0:ny, 0:nx].astype(np.float64)
    img = np.zeros((ny, nx))
    for _ in range(n_blobs):
        cx, cy = rng.uniform(0, nx), rng.uniform(0, ny)
        s = rng.uniform(4, 20) * min(nx, ny) / 256.0
        a = rng.uniform(0.2, 1.0)
        img += a * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * s * s))
    img += rng.normal(0.0, noise, img.shape)
    return img.astype(np.float32)


def _bernstein(t: np.ndarray) -> np.ndarray:
    return np.stack([(1 - t) ** 3, 3 * t * (1 - t) ** 2, 3 * t ** 2 * (1 - t), t ** 3])


def ellipsoid_phantom_3d(size=(182, 218, 182), seed=SEED_BASE, noise=0.02, blur=2.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    nx, ny, nz = size
    z, y, x = np.meshgrid(np.linspace(-1, 1, nz), np.linspace(-1, 1, ny), np.linspace(-1, 1, nx), indexing="ij")
    img = np.zeros((nz, ny, nx))
    c = rng.uniform(-0.05, 0.05, 3)
    axes = np.array([0.85, 0.85, 0.85]) * rng.uniform(0.9, 1.0, 3)
    for level, val in enumerate((0.1, 0.4, 0.7, 1.0)):
        a = axes * (1.0 - 0.22 * level) * rng.uniform(0.92, 1.0, 3)
        cc = c + rng.uniform(-0.04, 0.04, 3) * level
        r = ((x - cc[0]) / a[0]) ** 2 + ((y - cc[1]) / a[1]) ** 2 + ((z - cc[2]) / a[2]) ** 2
        img[r <= 1.0] = val
    ctrl = rng.uniform(-0.15, 0.15, (4, 4, 4))
    bz, by, bx = _bernstein(np.linspace(0, 1, nz)), _bernstein(np.linspace(0, 1, ny)), _bernstein(np.linspace(0, 1, nx))
    bias = np.einsum("ijk,iz,jy,kx->zyx", ctrl, bz, by, bx)
    img = img * (1.0 + bias)
    img += rng.normal(0.0, noise, img.shape)
    img = ndimage.gaussian_filter(img, blur, mode="nearest")
    return img.astype(np.float32)


def pair_2d(size=(256, 256), seed=SEED_BASE, field_sigma=12.0, max_disp=4.0):
    """Fixed blobs image and moving = fixed warped by a smooth field (2-D workload recipe)."""
    fixed = blobs_2d(size, seed=seed)
    rng = np.random.default_rng(seed + 1)
    u = smooth_field(fixed.shape, field_sigma * min(size) / 256.0, max_disp, rng)
    moving = warp_linear(fixed.astype(np.float64), u).astype(np.float32)
    return fixed, moving


def pair_3d(size=(182, 218, 182), seed=SEED_BASE, field_sigma=10.0, max_disp=8.0):
    """Fixed ellipsoid phantom and moving = fixed warped by a smooth field (3-D workload recipe)."""
    fixed = ellipsoid_phantom_3d(size, seed=seed)
    rng = np.random.default_rng(seed + 1)
    scale = min(size) / 182.0
    u = smooth_field(fixed.shape, max(field_sigma * scale, 1.0), max(max_disp * scale, 0.5), rng)
    moving = warp_linear(fixed.astype(np.float64), u).astype(np.float32)
    return fixed, moving
