"""Seeded synthetic inputs for the B-spline cost function.

No public dataset is involved: these generators stand in for CT volumes and
registration pairs with the shapes, spacings and value distributions of the
workloads the library is measured on.  All use numpy's PCG64 generator, so a
(seed, shape) pair always gives the same volume.

Volumes are float32 numpy arrays shaped (nz, ny, nx); flat index
i + nx*(j + ny*k), the same voxel order as Plastimatch's Volume.
"""
from __future__ import annotations

import numpy as np

from .geometry import BsplineGrid, Volume

SEED_BASE = 20261203


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def gaussian_blobs(dim, spacing=(1.0, 1.0, 1.0), n_blobs=20, seed=SEED_BASE,
                   noise_sigma=10.0, origin=(0.0, 0.0, 0.0)) -> Volume:
    """Sum of `n_blobs` Gaussian blobs (centres uniform in the volume,
    amplitude U[100,1000], sigma U[3,10] voxels) plus N(0, noise_sigma)."""
    g = rng(seed)
    nx, ny, nz = (int(d) for d in dim)
    z = np.arange(nz, dtype=np.float64)
    y = np.arange(ny, dtype=np.float64)
    x = np.arange(nx, dtype=np.float64)
    ez = np.empty((n_blobs, nz))
    ey = np.empty((n_blobs, ny))
    ex = np.empty((n_blobs, nx))
    for b in range(n_blobs):
        cx, cy, cz = g.uniform(0, nx), g.uniform(0, ny), g.uniform(0, nz)
        amp = g.uniform(100.0, 1000.0)
        sig = g.uniform(3.0, 10.0)
        ez[b] = amp * np.exp(-((z - cz) ** 2) / (2 * sig * sig))
        ey[b] = np.exp(-((y - cy) ** 2) / (2 * sig * sig))
        ex[b] = np.exp(-((x - cx) ** 2) / (2 * sig * sig))
    # each blob is separable: the sum is one (z*y) x blobs x (x) product
    zy = (ez[:, :, None] * ey[:, None, :]).reshape(n_blobs, nz * ny)
    img = (zy.T @ ex).reshape(nz, ny, nx)
    img += g.normal(0.0, noise_sigma, img.shape)
    return Volume(img.astype(np.float32), origin=origin, spacing=spacing)


def _ellipsoid(shape, centre, radii):
    nz, ny, nx = shape
    z = (np.arange(nz)[:, None, None] - centre[2]) / radii[2]
    y = (np.arange(ny)[None, :, None] - centre[1]) / radii[1]
    x = (np.arange(nx)[None, None, :] - centre[0]) / radii[0]
    return x * x + y * y + z * z <= 1.0


def ct_phantom(dim, spacing=(0.98, 0.98, 2.5), seed=SEED_BASE + 1,
               noise_sigma=20.0, origin=(0.0, 0.0, 0.0)) -> Volume:
    """CT-like int16 volume converted to float32: air -1000 HU, a body
    ellipsoid at 0 HU, two lung ellipsoids at -800 HU, a spine and a few rib
    ellipsoids at +700..+2000 HU, N(0, noise_sigma) noise, clipped to
    [-1000, 2000] and rounded to int16."""
    g = rng(seed)
    nx, ny, nz = (int(d) for d in dim)
    shape = (nz, ny, nx)
    img = np.full(shape, -1000.0, np.float64)
    c = (nx / 2, ny / 2, nz / 2)
    body = _ellipsoid(shape, c, (0.42 * nx, 0.30 * ny, 0.55 * nz))
    img[body] = 0.0
    for s in (-1, 1):
        lung = _ellipsoid(shape, (c[0] + s * 0.18 * nx, c[1] - 0.02 * ny, c[2]),
                          (0.13 * nx, 0.17 * ny, 0.40 * nz))
        img[lung & body] = -800.0
    spine = _ellipsoid(shape, (c[0], c[1] + 0.20 * ny, c[2]),
                       (0.05 * nx, 0.05 * ny, 0.60 * nz))
    img[spine & body] = g.uniform(700.0, 2000.0)
    for _ in range(6):
        cx = c[0] + g.uniform(-0.35, 0.35) * nx
        cy = c[1] + g.uniform(-0.25, 0.25) * ny
        cz = c[2] + g.uniform(-0.4, 0.4) * nz
        rib = _ellipsoid(shape, (cx, cy, cz),
                         (g.uniform(0.01, 0.04) * nx, g.uniform(0.01, 0.04) * ny,
                          g.uniform(0.05, 0.2) * nz))
        img[rib & body] = g.uniform(700.0, 2000.0)
    img += g.normal(0.0, noise_sigma, shape)
    img = np.clip(np.rint(img), -1000, 2000).astype(np.int16)
    return Volume(img.astype(np.float32), origin=origin, spacing=spacing)


def random_coeff(grid: BsplineGrid, sigma_mm: float, seed: int) -> np.ndarray:
    """Coefficients N(0, sigma_mm), interleaved xyz per knot (float32)."""
    return rng(seed).normal(0.0, sigma_mm, grid.num_coeff).astype(np.float32)


def intensity_remap(vol: Volume, gamma: float, noise_sigma: float,
                    seed: int) -> Volume:
    """Monotone remap I' = lo + (hi-lo)*((I-lo)/(hi-lo))^gamma plus noise."""
    img = vol.img.astype(np.float64)
    lo, hi = float(img.min()), float(img.max())
    out = lo + (hi - lo) * ((img - lo) / max(hi - lo, 1e-12)) ** gamma
    out += rng(seed).normal(0.0, noise_sigma, img.shape)
    return Volume(out.astype(np.float32), origin=vol.origin,
                  spacing=vol.spacing, dcos=vol.dcos)


def bspline_field(grid: BsplineGrid, coeff: np.ndarray) -> np.ndarray:
    """Dense displacement field (nz, ny, nx, 3) of the cubic B-spline grid
    over its ROI, in double precision (separable tensor-product
    evaluation)."""
    vpr = grid.vox_per_rgn
    rd = grid.roi_dim
    c = coeff.reshape(grid.cdims[2], grid.cdims[1], grid.cdims[0], 3)
    c = c.astype(np.float64)

    def basis_1d(n, v):
        i = np.arange(n)
        p, u = i // v, (i % v) / v
        w = np.stack([(1 - u) ** 3 / 6, (3 * u ** 3 - 6 * u ** 2 + 4) / 6,
                      (-3 * u ** 3 + 3 * u ** 2 + 3 * u + 1) / 6, u ** 3 / 6], 1)
        return p, w

    px, wx = basis_1d(rd[0], vpr[0])
    py, wy = basis_1d(rd[1], vpr[1])
    pz, wz = basis_1d(rd[2], vpr[2])
    out = np.zeros((rd[2], rd[1], rd[0], 3))
    for k in range(4):
        for j in range(4):
            for i in range(4):
                w = (wz[:, k][:, None, None] * wy[:, j][None, :, None]
                     * wx[:, i][None, None, :])
                out += w[..., None] * c[pz + k][:, py + j][:, :, px + i]
    return out


def warp_trilinear(moving: Volume, fixed_like: Volume, grid: BsplineGrid,
                   coeff: np.ndarray, default: float = 0.0) -> Volume:
    """Warp `moving` onto the fixed grid with the B-spline field (trilinear,
    `default` outside), as Plastimatch's bspline_warp does."""
    d = bspline_field(grid, coeff)
    nz, ny, nx = fixed_like.img.shape
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx),
                             indexing="ij")
    step = fixed_like.step()
    pos = [fixed_like.origin[r] + ii * step[r, 0] + jj * step[r, 1]
           + kk * step[r, 2] + d[..., r] for r in range(3)]
    proj = moving.proj()
    rel = [pos[r] - moving.origin[r] for r in range(3)]
    mijk = [rel[0] * proj[r, 0] + rel[1] * proj[r, 1] + rel[2] * proj[r, 2]
            for r in range(3)]
    mdim = moving.dim
    inside = np.ones(mijk[0].shape, bool)
    for r in range(3):
        inside &= (mijk[r] > -0.5) & (mijk[r] < mdim[r] - 0.5)
    f, w2 = [], []
    for r in range(3):
        m = np.clip(mijk[r], 0, mdim[r] - 1)
        fl = np.minimum(np.floor(m), mdim[r] - 2).astype(np.int64)
        f.append(fl)
        w2.append(m - fl)
    img = moving.img.astype(np.float64)
    out = np.zeros(mijk[0].shape)
    for c in range(8):
        wx = w2[0] if c & 1 else 1 - w2[0]
        wy = w2[1] if c & 2 else 1 - w2[1]
        wz = w2[2] if c & 4 else 1 - w2[2]
        out += wx * wy * wz * img[f[2] + (c >> 2 & 1), f[1] + (c >> 1 & 1),
                                  f[0] + (c & 1)]
    out = np.where(inside, out, default)
    return Volume(out.astype(np.float32), origin=fixed_like.origin,
                  spacing=fixed_like.spacing, dcos=fixed_like.dcos)
