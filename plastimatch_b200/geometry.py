"""Geometry types mirroring Plastimatch's Volume and Bspline_header.

Volume       <- src/base/volume.h:37-57 (dim, origin, spacing, direction
                cosines, step = dc*spacing, proj = inv(dc)/spacing)
BsplineGrid  <- src/base/bspline_header.cxx:28-62 (roi, vox_per_rgn,
                rdims = 1 + (roi_dim-1)/vpr, cdims = rdims + 3)

Both are plain host-side descriptions; images stay numpy float32 arrays
shaped (nz, ny, nx) (x fastest), coefficients a float32 vector interleaved
xyz per knot, the layouts the reference uses.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

IDENTITY_DCOS = (1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0)


def _inv3_f32(m: np.ndarray) -> np.ndarray:
    """Cofactor inverse in float32, as direction_cosines.cxx:135-158."""
    m = m.astype(np.float32).ravel()
    det = np.float32(m[0] * (m[4] * m[8] - m[5] * m[7])
                     - m[1] * (m[3] * m[8] - m[5] * m[6])
                     + m[2] * (m[3] * m[7] - m[4] * m[6]))
    if abs(det) < 1e-8:
        raise ValueError("singular matrix of direction cosines")
    out = np.empty(9, np.float32)
    out[0] = (m[4] * m[8] - m[5] * m[7]) / det
    out[1] = -(m[1] * m[8] - m[2] * m[7]) / det
    out[2] = (m[1] * m[5] - m[2] * m[4]) / det
    out[3] = -(m[3] * m[8] - m[5] * m[6]) / det
    out[4] = (m[0] * m[8] - m[2] * m[6]) / det
    out[5] = -(m[0] * m[5] - m[2] * m[3]) / det
    out[6] = (m[3] * m[7] - m[4] * m[6]) / det
    out[7] = -(m[0] * m[7] - m[1] * m[6]) / det
    out[8] = (m[0] * m[4] - m[1] * m[3]) / det
    return out.reshape(3, 3)


@dataclass
class Volume:
    """A float32 image and its physical geometry (mm)."""
    img: np.ndarray
    origin: tuple = (0.0, 0.0, 0.0)
    spacing: tuple = (1.0, 1.0, 1.0)
    dcos: tuple = IDENTITY_DCOS

    def __post_init__(self):
        self.img = np.ascontiguousarray(self.img, dtype=np.float32)
        self.origin = tuple(float(v) for v in self.origin)
        self.spacing = tuple(float(v) for v in self.spacing)
        self.dcos = tuple(float(v) for v in self.dcos)

    @property
    def dim(self) -> tuple:
        nz, ny, nx = self.img.shape[:3]
        return (nx, ny, nz)

    @property
    def npix(self) -> int:
        nx, ny, nz = self.dim
        return nx * ny * nz

    def step(self) -> np.ndarray:
        dc = np.asarray(self.dcos, np.float32).reshape(3, 3)
        return (dc * np.asarray(self.spacing, np.float32)[None, :]).astype(
            np.float32)

    def proj(self) -> np.ndarray:
        inv = _inv3_f32(np.asarray(self.dcos, np.float32))
        return (inv / np.asarray(self.spacing, np.float32)[:, None]).astype(
            np.float32)


@dataclass
class Roi:
    """An image region of interest: a uint8 mask (nonzero = inside) shaped
    (nz, ny, nx) with its own geometry, as Plastimatch's fixed_roi /
    moving_roi volumes (src/register/bspline_state.h:44-45)."""
    mask: np.ndarray
    origin: tuple = (0.0, 0.0, 0.0)
    spacing: tuple = (1.0, 1.0, 1.0)
    dcos: tuple = IDENTITY_DCOS

    def __post_init__(self):
        self.mask = np.ascontiguousarray(self.mask, dtype=np.uint8)
        self.origin = tuple(float(v) for v in self.origin)
        self.spacing = tuple(float(v) for v in self.spacing)
        self.dcos = tuple(float(v) for v in self.dcos)

    @property
    def dim(self) -> tuple:
        nz, ny, nx = self.mask.shape
        return (nx, ny, nz)

    @classmethod
    def like(cls, vol: Volume, mask) -> "Roi":
        """A mask on the voxel grid of `vol`."""
        return cls(mask, vol.origin, vol.spacing, vol.dcos)

    @classmethod
    def from_window(cls, vol: Volume, lo: float, hi: float) -> "Roi":
        """Voxels of `vol` with lo <= value <= hi: the mask a registration
        stage builds from its MI intensity window on an image without a
        ROI (update_roi, src/register/bspline_stage.cxx:72-95)."""
        img = vol.img
        return cls.like(vol, ((img >= lo) & (img <= hi)).astype(np.uint8))


@dataclass
class BsplineGrid:
    """The B-spline control grid over a fixed image's ROI."""
    img_origin: tuple
    img_spacing: tuple
    img_dim: tuple
    roi_offset: tuple
    roi_dim: tuple
    vox_per_rgn: tuple
    dcos: tuple = IDENTITY_DCOS
    rdims: tuple = field(init=False)
    cdims: tuple = field(init=False)

    def __post_init__(self):
        self.img_origin = tuple(float(v) for v in self.img_origin)
        self.img_spacing = tuple(float(v) for v in self.img_spacing)
        self.img_dim = tuple(int(v) for v in self.img_dim)
        self.roi_offset = tuple(int(v) for v in self.roi_offset)
        self.roi_dim = tuple(int(v) for v in self.roi_dim)
        self.vox_per_rgn = tuple(int(v) for v in self.vox_per_rgn)
        for d in range(3):
            if self.vox_per_rgn[d] < 1 or self.roi_dim[d] < 1:
                raise ValueError("vox_per_rgn and roi_dim must be >= 1")
            if self.roi_offset[d] < 0 or (self.roi_offset[d] + self.roi_dim[d]
                                          > self.img_dim[d]):
                raise ValueError("ROI outside the image")
        self.rdims = tuple(1 + (self.roi_dim[d] - 1) // self.vox_per_rgn[d]
                           for d in range(3))
        self.cdims = tuple(r + 3 for r in self.rdims)

    @classmethod
    def for_volume(cls, vol: Volume, vox_per_rgn, roi_offset=(0, 0, 0),
                   roi_dim=None) -> "BsplineGrid":
        if isinstance(vox_per_rgn, int):
            vox_per_rgn = (vox_per_rgn,) * 3
        return cls(vol.origin, vol.spacing, vol.dim, roi_offset,
                   roi_dim or vol.dim, vox_per_rgn, vol.dcos)

    @classmethod
    def for_grid_spacing(cls, vol: Volume, grid_spac_mm) -> "BsplineGrid":
        """vox_per_rgn = round(grid_spac / |spacing|), at least 4
        (src/base/bspline_header.cxx:64-95)."""
        if np.isscalar(grid_spac_mm):
            grid_spac_mm = (grid_spac_mm,) * 3
        vpr = []
        for d in range(3):
            x = grid_spac_mm[d] / abs(vol.spacing[d])
            v = int(x + 0.5) if x >= 0 else -int(-x + 0.5)
            vpr.append(max(v, 4))
        return cls.for_volume(vol, tuple(vpr))

    @property
    def num_tiles(self) -> int:
        return self.rdims[0] * self.rdims[1] * self.rdims[2]

    @property
    def num_knots(self) -> int:
        return self.cdims[0] * self.cdims[1] * self.cdims[2]

    @property
    def num_coeff(self) -> int:
        return 3 * self.num_knots

    @property
    def num_roi_voxels(self) -> int:
        return self.roi_dim[0] * self.roi_dim[1] * self.roi_dim[2]

    @property
    def grid_spac(self) -> tuple:
        return tuple(float(np.float32(self.vox_per_rgn[d])
                           * np.float32(abs(self.img_spacing[d])))
                     for d in range(3))
