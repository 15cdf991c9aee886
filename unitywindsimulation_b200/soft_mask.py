"""Soft building mask: buildings whose heights are continuous parameters.

The reference marks obstacles with binary cell flags (InitFlags,
FvmSolverGpu.cs:972-987), which have no derivative with respect to a
building's height.  Here a building is a footprint (x0 <= x < x1,
z0 <= z < z1) with a height h in cells, and every cell of the footprint
column gets the solid fraction

    alpha(y) = sigmoid((h - (y + 0.5)) / width)

(1 well below the roof, 0 well above it, 1/2 at the roof line).  The
fraction acts through a Brinkman drag chi = chi_max * alpha added to the
momentum diagonal (WF_FIELD_DRAG), with every cell left fluid, so the flow
depends smoothly on h.  ``height_gradient`` chains dJ/dchi (from the
adjoint) to dJ/dh.
"""
from __future__ import annotations

import dataclasses

import numpy as np


def _sigmoid(t):
    return 0.5 * (1.0 + np.tanh(0.5 * t))


@dataclasses.dataclass
class SoftBuildings:
    footprints: list          # (x0, x1, z0, z1) per building, cells
    heights: np.ndarray       # float64, cells
    chi_max: float            # drag of a fully solid cell, 1/s
    width: float = 1.0        # sigmoid width, cells
    angle_deg: float = 0.0    # footprints rotated about the domain centre (x-z plane)
    margin: int = 0           # cells this close to the x/z boundaries stay free

    def __post_init__(self):
        self.heights = np.asarray(self.heights, dtype=np.float64)
        if len(self.footprints) != self.heights.size:
            raise ValueError("one height per footprint")

    def with_heights(self, heights) -> "SoftBuildings":
        return dataclasses.replace(self, heights=np.asarray(heights, dtype=np.float64).copy())

    def footprint_mask(self, i: int, nx: int, nz: int) -> np.ndarray:
        """Cells (nz, nx) of footprint i: cell centres inside the rectangle
        after rotating it by angle_deg about the domain centre, outside the
        boundary margin (the rule of the binary rasteriser in cases.py)."""
        x0, x1, z0, z1 = self.footprints[i]
        X, Z = np.meshgrid(np.arange(nx) + 0.5, np.arange(nz) + 0.5)
        if self.angle_deg == 0.0:
            m = (X >= x0) & (X < x1) & (Z >= z0) & (Z < z1)
        else:
            cx, cz = nx / 2.0, nz / 2.0
            th = np.radians(self.angle_deg)
            c, s = np.cos(th), np.sin(th)
            xr = cx + (X - cx) * c + (Z - cz) * s
            zr = cz - (X - cx) * s + (Z - cz) * c
            m = (xr >= x0) & (xr < x1) & (zr >= z0) & (zr < z1)
        if self.margin > 0:
            m &= (X > self.margin) & (X < nx - self.margin) & (Z > self.margin) & (Z < nz - self.margin)
        return m

    def drag(self, nx: int, ny: int, nz: int, dtype=np.float32) -> np.ndarray:
        """Drag field chi, shape (nz, ny, nx)."""
        out = np.zeros((nz, ny, nx), dtype=np.float64)
        yc = np.arange(ny, dtype=np.float64) + 0.5
        for i, h in enumerate(self.heights):
            a = self.chi_max * _sigmoid((h - yc) / self.width)
            m = self.footprint_mask(i, nx, nz)
            col = np.where(m[:, None, :], a[None, :, None], 0.0)
            np.maximum(out, col, out=out)
        return out.astype(dtype)

    def height_gradient(self, dJ_ddrag: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
        """dJ/dh per building from dJ/dchi (any shape with nz*ny*nx values).
        Footprints must not overlap (the max in ``drag`` is then a plain
        assignment)."""
        g = np.asarray(dJ_ddrag, dtype=np.float64).reshape(nz, ny, nx)
        yc = np.arange(ny, dtype=np.float64) + 0.5
        out = np.zeros(self.heights.size)
        for i, h in enumerate(self.heights):
            s = _sigmoid((h - yc) / self.width)
            dchi_dh = self.chi_max * s * (1.0 - s) / self.width
            m = self.footprint_mask(i, nx, nz)
            out[i] = float((g.transpose(1, 0, 2)[:, m].sum(axis=1) * dchi_dh).sum())
        return out
