"""Cartesian mesh of the structured path.

Mirrors ``LSQMesh.create_2d(domain=(x0, x1, y0, y1), nx, ny)`` as the
reference's tests call it (``tests/runtime/test_swe_2d.py:34``): cell
``(i, j)`` (``i`` along x) is cell ``i * ny + j``, faces are unit-area-scaled
edges, the cell inradius is ``2 |cell| / perimeter``.  Only the scalars live
here: the kernels rebuild the geometry and the least-squares stencil weights
from them, so no connectivity array ever travels to the device.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

TAGS = ("left", "right", "bottom", "top")


@dataclass(frozen=True)
class CartesianMesh:
    x0: float
    x1: float
    y0: float
    y1: float
    nx: int
    ny: int
    dimension: int = 2

    @property
    def dx(self):
        return (self.x1 - self.x0) / self.nx

    @property
    def dy(self):
        return (self.y1 - self.y0) / self.ny

    @property
    def n_inner_cells(self):
        return self.nx * self.ny

    n_cells = n_inner_cells

    @property
    def cell_volume(self):
        return self.dx * self.dy

    @property
    def cell_inradius(self):
        return self.dx * self.dy / (self.dx + self.dy)

    def cell_centers(self):
        """``(2, C)`` cell centres in cell order (host array)."""
        i, j = np.divmod(np.arange(self.n_cells), self.ny)
        return np.stack([self.x0 + (i + 0.5) * self.dx,
                         self.y0 + (j + 0.5) * self.dy])

    @staticmethod
    def create_2d(domain, nx, ny):
        x0, x1, y0, y1 = (float(v) for v in domain)
        if nx < 3 or ny < 3:
            raise ValueError("the Cartesian path needs at least 3x3 cells")
        return CartesianMesh(x0, x1, y0, y1, int(nx), int(ny))


def create_2d(domain, nx, ny):
    return CartesianMesh.create_2d(domain, nx, ny)
