"""Uniform cell-centred grid, laid out as the reference lays it out.

Mirrors ``Grid<Real, backend::Host>``'s serial constructor
(miso/include/miso/grid.hpp:316-337) and ``AxisGrid`` (grid.hpp:34-99):

* an axis of size 1 is degenerate: margin 0, stride flag 0, ``ds = 1e30``,
  ``dsi = 0`` (grid.hpp:67-90);
* every other axis carries ``margin`` ghost cells on each side;
* ``min_dxyz`` is the float-rounded minimum of the first spacing of each axis
  (grid.hpp:241), because ``util::min3`` goes through ``fminf``
  (utility.hpp:91-124).

Arrays are (i_total, j_total, k_total), k fastest (array3d.hpp:54-60).
"""
from __future__ import annotations

import numpy as np


def _axis(size: int, margin: int, lo: float, hi: float):
    """grid.hpp:22-31 (UniformAxisProvider) and 53-99 (AxisGrid)."""
    stride = 1 if size > 1 else 0
    m = margin * stride
    total = size + 2 * m
    if size == 1:
        sp = (hi - lo) / float(size)
        return (np.array([lo + 0.5 * sp]), np.array([1.0e30]), np.array([0.0]), m, stride, total)
    s = np.empty(total)
    ds = np.empty(total)
    dsi = np.empty(total)
    for i in range(total):
        ig = i - m
        sp = (hi - lo) / float(size)
        s[i] = lo + (float(ig) + 0.5) * sp
        ds[i] = sp
        dsi[i] = 1.0 / sp
    return s, ds, dsi, m, stride, total


class Grid:
    """Serial grid (one rank owns the whole domain)."""

    def __init__(self, i_size: int, j_size: int, k_size: int, margin: int = 2,
                 x_min: float = 0.0, x_max: float = 1.0, y_min: float = 0.0,
                 y_max: float = 1.0, z_min: float = 0.0, z_max: float = 1.0):
        # grid.hpp:244-276 argument checks
        if margin < 1:
            raise ValueError("Invalid margin size: margin < 1")
        if i_size <= 0 or j_size <= 0 or k_size <= 0:
            raise ValueError("Invalid grid size: i_size <= 0 or j_size <= 0 or k_size <= 0")
        if x_min >= x_max or y_min >= y_max or z_min >= z_max:
            raise ValueError("Invalid grid range: x_min >= x_max or y_min >= y_max or z_min >= z_max")
        self.i_size, self.j_size, self.k_size = int(i_size), int(j_size), int(k_size)
        self.margin = int(margin)
        self.x_min, self.x_max = float(x_min), float(x_max)
        self.y_min, self.y_max = float(y_min), float(y_max)
        self.z_min, self.z_max = float(z_min), float(z_max)
        self.x, self.dx, self.dxi, self.i_margin, self.is_, self.i_total = _axis(
            self.i_size, self.margin, self.x_min, self.x_max)
        self.y, self.dy, self.dyi, self.j_margin, self.js, self.j_total = _axis(
            self.j_size, self.margin, self.y_min, self.y_max)
        self.z, self.dz, self.dzi, self.k_margin, self.ks, self.k_total = _axis(
            self.k_size, self.margin, self.z_min, self.z_max)
        f = np.float32
        self.min_dxyz = float(min(f(self.dx[0]), f(self.dy[0]), f(self.dz[0])))
        for a, n, m in (("x", self.i_size, self.i_margin), ("y", self.j_size, self.j_margin),
                        ("z", self.k_size, self.k_margin)):
            if m and n < m:
                raise ValueError(f"axis {a}: size {n} smaller than margin {m}")

    @property
    def shape(self):
        return (self.i_total, self.j_total, self.k_total)

    @property
    def interior(self):
        """Slices of the interior (non-ghost) cells."""
        return (slice(self.i_margin, self.i_total - self.i_margin),
                slice(self.j_margin, self.j_total - self.j_margin),
                slice(self.k_margin, self.k_total - self.k_margin))

    @property
    def n_interior(self) -> int:
        return self.i_size * self.j_size * self.k_size

    @property
    def ndim(self) -> int:
        return self.is_ + self.js + self.ks

    def __repr__(self):
        return (f"Grid({self.i_size}x{self.j_size}x{self.k_size}, margin={self.margin}, "
                f"total={self.shape})")
