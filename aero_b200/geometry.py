"""Obstacle shapes: solid masks and signed-distance fields on the lattice.

Same constructors, conventions and floating-point expressions as the
reference shapes, so masks and q values come out bit for bit equal:
  Cylinder  aero/geometry/cylinder.py:8-42
  Rectangle aero/geometry/rectangle.py:8-55
  Sphere    aero/geometry3d/sphere.py:7-51
  Box       aero/geometry3d/box.py:7-69
Masks use integer cell coordinates with an inclusive bound; the SDF is
sampled at cell centres (coordinate + 0.5), negative inside.
"""

from __future__ import annotations

from typing import Tuple

import numpy as np


def _axes(n: int, half: bool) -> np.ndarray:
    a = np.arange(n, dtype=np.float64)
    return a + 0.5 if half else a


class Cylinder:
    def __init__(self, radius: float = 20.0, cx_frac: float = 1 / 3, cy_frac: float = 0.5):
        self.radius = radius
        self.cx_frac = cx_frac
        self.cy_frac = cy_frac

    def center(self, Ny: int, Nx: int) -> Tuple[float, float]:
        return self.cx_frac * Nx, self.cy_frac * Ny

    def reference_length(self) -> float:
        return 2.0 * self.radius

    def _d2(self, Ny, Nx, half):
        cx, cy = self.center(Ny, Nx)
        x = _axes(Nx, half)[None, :]
        y = _axes(Ny, half)[:, None]
        return (x - cx) ** 2 + (y - cy) ** 2

    def mark_solid(self, Ny: int, Nx: int) -> np.ndarray:
        return self._d2(Ny, Nx, False) <= self.radius ** 2

    def sdf_field(self, Ny: int, Nx: int) -> np.ndarray:
        return np.sqrt(self._d2(Ny, Nx, True)) - self.radius


class Rectangle:
    def __init__(self, width: float = 40.0, height: float = 20.0, cx_frac: float = 1 / 3,
                 cy_frac: float = 0.5):
        self.width = width
        self.height = height
        self.cx_frac = cx_frac
        self.cy_frac = cy_frac

    def center(self, Ny: int, Nx: int) -> Tuple[float, float]:
        return self.cx_frac * Nx, self.cy_frac * Ny

    def reference_length(self) -> float:
        return self.height

    def mark_solid(self, Ny: int, Nx: int) -> np.ndarray:
        cx, cy = self.center(Ny, Nx)
        x = _axes(Nx, False)[None, :]
        y = _axes(Ny, False)[:, None]
        return (np.abs(x - cx) <= self.width / 2) & (np.abs(y - cy) <= self.height / 2)

    def sdf_field(self, Ny: int, Nx: int) -> np.ndarray:
        cx, cy = self.center(Ny, Nx)
        x = _axes(Nx, True)[None, :]
        y = _axes(Ny, True)[:, None]
        dx = np.abs(x - cx) - self.width / 2.0
        dy = np.abs(y - cy) - self.height / 2.0
        dx, dy = np.broadcast_arrays(dx, dy)
        return (np.sqrt(np.maximum(dx, 0.0) ** 2 + np.maximum(dy, 0.0) ** 2)
                + np.minimum(np.maximum(dx, dy), 0.0))


class Sphere:
    def __init__(self, radius: float = 10.0, cx_frac: float = 1 / 3, cy_frac: float = 0.5,
                 cz_frac: float = 0.5):
        self.radius = radius
        self.cx_frac = cx_frac
        self.cy_frac = cy_frac
        self.cz_frac = cz_frac

    def center(self, Nz: int, Ny: int, Nx: int) -> Tuple[float, float, float]:
        return self.cx_frac * Nx, self.cy_frac * Ny, self.cz_frac * Nz

    def reference_length(self) -> float:
        return 2.0 * self.radius

    def _d2(self, Nz, Ny, Nx, half):
        cx, cy, cz = self.center(Nz, Ny, Nx)
        x = _axes(Nx, half)[None, None, :]
        y = _axes(Ny, half)[None, :, None]
        z = _axes(Nz, half)[:, None, None]
        return (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2

    def mark_solid(self, Nz: int, Ny: int, Nx: int) -> np.ndarray:
        return self._d2(Nz, Ny, Nx, False) <= self.radius ** 2

    def sdf_field(self, Nz: int, Ny: int, Nx: int) -> np.ndarray:
        return np.sqrt(self._d2(Nz, Ny, Nx, True)) - self.radius


class Box:
    def __init__(self, width: float = 10.0, height: float = 10.0, depth: float = 10.0,
                 cx_frac: float = 1 / 3, cy_frac: float = 0.5, cz_frac: float = 0.5):
        self.width = width
        self.height = height
        self.depth = depth
        self.cx_frac = cx_frac
        self.cy_frac = cy_frac
        self.cz_frac = cz_frac

    def center(self, Nz: int, Ny: int, Nx: int) -> Tuple[float, float, float]:
        return self.cx_frac * Nx, self.cy_frac * Ny, self.cz_frac * Nz

    def reference_length(self) -> float:
        return self.height

    def mark_solid(self, Nz: int, Ny: int, Nx: int) -> np.ndarray:
        cx, cy, cz = self.center(Nz, Ny, Nx)
        x = _axes(Nx, False)[None, None, :]
        y = _axes(Ny, False)[None, :, None]
        z = _axes(Nz, False)[:, None, None]
        return ((np.abs(x - cx) <= self.width / 2.0) & (np.abs(y - cy) <= self.height / 2.0)
                & (np.abs(z - cz) <= self.depth / 2.0))

    def sdf_field(self, Nz: int, Ny: int, Nx: int) -> np.ndarray:
        cx, cy, cz = self.center(Nz, Ny, Nx)
        x = _axes(Nx, True)[None, None, :]
        y = _axes(Ny, True)[None, :, None]
        z = _axes(Nz, True)[:, None, None]
        dx, dy, dz = np.broadcast_arrays(np.abs(x - cx) - self.width / 2.0,
                                         np.abs(y - cy) - self.height / 2.0,
                                         np.abs(z - cz) - self.depth / 2.0)
        return (np.sqrt(np.maximum(dx, 0.0) ** 2 + np.maximum(dy, 0.0) ** 2
                        + np.maximum(dz, 0.0) ** 2)
                + np.minimum(np.maximum(np.maximum(dx, dy), dz), 0.0))
