"""Synthetic inflow: the transverse inlet velocities of every step.

Restates the reference's generator, including its random stream, so that a
solver seeded alike sees the same fields step for step:
2D ``Solver._update_synthetic_inflow`` (aero/lbm/solver.py:259-270) and 3D
``Solver3D._update_synthetic_inflow`` (aero/lbm/solver3d.py:297-321).  Each
step draws standard normals from ``numpy.random.default_rng(seed)`` (one
plane in 2D; uy then uz planes in 3D), smooths them with a 3-point (2D) or
5-point periodic (3D) average, blends them into the previous field (0.75 /
0.25 in 2D, 0.8 / 0.2 in 3D), removes the mean and rescales the RMS to
intensity x u0.  The fields run on the host (they are the reference's
random numbers) and reach the device through ``aero_set_inflow``.
"""

from __future__ import annotations

import numpy as np


class SyntheticInflow:
    def __init__(self, dims: int, ny: int, nz: int, u0: float, intensity: float, seed: int):
        self.dims = int(dims)
        self.shape = (int(ny),) if self.dims == 2 else (int(nz), int(ny))
        self.target = float(intensity) * float(u0)
        self.rng = np.random.default_rng(int(seed))
        self.uy = np.zeros(self.shape, dtype=np.float64)
        self.uz = np.zeros(self.shape, dtype=np.float64) if self.dims == 3 else None

    def _next(self) -> np.ndarray:
        if self.dims == 2:
            noise = self.rng.standard_normal(self.shape[0])
            filt = (noise + np.roll(noise, 1) + np.roll(noise, -1)) / 3.0
            self.uy = 0.75 * self.uy + 0.25 * filt
            self.uy -= float(np.mean(self.uy))
            rms = float(np.sqrt(np.mean(self.uy ** 2)))
            if rms > 1e-12 and self.target > 0.0:
                self.uy *= self.target / rms
            return self.uy.copy()[None]
        ny_, nz_ = self.rng.standard_normal(self.shape), self.rng.standard_normal(self.shape)

        def smooth(a):
            return (a + np.roll(a, 1, axis=0) + np.roll(a, -1, axis=0) + np.roll(a, 1, axis=1)
                    + np.roll(a, -1, axis=1)) / 5.0
        self.uy = 0.8 * self.uy + 0.2 * smooth(ny_)
        self.uz = 0.8 * self.uz + 0.2 * smooth(nz_)
        self.uy -= float(np.mean(self.uy))
        self.uz -= float(np.mean(self.uz))
        rms = float(np.sqrt(np.mean(self.uy ** 2 + self.uz ** 2)))
        if rms > 1e-12 and self.target > 0.0:
            s = self.target / rms
            self.uy *= s
            self.uz *= s
        return np.stack([self.uy, self.uz])

    def fields(self, n: int) -> np.ndarray:
        """The next n steps' fields: (n, dims-1, nz*ny) doubles, (z, y) order."""
        out = np.empty((int(n), self.dims - 1, int(np.prod(self.shape))), dtype=np.float64)
        for k in range(int(n)):
            out[k] = self._next().reshape(self.dims - 1, -1)
        return out
