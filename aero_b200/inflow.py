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


class SEMInflow:
    """Synthetic-eddy inlet fluctuations, step by step.

    Restates the reference's SEMInlet (aero/lbm/sem_inlet.py:15-136, after
    Jarrin et al. 2006) with its random stream: N eddies with random
    positions in a box of half-width 3 sigma around the inlet plane and
    random signs per component, advected by u0 per step and re-drawn when
    they leave; the fluctuations are sums of tent kernels
    max(0, 1 - r / sigma) / sqrt(N) at the plane's cell centres; (v, w) are
    made divergence-free in the plane by a Fourier projection (Nyquist modes
    removed first); u, and (v, w) jointly, are rescaled to RMS Tu u0.  The
    solver calls step() then fluctuation() once per time step
    (solver3d.py:433-438); the reference constructs it without a seed, so
    the stream starts from default_rng(0)."""

    def __init__(self, ny: int, nz: int, u0: float, Tu: float, L_int: float, N: int, seed: int = 0):
        self.ny, self.nz = int(ny), int(nz)
        self.u0, self.Tu, self.sigma, self.N = float(u0), float(Tu), float(L_int), int(N)
        self.half = 3.0 * self.sigma
        self.rng = np.random.default_rng(seed)
        self.x = self.rng.uniform(-self.half, self.half, self.N)
        self.y = self.rng.uniform(0.0, float(self.ny), self.N)
        self.z = self.rng.uniform(0.0, float(self.nz), self.N)
        self.sign = self.rng.choice(np.array([-1.0, 1.0]), size=(3, self.N)).astype(np.float64)

    def _advect(self):
        self.x += self.u0
        out = self.x > self.half
        k = int(np.sum(out))
        if k > 0:
            self.x[out] = -self.half
            self.y[out] = self.rng.uniform(0.0, float(self.ny), k)
            self.z[out] = self.rng.uniform(0.0, float(self.nz), k)
            self.sign[:, out] = self.rng.choice(np.array([-1.0, 1.0]), size=(3, k)).astype(np.float64)

    def _fluctuation(self) -> np.ndarray:
        shape = (self.nz, self.ny)
        if self.Tu <= 0.0 or self.sigma <= 0.0 or self.N == 0:
            return np.zeros((3,) + shape)
        zc = np.arange(self.nz, dtype=np.float64) + 0.5
        yc = np.arange(self.ny, dtype=np.float64) + 0.5
        Z, Y = np.meshgrid(zc, yc, indexing="ij")
        r = np.sqrt(self.x[:, None, None] ** 2 + (Y[None] - self.y[:, None, None]) ** 2
                    + (Z[None] - self.z[:, None, None]) ** 2)
        tent = np.maximum(0.0, 1.0 - r / self.sigma)
        norm = 1.0 / np.sqrt(float(self.N))
        raw = [norm * (self.sign[c, :, None, None] * tent).sum(axis=0) for c in range(3)]
        vh, wh = np.fft.fft2(raw[1]), np.fft.fft2(raw[2])
        if self.nz % 2 == 0:
            vh[self.nz // 2, :] = 0.0
            wh[self.nz // 2, :] = 0.0
        if self.ny % 2 == 0:
            vh[:, self.ny // 2] = 0.0
            wh[:, self.ny // 2] = 0.0
        kz = (np.fft.fftfreq(self.nz) * 2.0 * np.pi)[:, None]
        ky = (np.fft.fftfreq(self.ny) * 2.0 * np.pi)[None, :]
        k2 = kz ** 2 + ky ** 2
        k2[0, 0] = 1.0
        div = ky * vh + kz * wh
        vh -= ky / k2 * div
        wh -= kz / k2 * div
        v, w = np.real(np.fft.ifft2(vh)), np.real(np.fft.ifft2(wh))
        target = self.Tu * self.u0
        su = float(np.std(raw[0]))
        svw = float(np.sqrt(np.mean(v ** 2 + w ** 2) / 2.0))
        u = raw[0] * (target / su) if su > 1e-14 else np.zeros(shape)
        if svw > 1e-14:
            v, w = v * (target / svw), w * (target / svw)
        else:
            v, w = np.zeros(shape), np.zeros(shape)
        return np.stack([u, v, w])

    def fields(self, n: int) -> np.ndarray:
        """The next n steps' fluctuations: (n, 3, nz*ny) doubles (u', v', w'), (z, y) order."""
        out = np.empty((int(n), 3, self.nz * self.ny), dtype=np.float64)
        for k in range(int(n)):
            self._advect()
            out[k] = self._fluctuation().reshape(3, -1)
        return out
