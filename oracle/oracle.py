"""Parity oracle: ctypes wrapper around the FP64 C restatement (lbm_oracle.c).

TEST INFRASTRUCTURE ONLY.  ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module as the checker.  The product
package ``aero_b200`` never imports it.

``OracleSolver`` mirrors the constructor of the reference ``Solver`` /
``Solver3D`` (aero/lbm/solver.py:75-116, aero/lbm/solver3d.py:71-119) for the
hot-path options and exposes ``step()`` returning the per-step coefficients in
the reference's order.  Its link builder, lattice tables and MRT matrices are
written independently of the product's so that the two check each other.
"""

from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess
from typing import Optional

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "liblbm_oracle.so"

# --- lattice tables (aero/lbm/d2q9.py:18-38, aero/lbm/d3q19.py:37-73) ------
E2 = np.array([(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1)])
W2 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
OPP2 = np.array([0, 3, 4, 1, 2, 7, 8, 5, 6])
E3 = np.array([
    (0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
    (1, 1, 0), (-1, 1, 0), (1, -1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, 1), (1, 0, -1),
    (-1, 0, -1), (0, 1, 1), (0, -1, 1), (0, 1, -1), (0, -1, -1)])
W3 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
OPP3 = np.array([0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15])

# --- MRT bases: D2Q9 written out as the table of aero/lbm/mrt2d.py:36-46,
#     D3Q19 assembled row by row from the moment definitions listed in
#     aero/lbm/mrt3d.py:46-87 (rank 16, inverted with pinv as mrt3d.py:91);
#     relaxation vectors mrt2d.py:51-77, mrt3d.py:94-135. -----------------
M9_TABLE = np.array([
    [1, 1, 1, 1, 1, 1, 1, 1, 1],
    [-4, -1, -1, -1, -1, 2, 2, 2, 2],
    [4, -2, -2, -2, -2, 1, 1, 1, 1],
    [0, 1, 0, -1, 0, 1, -1, -1, 1],
    [0, -2, 0, 2, 0, 1, -1, -1, 1],
    [0, 0, 1, 0, -1, 1, 1, -1, -1],
    [0, 0, -2, 0, 2, 1, 1, -1, -1],
    [0, 1, -1, 1, -1, 0, 0, 0, 0],
    [0, 0, 0, 0, 0, 1, -1, 1, -1]], dtype=np.float64)


def _m19_table() -> np.ndarray:
    rows = []
    ex, ey, ez = E3[:, 0], E3[:, 1], E3[:, 2]
    e2 = ex * ex + ey * ey + ez * ez
    face = e2 == 1
    rows.append(np.ones(19))
    rows.append(np.select([e2 == 0, face], [-30, -11], 8))
    rows.append(np.select([e2 == 0, face], [12, -4], 1))
    for comp in (ex, ey, ez):
        rows.append(comp)
        rows.append(np.where(face, -4, 1) * comp)
    rows.append(2 * ex * ex - ey * ey - ez * ez)
    rows.append(ey * ey - ez * ez)
    rows.append(ex * ey)
    rows.append(ey * ez)
    rows.append(ex * ez)
    for comp in (ex, ey, ez):
        rows.append(np.where(face, -2, 1) * comp)
    rows.append(ex * (ey * ey - ez * ez))
    rows.append(ey * (ex * ex - ez * ez))
    return np.array(rows, dtype=np.float64)


M19_TABLE = _m19_table()


def mrt_s9(omega: float) -> np.ndarray:
    sq = 8.0 * (2.0 - omega) / (8.0 - omega)
    return np.array([1.0, 1.64, 1.54, 1.0, sq, 1.0, sq, omega, omega])


def mrt_s19(omega: float) -> np.ndarray:
    return np.array([1.0, 1.19, 1.40, 1.0, 1.20, 1.0, 1.20, 1.0, 1.20] + [omega] * 5 + [1.0] * 5)


def build_links(solid: np.ndarray, phi: Optional[np.ndarray]):
    """Surface links (aero/lbm/boundary.py:232-280, boundary3d.py:279-329).

    Direction-major, then C order over cells; the neighbour index is clipped
    to the grid; q = clip(float32(phi[cell]), 1e-4, 1) when phi is given,
    else 0.5.
    """
    dims = solid.ndim
    E = E2 if dims == 2 else E3
    fluid = ~solid
    shape = solid.shape
    links = []
    for i in range(1, len(E)):
        # e in (x, y[, z]) order; array axes are ([z,] y, x)
        shift = E[i][::-1]
        idx = np.indices(shape)
        nb = tuple(np.clip(idx[a] + shift[a], 0, shape[a] - 1) for a in range(dims))
        hit = np.argwhere(fluid & solid[nb])
        if hit.size:
            links.append(np.concatenate([np.full((len(hit), 1), i), hit], axis=1))
    if not links:
        return np.empty((0, dims + 1), np.int32), np.empty(0, np.float32)
    links = np.concatenate(links).astype(np.int32)
    if phi is None:
        q = np.full(len(links), 0.5, np.float32)
    else:
        q = np.clip(phi[tuple(links[:, 1 + a] for a in range(dims))].astype(np.float32),
                    np.float32(1e-4), np.float32(1.0))
    return links, q


class _OracleLattice(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in (
        "dims", "nx", "ny", "nz", "collision", "les", "les_model", "van_driest", "bouzidi",
        "ibm_enabled", "wall_bc", "inlet_bc", "outlet_bc", "streamwise_bc", "sponge_thickness",
        "thermal", "buoyancy", "scalar_reduced")] + [
        ("step_count", ctypes.c_int64), ("n_links", ctypes.c_int64)] + [
        (n, ctypes.c_double) for n in (
            "omega", "u0", "rho_in", "rho_out", "inlet_perturbation", "trt_lambda",
            "sponge_strength", "les_cs", "van_driest_A", "wall_velocity_top",
            "wall_velocity_bottom")] + [
        ("body_force", ctypes.c_double * 3)] + [
        (n, ctypes.c_double) for n in ("omega_T", "T_hot", "T_cold", "g_gravity", "beta", "T_ref")
    ] + [("center", ctypes.c_double * 3)] + [
        (n, ctypes.c_void_p) for n in (
            "f", "g", "f_outlet_prev", "solid", "phi", "links", "q_vals", "mrt_M", "mrt_Minv",
            "mrt_s", "work_a", "work_b", "work_om", "work_g", "inflow", "sem")]


def build(force: bool = False) -> pathlib.Path:
    """Compile the oracle with gcc (-O2 -fopenmp) into oracle/liblbm_oracle.so."""
    src = HERE / "lbm_oracle.c"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-o", str(LIB_PATH),
                               str(src), "-lm"])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        _lib.oracle_step.argtypes = [ctypes.POINTER(_OracleLattice), ctypes.c_void_p, ctypes.c_void_p]
        _lib.oracle_step.restype = ctypes.c_int
        _lib.oracle_collide_only.argtypes = [ctypes.POINTER(_OracleLattice), ctypes.c_void_p]
        _lib.oracle_omega_field.argtypes = [ctypes.POINTER(_OracleLattice), ctypes.c_void_p]
    return _lib


_WALL = {"none": 0, "slip": 1, "noslip": 2, "moving": 3}
_INLET = {"none": 0, "velocity": 1, "pressure": 2}
_OUTLET = {"none": 0, "convective": 1, "zerogradient": 2, "pressure": 3}
_COLL = {"bgk": 0, "trt": 1, "mrt": 2}


def _ptr(a):
    return None if a is None else a.ctypes.data


class OracleSolver:
    """FP64 CPU oracle with the reference Solver/Solver3D constructor options."""

    def __init__(self, *, solid: np.ndarray, omega: float, u0: float, D: float,
                 rho0: float = 1.0, wall_bc: str = "slip", inlet_bc: str = "velocity",
                 outlet_bc: str = "convective", streamwise_bc: str = "open",
                 rho_in: float = 1.0, rho_out: float = 1.0, collision: str = "bgk",
                 inlet_perturbation: float = 0.0, trt_lambda: float = 0.25,
                 sponge_thickness: int = 0, sponge_strength: float = 0.1, les: bool = False,
                 les_cs: float = 0.16, les_model: str = "smagorinsky",
                 phi: Optional[np.ndarray] = None, bouzidi: bool = False,
                 van_driest: bool = False, van_driest_A: float = 25.0,
                 body_force_x: float = 0.0, body_force_y: float = 0.0,
                 body_force_z: float = 0.0, wall_velocity_top: float = 0.0,
                 wall_velocity_bottom: float = 0.0, thermal: bool = False,
                 T_hot: float = 1.0, T_cold: float = 0.0, alpha_T: float = 1e-3,
                 buoyancy: bool = False, g_gravity: float = 0.0, beta: float = 1e-3,
                 T_ref: float = 0.5, scalar_lattice: str = "full", threads: Optional[int] = None,
                 synthetic_inflow: bool = False, synthetic_inflow_intensity: float = 0.03,
                 synthetic_inflow_seed: int = 12345, sem_inlet: bool = False, sem_Tu: float = 0.05,
                 sem_L_int: float = 10.0, sem_N: int = 200, **_ignored):
        solid = np.ascontiguousarray(solid, dtype=np.bool_)
        self.dims = solid.ndim
        if self.dims == 2:
            self.ny, self.nx = solid.shape
            self.nz = 1
        else:
            self.nz, self.ny, self.nx = solid.shape
        self.Q = 9 if self.dims == 2 else 19
        self.E = E2 if self.dims == 2 else E3
        self.W = W2 if self.dims == 2 else W3
        self.solid = solid
        self.solid_u8 = np.ascontiguousarray(solid.astype(np.uint8))
        self.u0, self.D, self.rho0 = float(u0), float(D), float(rho0)
        self.phi = None if phi is None else np.ascontiguousarray(phi, dtype=np.float64)
        self.surface_links, self.q_vals = build_links(solid, self.phi if bouzidi else None)
        self.links = np.ascontiguousarray(self.surface_links, dtype=np.int32)
        self.q = np.ascontiguousarray(self.q_vals, dtype=np.float32)
        shp = (self.Q,) + solid.shape
        self.f = np.ascontiguousarray(self.feq(np.full(solid.shape, rho0),
                                               np.full(solid.shape, u0)))
        self.f_outlet_prev = np.ascontiguousarray(self.f[..., -1])
        reduced = scalar_lattice == "reduced"
        if thermal:
            Wg = self.W if not reduced else (np.array([1 / 3] + [1 / 6] * 4) if self.dims == 2
                                             else np.array([1 / 4] + [1 / 8] * 6))
            self.Wg = Wg
            self.g = np.ascontiguousarray(Wg.reshape((-1,) + (1,) * self.dims) * T_ref *
                                          np.ones((len(Wg),) + solid.shape))
        else:
            self.g = None
        self._work_a = np.empty(shp)
        self._work_b = np.empty(shp)
        self._work_om = np.empty(solid.shape)
        self._work_g = None if self.g is None else np.empty_like(self.g)
        if collision == "mrt":
            M = M9_TABLE if self.dims == 2 else M19_TABLE
            Minv = np.linalg.inv(M) if self.dims == 2 else np.linalg.pinv(M)
            svec = mrt_s9(omega) if self.dims == 2 else mrt_s19(omega)
            self._M, self._Minv, self._s = (np.ascontiguousarray(a) for a in (M, Minv, svec))
        else:
            self._M = self._Minv = self._s = None
        idx = np.nonzero(solid)
        ctr = [float(np.mean(a)) if a.size else 0.5 * (n - 1) for a, n in zip(idx, solid.shape)]
        # solid.shape order is ([z,] y, x); center is stored as (x, y, z)
        ctr = ctr[::-1] + ([0.0] if self.dims == 2 else [])
        alpha_scale = 4.0 if (reduced and self.dims == 3) else 3.0
        s = _OracleLattice()
        s.dims, s.nx, s.ny, s.nz = self.dims, self.nx, self.ny, self.nz
        s.collision = _COLL[collision]
        s.les = int(bool(les))
        s.les_model = 1 if les_model == "wale" else 0
        s.van_driest = int(bool(van_driest))
        s.bouzidi = int(bool(bouzidi))
        s.wall_bc = _WALL.get(wall_bc, 0)
        s.inlet_bc = _INLET.get(inlet_bc, 0)
        s.outlet_bc = _OUTLET.get(outlet_bc, 2)
        s.streamwise_bc = {"open": 0, "periodic": 1, "recycling": 2}[streamwise_bc]
        # synthetic inflow (solver.py:259-270, solver3d.py:297-321): transverse
        # inlet velocities drawn step by step from the seeded generator
        self._inflow_on = bool(synthetic_inflow) and inlet_bc == "velocity" and (
            self.dims == 2 or streamwise_bc == "open")
        self._inflow_target = float(synthetic_inflow_intensity) * float(u0)
        self._inflow_rng = np.random.default_rng(int(synthetic_inflow_seed))
        plane = (self.ny,) if self.dims == 2 else (self.nz, self.ny)
        self._inflow_u = [np.zeros(plane) for _ in range(self.dims - 1)]
        self._inflow_buf = None
        # SEM inlet (sem_inlet.py:15-136, used first when enabled, solver3d.py:433-438);
        # the reference builds it without a seed: default_rng(0)
        self._sem_on = bool(sem_inlet) and self.dims == 3 and inlet_bc == "velocity" and streamwise_bc == "open"
        if self._sem_on:
            self._inflow_on = False
            g = np.random.default_rng(0)
            self._sem = dict(Tu=float(sem_Tu), sig=float(sem_L_int), N=int(sem_N), rng=g)
            r = 3.0 * float(sem_L_int)
            n = int(sem_N)
            self._sem["x"] = g.uniform(-r, r, n)
            self._sem["y"] = g.uniform(0.0, float(self.ny), n)
            self._sem["z"] = g.uniform(0.0, float(self.nz), n)
            self._sem["eps"] = g.choice(np.array([-1.0, 1.0]), size=(3, n)).astype(np.float64)
        s.sponge_thickness = int(sponge_thickness)
        s.thermal = int(bool(thermal))
        s.buoyancy = int(bool(buoyancy))
        s.scalar_reduced = int(reduced)
        s.n_links = len(self.links)
        s.omega, s.u0, s.rho_in, s.rho_out = omega, u0, rho_in, rho_out
        s.inlet_perturbation = max(float(inlet_perturbation), 0.0)
        s.trt_lambda, s.sponge_strength, s.les_cs = trt_lambda, sponge_strength, les_cs
        s.van_driest_A = van_driest_A
        s.wall_velocity_top, s.wall_velocity_bottom = wall_velocity_top, wall_velocity_bottom
        s.body_force[:] = [body_force_x, body_force_y, body_force_z]
        s.omega_T = 1.0 / (alpha_scale * alpha_T + 0.5)
        s.T_hot, s.T_cold, s.g_gravity, s.beta, s.T_ref = T_hot, T_cold, g_gravity, beta, T_ref
        s.center[:] = ctr
        self._s_struct = s
        self.step_count = 0
        self.nprof = self.nz if self.dims == 3 else self.ny
        if threads is not None:
            os.environ["OMP_NUM_THREADS"] = str(int(threads))

    # feq for the current lattice (aero/lbm/d2q9.py:66-89, d3q19.py:105-129)
    def feq(self, rho, ux, uy=None, uz=None):
        uy = np.zeros_like(rho) if uy is None else uy
        uz = np.zeros_like(rho) if uz is None else uz
        usq = ux * ux + uy * uy + uz * uz
        out = np.empty((self.Q,) + rho.shape)
        for i in range(self.Q):
            e = self.E[i]
            eu = e[0] * ux + e[1] * uy + (e[2] * uz if self.dims == 3 else 0.0)
            out[i] = self.W[i] * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * usq)
        return out

    def _bind(self):
        s = self._s_struct
        self.f = np.ascontiguousarray(self.f, dtype=np.float64)
        self.f_outlet_prev = np.ascontiguousarray(self.f_outlet_prev, dtype=np.float64)
        if self.g is not None:
            self.g = np.ascontiguousarray(self.g, dtype=np.float64)
        s.f, s.g, s.f_outlet_prev = _ptr(self.f), _ptr(self.g), _ptr(self.f_outlet_prev)
        s.solid, s.phi = _ptr(self.solid_u8), _ptr(self.phi)
        s.links, s.q_vals = _ptr(self.links), _ptr(self.q)
        s.mrt_M, s.mrt_Minv, s.mrt_s = _ptr(self._M), _ptr(self._Minv), _ptr(self._s)
        s.work_a, s.work_b = _ptr(self._work_a), _ptr(self._work_b)
        s.work_om, s.work_g = _ptr(self._work_om), _ptr(self._work_g)
        s.step_count = self.step_count

    def _next_inflow(self):
        """The next step's transverse inlet velocities, as the reference draws them."""
        rng, t = self._inflow_rng, self._inflow_target
        if self.dims == 2:
            n = rng.standard_normal(self.ny)
            filt = (n + np.roll(n, 1) + np.roll(n, -1)) / 3.0
            u = 0.75 * self._inflow_u[0] + 0.25 * filt
            u = u - float(np.mean(u))
            rms = float(np.sqrt(np.mean(u ** 2)))
            if rms > 1e-12 and t > 0.0:
                u = u * (t / rms)
            self._inflow_u = [u]
        else:
            raw = [rng.standard_normal((self.nz, self.ny)), rng.standard_normal((self.nz, self.ny))]
            new = []
            for prev, n in zip(self._inflow_u, raw):
                sm = (n + np.roll(n, 1, 0) + np.roll(n, -1, 0) + np.roll(n, 1, 1) + np.roll(n, -1, 1)) / 5.0
                u = 0.8 * prev + 0.2 * sm
                new.append(u - float(np.mean(u)))
            rms = float(np.sqrt(np.mean(new[0] ** 2 + new[1] ** 2)))
            if rms > 1e-12 and t > 0.0:
                new = [u * (t / rms) for u in new]
            self._inflow_u = new
        return np.ascontiguousarray(np.stack(self._inflow_u), dtype=np.float64)

    def _next_sem(self):
        """Advance the eddies one step and return (u', v', w') as (3, nz, ny)."""
        S = self._sem
        g, sig, N, r = S["rng"], S["sig"], S["N"], 3.0 * S["sig"]
        S["x"] = S["x"] + self.u0
        out = S["x"] > r
        k = int(out.sum())
        if k:
            S["x"][out] = -r
            S["y"][out] = g.uniform(0.0, float(self.ny), k)
            S["z"][out] = g.uniform(0.0, float(self.nz), k)
            S["eps"][:, out] = g.choice(np.array([-1.0, 1.0]), size=(3, k)).astype(np.float64)
        shape = (self.nz, self.ny)
        if S["Tu"] <= 0.0 or sig <= 0.0 or N == 0:
            return np.zeros((3,) + shape)
        zz, yy = np.meshgrid(np.arange(self.nz) + 0.5, np.arange(self.ny) + 0.5, indexing="ij")
        dist = np.sqrt(S["x"][:, None, None] ** 2 + (yy[None] - S["y"][:, None, None]) ** 2
                       + (zz[None] - S["z"][:, None, None]) ** 2)
        tent = np.maximum(0.0, 1.0 - dist / sig)
        comp = [(S["eps"][c][:, None, None] * tent).sum(axis=0) / np.sqrt(float(N)) for c in range(3)]
        vh, wh = np.fft.fft2(comp[1]), np.fft.fft2(comp[2])
        if self.nz % 2 == 0:
            vh[self.nz // 2, :] = 0.0
            wh[self.nz // 2, :] = 0.0
        if self.ny % 2 == 0:
            vh[:, self.ny // 2] = 0.0
            wh[:, self.ny // 2] = 0.0
        kz = (np.fft.fftfreq(self.nz) * 2 * np.pi)[:, None]
        ky = (np.fft.fftfreq(self.ny) * 2 * np.pi)[None, :]
        k2 = kz ** 2 + ky ** 2
        k2[0, 0] = 1.0
        dv = ky * vh + kz * wh
        v = np.real(np.fft.ifft2(vh - ky / k2 * dv))
        w = np.real(np.fft.ifft2(wh - kz / k2 * dv))
        t = S["Tu"] * self.u0
        su = float(np.std(comp[0]))
        svw = float(np.sqrt(np.mean(v ** 2 + w ** 2) / 2.0))
        u = comp[0] * (t / su) if su > 1e-14 else np.zeros(shape)
        v, w = ((v * (t / svw), w * (t / svw)) if svw > 1e-14 else (np.zeros(shape), np.zeros(shape)))
        return np.stack([u, v, w])

    def step_raw(self):
        """One step; returns (raw 12-vector of forces/moments, profile (nprof, 3))."""
        self._bind()
        if self._sem_on:
            self._sem_buf = np.ascontiguousarray(self._next_sem(), dtype=np.float64)
            self._s_struct.sem = self._sem_buf.ctypes.data
        if self._inflow_on:
            self._inflow_buf = self._next_inflow()
            self._s_struct.inflow = self._inflow_buf.ctypes.data
        out = np.zeros(12)
        prof = np.zeros((self.nprof, 3))
        rc = lib().oracle_step(ctypes.byref(self._s_struct), out.ctypes.data, prof.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"oracle_step failed ({rc})")
        self.step_count += 1
        return out, prof

    def step(self):
        """One step; returns a dict of coefficients (forces.py:78-139, forces3d.py:70-145)."""
        raw, prof = self.step_raw()
        return coefficients(raw, self.dims, self.rho0, self.u0, self.D), prof

    def collide_only(self):
        self._bind()
        out = np.empty_like(self.f)
        lib().oracle_collide_only(ctypes.byref(self._s_struct), out.ctypes.data)
        return out

    def omega_field(self):
        self._bind()
        out = np.empty(self.solid.shape)
        lib().oracle_omega_field(ctypes.byref(self._s_struct), out.ctypes.data)
        return out


def coefficients(raw: np.ndarray, dims: int, rho0: float, u0: float, D: float) -> dict:
    """Coefficient normalisation: 2D 0.5 rho u^2 D (moment x D), 3D 0.5 rho u^2 D^2."""
    fdyn = 0.5 * rho0 * u0 * u0 * D * (D if dims == 3 else 1.0)
    mdyn = fdyn * D
    if fdyn == 0.0:
        return {k: 0.0 for k in ("Cd", "Cl", "Cly", "Clz", "Cm", "Cmx", "Cmy", "Cmz", "Cd_p", "Cd_v")}
    c = {
        "Cd": raw[0] / fdyn, "Cd_p": raw[3] / fdyn, "Cd_v": raw[6] / fdyn,
    }
    if dims == 2:
        c.update(Cl=raw[1] / fdyn, Cm=raw[11] / mdyn)
    else:
        c.update(Cly=raw[1] / fdyn, Clz=raw[2] / fdyn, Cmx=raw[9] / mdyn, Cmy=raw[10] / mdyn,
                 Cmz=raw[11] / mdyn)
    return c
