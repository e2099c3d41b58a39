"""Shared host logic of Solver (2D) and Solver3D: state mirroring, stepping,
force histories, run loop and checkpoints.

The public behaviour follows the reference solvers (aero/lbm/solver.py:74-727,
aero/lbm/solver3d.py:70-838): same constructor options, same attributes
(f, g, _f_outlet_prev, surface_links, q_vals, step_count, *_history), same
_step() return values and run() result keys, same .npz checkpoint keys.  What
changes is where the step runs: on the GPU, many steps per call, with the
per-step forces kept in a device ring and read back in chunks.
"""

from __future__ import annotations

import json
import os
import pathlib
import threading
import time
import warnings
from typing import Optional

import numpy as np

from . import _lib
from .diagnostics import FieldHealth, detect_statistical_stationarity
from .engine import Engine, copy_to_host
from .lattice import feq, macroscopic, scalar_weights, tables
from .links import build_surface_links

BACKENDS = ("b200", "auto")
PRECISIONS = tuple(_lib.STORE)
_PRISTINE_LIMIT = 1 << 28  # elements; above this a handed-out array is always re-uploaded


LAYOUTS = {"ab": 0, "aa": 1}


def _check_layout(layout: str) -> None:
    """Population layout: "ab" (two buffers; every step kernel), "aa" (one
    buffer updated in place, the AA pattern: half the population memory; the
    per-cell step kernel only; in batches with at least 2^20 cells) or
    "auto" (the faster "ab" when its workspace fits the device's free memory
    with headroom, else "aa"; the choice is in the solver's `layout`
    attribute)."""
    if layout not in LAYOUTS and layout != "auto":
        raise ValueError(f"Unknown layout '{layout}'. Choose 'ab', 'aa' or 'auto'.")


def _open_checkpoint(path: str):
    """np.load of a checkpoint, with a truncated or corrupt file reported as
    ValueError (before anything touches the GPU)."""
    import zipfile
    import zlib
    try:
        with np.load(path, allow_pickle=False) as npz:
            return {k: npz[k] for k in npz.files}
    except (OSError, ValueError, EOFError, KeyError, zipfile.BadZipFile, zlib.error) as e:
        raise ValueError(f"corrupt or unreadable checkpoint {path}: {e}") from e


class LatticeSolverBase:
    dims = 2

    # ------------------------------------------------------------------ set-up
    def _setup(self, *, shape, solid, omega, u0, D, rho0, wall_bc, inlet_bc, outlet_bc,
               streamwise_bc, backend, collision, inlet_perturbation, trt_lambda,
               sponge_thickness, sponge_strength, les, les_cs, les_model, ibm_enabled, phi,
               bouzidi, van_driest, van_driest_A, body_force, wall_velocity_top,
               wall_velocity_bottom, synthetic_inflow, synthetic_inflow_intensity,
               synthetic_inflow_seed, thermal, T_hot, T_cold, alpha_T, buoyancy, g_gravity, beta,
               T_ref, precision, scalar_lattice, device, hist_capacity, rho_in=1.0, rho_out=1.0, sem=None,
               layout="ab"):
        if backend not in BACKENDS:
            raise ValueError(f"Unknown backend '{backend}'. Choose 'b200' or 'auto'.")
        if collision not in ("bgk", "mrt", "trt"):
            raise ValueError(f"Unknown collision '{collision}'. Choose 'bgk', 'mrt', or 'trt'.")
        if les_model not in ("smagorinsky", "wale"):
            raise ValueError("les_model must be 'smagorinsky' or 'wale'.")
        if precision not in PRECISIONS:
            raise ValueError(f"Unknown precision '{precision}'. Choose one of {PRECISIONS}.")
        if scalar_lattice not in ("full", "reduced"):
            raise ValueError("scalar_lattice must be 'full' or 'reduced'.")
        if ibm_enabled:
            raise NotImplementedError("ibm_enabled: immersed-boundary forcing is not part of the b200 engine")
        self.backend = "b200"
        self.solid = np.ascontiguousarray(solid, dtype=np.bool_)
        if self.solid.shape != tuple(shape):
            raise ValueError(f"solid has shape {self.solid.shape}, expected {tuple(shape)}")
        self.fluid = ~self.solid
        self.omega = float(omega)
        self.u0 = float(u0)
        self.D = float(D)
        self.rho0 = float(rho0)
        self.wall_bc = wall_bc
        self.inlet_bc = inlet_bc
        self.outlet_bc = outlet_bc
        self.rho_in = float(rho_in)
        self.rho_out = float(rho_out)
        self.collision = collision
        self.inlet_perturbation = max(float(inlet_perturbation), 0.0)
        self.trt_lambda = float(trt_lambda)
        self.sponge_thickness = int(sponge_thickness)
        self.sponge_strength = float(sponge_strength)
        self.les = bool(les)
        self.les_cs = float(les_cs)
        self.les_model = str(les_model)
        self.ibm_enabled = False
        self.phi = phi
        self.bouzidi = bool(bouzidi)
        self.van_driest = bool(van_driest)
        self.van_driest_A = float(van_driest_A)
        self.wall_velocity_top = float(wall_velocity_top)
        self.wall_velocity_bottom = float(wall_velocity_bottom)
        self.synthetic_inflow = bool(synthetic_inflow)
        self.synthetic_inflow_intensity = float(synthetic_inflow_intensity)
        self.synthetic_inflow_seed = int(synthetic_inflow_seed)
        self.thermal = bool(thermal)
        self.T_hot = float(T_hot)
        self.T_cold = float(T_cold)
        self.alpha_T = float(alpha_T)
        self.scalar_lattice = scalar_lattice
        cs2inv = 4.0 if (scalar_lattice == "reduced" and self.dims == 3) else 3.0
        self.omega_T = float(1.0 / (cs2inv * alpha_T + 0.5))
        self.buoyancy = bool(buoyancy)
        self.g_gravity = float(g_gravity)
        self.beta = float(beta)
        self.T_ref = float(T_ref)
        self.tau = 1.0 / self.omega
        self._base_nu = (self.tau - 0.5) / 3.0
        self.precision = precision
        self.streamwise_bc = streamwise_bc
        self._body_force = tuple(float(v) for v in body_force)

        phi_q = phi if (bouzidi and phi is not None) else None
        self.surface_links, self.q_vals = build_surface_links(self.solid, phi_q)
        idx = np.nonzero(self.solid)
        ctr = [float(np.mean(a)) if a.size else 0.5 * (n - 1) for a, n in zip(idx, self.solid.shape)]
        self._ref_center = ctr[::-1] + ([0.0] if self.dims == 2 else [])  # (x, y, z)

        P = _lib.AeroParams()
        P.abi_version = _lib.ABI_VERSION
        P.dims = self.dims
        if self.dims == 2:
            P.ny, P.nx = shape
            P.nz = 1
        else:
            P.nz, P.ny, P.nx = shape
        P.storage = _lib.STORE[precision]
        P.collision = _lib.COLLISION[collision]
        P.inlet_bc = _lib.INLET.get(inlet_bc, 0)
        if self.dims == 2:
            P.outlet_bc = _lib.OUTLET.get(outlet_bc, 0)
        else:  # solver3d.py:454-457: anything but "convective" is zero-gradient
            P.outlet_bc = _lib.OUTLET["convective"] if outlet_bc == "convective" else _lib.OUTLET["zerogradient"]
        P.wall_bc = _lib.WALL.get(wall_bc, 0)
        P.streamwise_open = 1 if streamwise_bc == "open" else 0
        P.les = int(self.les)
        P.les_model = _lib.LES_MODEL[les_model]
        P.van_driest = int(self.van_driest and phi is not None)
        P.bouzidi = int(self.bouzidi)
        P.thermal = int(self.thermal)
        P.buoyancy = int(self.buoyancy)
        P.scalar_reduced = int(scalar_lattice == "reduced")
        P.sponge_thickness = self.sponge_thickness
        P.hist_capacity = int(hist_capacity)
        P.omega, P.u0, P.rho0 = self.omega, self.u0, self.rho0
        P.rho_in, P.rho_out = self.rho_in, self.rho_out
        P.inlet_perturbation = self.inlet_perturbation
        P.trt_lambda = self.trt_lambda
        P.sponge_strength = self.sponge_strength
        P.les_cs, P.van_driest_A = self.les_cs, self.van_driest_A
        P.wall_velocity_top, P.wall_velocity_bottom = self.wall_velocity_top, self.wall_velocity_bottom
        P.body_force[:] = list(self._body_force)
        P.alpha_T, P.T_hot, P.T_cold = self.alpha_T, self.T_hot, self.T_cold
        P.g_gravity, P.beta, P.T_ref = self.g_gravity, self.beta, self.T_ref
        P.center[:] = self._ref_center
        # synthetic inflow only drives an open velocity inlet (solver.py:385-392,
        # solver3d.py:432-445); the fields come from the reference's random stream
        self._inflow = None
        if sem is not None and self.dims == 3 and inlet_bc == "velocity" and streamwise_bc == "open":
            # SEM takes precedence over synthetic inflow (solver3d.py:433-445)
            from .inflow import SEMInflow
            self._inflow = SEMInflow(shape[-2], shape[0], self.u0, sem[0], sem[1], sem[2])
            P.inflow_field = 2
            P.inflow_ring = 64
        elif self.synthetic_inflow and inlet_bc == "velocity" and (self.dims == 2 or streamwise_bc == "open"):
            from .inflow import SyntheticInflow
            nz_ = shape[0] if self.dims == 3 else 1
            self._inflow = SyntheticInflow(self.dims, shape[-2], nz_, self.u0, self.synthetic_inflow_intensity,
                                           self.synthetic_inflow_seed)
            P.inflow_field = 1
            P.inflow_ring = 64
        P.recycling = 1 if (self.dims == 3 and streamwise_bc == "recycling") else 0
        P.layout = LAYOUTS["ab" if layout == "auto" else layout]
        self._params = P
        self._engine_phi = phi if (self.van_driest and phi is not None) else None
        self._engine = Engine(P, self.solid, self.surface_links, self.q_vals, self._engine_phi, device,
                              layout_auto=layout == "auto")
        self.layout = "aa" if P.layout == LAYOUTS["aa"] else "ab"

        # initial state: equilibrium at (rho0, u0, 0) everywhere, solids included
        # (solver.py:218-227, solver3d.py:239-247); built on the GPU
        e, w, _ = tables(self.dims)
        self.Q = len(w)
        self.step_count = 0
        self._f_host = self._prev_host = self._g_host = None
        self._pristine = {}
        self._engine.set_equilibrium()
        self._init_histories()

    def _uniform_state_device(self, ux=None, uy=None):
        """Equilibrium populations for rho0 and velocity (ux, uy, 0) as device
        tensors; ux defaults to u0 and uy to 0 everywhere.  Also returns the
        matching outlet column and the scalar at T_ref."""
        import torch
        dev = self._engine.device
        shape = self.solid.shape
        if ux is None and uy is not None:
            ux = torch.full(tuple(shape), self.u0, dtype=torch.float64, device=dev)
        if ux is None:
            vec = feq(self.dims, np.array(self.rho0), np.array(self.u0), np.array(0.0),
                      np.array(0.0) if self.dims == 3 else None)
            f0 = torch.tensor(vec, dtype=torch.float64, device=dev).reshape(
                (self.Q,) + (1,) * self.dims).expand((self.Q,) + tuple(shape)).contiguous()
        else:
            rho = torch.full(tuple(shape), self.rho0, dtype=torch.float64, device=dev)
            zero = torch.zeros_like(rho)
            f0 = feq(self.dims, rho, ux, zero if uy is None else uy, zero if self.dims == 3 else None, xp=torch)
        prev0 = f0[..., -1].contiguous()
        g0 = None
        if self.thermal:
            wg = scalar_weights(self.dims, self.scalar_lattice == "reduced")
            g0 = (torch.tensor(wg * self.T_ref, dtype=torch.float64, device=dev).reshape(
                (-1,) + (1,) * self.dims).expand((len(wg),) + tuple(shape)).contiguous())
        return f0, prev0, g0

    # ------------------------------------------------------------------ state
    def set_equilibrium_state(self, rho=None, ux=None, uy=None, uz=None, T=None) -> None:
        """Sets the state to the equilibrium of macroscopic fields -- what
        ``s.f = compute_feq(rho, ux, uy[, uz])`` with the outlet state taken
        from its last column and, with a scalar, ``s.g = w T`` would set --
        built on the GPU from the fields (no counterpart in the reference).
        One value per cell crosses to the device for each field given,
        instead of Q populations.  Each field is an array of the lattice
        shape (numpy or torch, host or device) or None for the uniform value
        (rho0, u0, 0, 0, T_ref).  The step count is kept."""
        if uz is not None and self.dims != 3:
            raise ValueError("uz is a 3D field")
        if T is not None and not self.thermal:
            raise ValueError("T needs thermal=True")
        self._handed = set()
        self._f_host = self._prev_host = self._g_host = None
        self._pristine = {}
        self._engine.set_equilibrium(rho, ux, uy, uz, T, self.step_count)

    def _cache(self):
        if self._f_host is None:
            f, p, g = self._engine.get_state()
            self._f_host, self._prev_host, self._g_host = f, p, g
            self._pristine = {}
            for k, a in (("f", f), ("prev", p), ("g", g)):
                if a is not None and a.size <= _PRISTINE_LIMIT:
                    self._pristine[k] = a.copy()

    def _mark_handed(self, key):
        self._handed = getattr(self, "_handed", set())
        self._handed.add(key)

    @property
    def f(self) -> np.ndarray:
        self._cache()
        self._mark_handed("f")
        return self._f_host

    @f.setter
    def f(self, value):
        self._cache()
        self._f_host = np.ascontiguousarray(value, dtype=np.float64)
        self._pristine.pop("f", None)
        self._mark_handed("f")

    @property
    def _f_outlet_prev(self) -> np.ndarray:
        self._cache()
        self._mark_handed("prev")
        return self._prev_host

    @_f_outlet_prev.setter
    def _f_outlet_prev(self, value):
        self._cache()
        self._prev_host = np.ascontiguousarray(value, dtype=np.float64)
        self._pristine.pop("prev", None)
        self._mark_handed("prev")

    @property
    def g(self) -> Optional[np.ndarray]:
        if not self.thermal:
            return None
        self._cache()
        self._mark_handed("g")
        return self._g_host

    @g.setter
    def g(self, value):
        if not self.thermal:
            if value is not None:
                raise ValueError("g can only be set when thermal=True")
            return
        self._cache()
        self._g_host = np.ascontiguousarray(value, dtype=np.float64)
        self._pristine.pop("g", None)
        self._mark_handed("g")

    def _flush_host_state(self):
        """Uploads host-side edits of f / _f_outlet_prev / g before stepping."""
        handed = getattr(self, "_handed", set())
        if handed and self._f_host is not None:
            changed = False
            for k, a in (("f", self._f_host), ("prev", self._prev_host), ("g", self._g_host)):
                if k not in handed or a is None:
                    continue
                ref = self._pristine.get(k)
                if ref is None or ref.shape != a.shape or not np.array_equal(ref, a):
                    changed = True
            if changed:
                self._engine.set_state(self._f_host, self._prev_host, self._g_host, self.step_count)
        self._handed = set()
        self._f_host = self._prev_host = self._g_host = None
        self._pristine = {}

    # ------------------------------------------------------------------ stepping
    def _advance(self, n: int) -> np.ndarray:
        """Runs n steps on the GPU and returns their raw force rows (n, 12)."""
        self._flush_host_state()
        rows = []
        left = int(n)
        cap = self._engine.hist_capacity
        ring = self._params.inflow_ring if self._inflow is not None else cap
        while left > 0:
            k = min(left, cap, ring)
            if self._inflow is not None:
                self._engine.set_inflow(self._inflow.fields(k), self.step_count + int(n) - left)
            self._engine.step(k)
            rows.append(self._engine.read_forces(k))
            left -= k
        self.step_count += int(n)
        raw = np.concatenate(rows) if rows else np.zeros((0, 12))
        if len(raw):
            self._set_last(raw[-1], self._engine.read_profile())
        return raw

    def _step(self):
        raw = self._advance(1)
        c = self._coefficients(raw)
        return self._step_return(c, 0)

    def autotune(self, steps: int = 20) -> dict:
        """Selects the fastest step kernel for this lattice by timing each one
        (see aero_b200.autotune); call before the first step."""
        from .autotune import autotune
        return autotune(self, steps=steps)

    def _drag_norm(self) -> float:
        """Force that makes Cd = 1: 0.5 rho0 u0^2 D (2D, forces.py:78-103) or
        0.5 rho0 u0^2 D^2 (3D, forces3d.py:70-101)."""
        fdyn = 0.5 * self.rho0 * self.u0 * self.u0 * self.D * (self.D if self.dims == 3 else 1.0)
        return fdyn if fdyn > 0.0 else 1.0

    def status(self) -> int:
        """Device divergence flags (bit 0: non-finite or non-positive density seen)."""
        return self._engine.status()

    def field_statistics(self) -> dict:
        """FP64 statistics of the whole current state, reduced on the GPU
        (no counterpart in the reference): the mass (sum of rho), mean
        density, largest |(ux, uy)|, NaN populations, cells with rho <= 0 and,
        with a scalar, its total and the Nusselt numbers at the two Dirichlet
        rows (mean -dT/dy at the row times (Ny - 1) / (T_hot - T_cold))."""
        self._flush_host_state()
        h = FieldHealth.from_stats(self._engine.field_stats())
        out = {"mass": h.mass, "mean_density": h.mean_density, "max_speed": h.max_speed,
               "nan_populations": h.nan_populations, "nonpositive_cells": h.nonpositive_cells,
               "cells": h.cells}
        if self.thermal:
            nu = h.nusselt(float(self.solid.shape[-2] - 1), self.T_hot - self.T_cold) or (None, None)
            out.update(scalar_total=h.scalar_total, Nu_bottom=nu[0], Nu_top=nu[1])
        return out

    # ------------------------------------------------------------------ checkpoints
    def save_checkpoint(self, path: str) -> None:
        """Writes the reference's checkpoint (solver.py:638-686,
        solver3d.py:727-780): the same keys and dtypes, params_json holding
        exactly the reference constructor's keywords (so the reference's
        from_checkpoint can rebuild the solver; backend "numpy" as the 3D
        reference writes it), and one extra key the reference ignores,
        b200_options, with the engine's own options (precision, scalar
        lattice)."""
        params = self._checkpoint_params()
        params["backend"] = "numpy"
        f = self.f
        kwargs = dict(
            f=f, f_outlet_prev=self._f_outlet_prev, solid=self.solid,
            surface_links=self.surface_links, q_vals=self.q_vals,
            step_count=np.array(self.step_count, dtype=np.int64),
            params_json=np.array(json.dumps(params)),
            b200_options=np.array(json.dumps(self._b200_options())),
            **{k: np.array(getattr(self, k), dtype=np.float64) for k in self._history_keys()},
        )
        if self.phi is not None:
            kwargs["phi"] = self.phi
        if self.thermal:
            kwargs["g"] = self.g
        np.savez_compressed(path, **kwargs)

    def _b200_options(self) -> dict:
        return {"precision": self.precision, "scalar_lattice": self.scalar_lattice, "layout": self.layout}

    def load_checkpoint(self, path: str) -> None:
        """Restores f, the outlet state, the scalar, the histories and the
        step count, and adopts the checkpoint's surface links and q values
        when it has them (solver.py:688-709, solver3d.py:782-811).  A link
        table that differs from the one built from the solid mask is
        uploaded to the engine (which checks it against the mask)."""
        data = _open_checkpoint(path)
        for key in ("f", "f_outlet_prev", "step_count"):
            if key not in data:
                raise ValueError(f"checkpoint {path} has no '{key}' entry")
        if tuple(data["f"].shape) != (self.Q,) + tuple(self.solid.shape):
            raise ValueError(f"checkpoint {path}: f has shape {tuple(data['f'].shape)}, "
                             f"the solver needs {(self.Q,) + tuple(self.solid.shape)}")
        links, q = data.get("surface_links"), data.get("q_vals")
        if links is not None and q is not None and (
                links.shape != self.surface_links.shape or not np.array_equal(links, self.surface_links)
                or not np.array_equal(q, self.q_vals)):
            if links.ndim != 2 or links.shape[1] != self.dims + 1 or len(q) != len(links):
                raise ValueError(f"checkpoint {path}: surface_links / q_vals have shapes {links.shape} / {q.shape}")
            self._adopt_links(np.ascontiguousarray(links, dtype=np.int32), np.ascontiguousarray(q, dtype=np.float32))
        for k in self._history_keys():
            if k in data:
                setattr(self, k, list(data[k]))
        self.step_count = int(data["step_count"])
        g = data["g"] if ("g" in data and self.thermal) else None
        if self.thermal and g is None:
            g = self.g
        self._handed = set()
        self._f_host = None
        self._engine.set_state(data["f"], data["f_outlet_prev"], g, self.step_count)

    def _adopt_links(self, links: np.ndarray, q: np.ndarray) -> None:
        """A new engine for this lattice with the given link table (the step
        kernel choice returns to the default)."""
        P, dev = self._params, self._engine.device
        old = self._engine
        self._engine = Engine(P, self.solid, links, q, self._engine_phi, dev)
        del old
        self.surface_links, self.q_vals = links, q

    @classmethod
    def from_checkpoint(cls, path: str, backend: Optional[str] = None, **overrides):
        """Rebuilds a solver from a checkpoint of this engine or of the
        reference: the constructor keywords from params_json (the reference's
        backend name replaced by "b200"), this engine's options from
        b200_options when present, then `overrides`."""
        data = _open_checkpoint(path)
        for key in ("params_json", "solid"):
            if key not in data:
                raise ValueError(f"checkpoint {path} has no '{key}' entry")
        try:
            params = json.loads(str(data["params_json"]))
            extra = json.loads(str(data["b200_options"])) if "b200_options" in data else {}
        except json.JSONDecodeError as e:
            raise ValueError(f"checkpoint {path}: unreadable params_json ({e})") from e
        params.update(extra)
        params["backend"] = "b200"
        params.update(overrides)
        solid = data["solid"]
        phi = data["phi"] if "phi" in data else None
        s = cls(solid=solid, phi=phi, **params)
        s.load_checkpoint(path)
        return s

    # ------------------------------------------------------------------ run loop
    def run(self, steps: int, check_every: int = 500, verbose: bool = True, callback=None,
            checkpoint_every: Optional[int] = None, checkpoint_dir: Optional[str] = None,
            auto_stop: bool = False, convergence_window: int = 5000, convergence_tol: float = 0.01,
            strouhal_window: int = 4096, strouhal_tol: float = 0.05, hdf5_path: Optional[str] = None,
            hdf5_every: Optional[int] = None) -> dict:
        """Runs ``steps`` steps with the semantics of Solver.run (solver.py:470-632)."""
        if verbose:
            self._print_banner()
        if hdf5_path:
            warnings.warn("hdf5_path is ignored by the b200 backend (h5py output is not part of the "
                          "engine)", RuntimeWarning)
        t0 = time.perf_counter()
        if self.dims == 3:
            # host arrays for the result's fields, their pages touched by a
            # helper thread while the GPU steps (a gigabyte of fresh pages
            # otherwise costs as long as the copy itself)
            self._field_host = _HostBuffer((4,) + tuple(self.solid.shape))
        avg_window = max(1, steps // 5)
        stop_reason = "max_steps"
        last_conv = last_st = None
        step = 0
        check_every = max(int(check_every), 1)
        while step < steps:
            nxt = steps
            nxt = min(nxt, (step // check_every + 1) * check_every)
            if checkpoint_every and checkpoint_dir:
                nxt = min(nxt, (step // checkpoint_every + 1) * checkpoint_every)
            raw = self._advance(nxt - step)
            self._append_histories(self._coefficients(raw))
            step = nxt
            if checkpoint_every and checkpoint_dir and step % checkpoint_every == 0:
                self.save_checkpoint(str(pathlib.Path(checkpoint_dir) / self._checkpoint_name()))
            if step % check_every == 0:
                macro = self._stability_check(step, want_fields=callback is not None)
                elapsed = time.perf_counter() - t0
                if verbose:
                    self._print_progress(step, steps, check_every, step / max(elapsed, 1e-12))
                if callback is not None:
                    self._callback(callback, step, macro)
                if auto_stop:
                    last_conv, last_st, stop = detect_statistical_stationarity(
                        self.Cd_history, self._lift_history_for_stop(strouhal_window), self.D, self.u0,
                        convergence_window=convergence_window, convergence_tol=convergence_tol,
                        strouhal_window=strouhal_window, strouhal_tol=strouhal_tol)
                    if stop:
                        stop_reason = "auto_converged"
                        break
        return self._result(avg_window, stop_reason, last_conv, last_st)

    # ------------------------------------------------------------------ helpers
    def _scalar_stats(self):
        if not self.thermal:
            return None, None
        T = self._scalar_field()
        return T, {
            "enabled": True, "mean": float(np.mean(T)), "std": float(np.std(T)),
            "min": float(np.min(T)), "max": float(np.max(T)), "wall_hot": float(self.T_hot),
            "wall_cold": float(self.T_cold), "diffusivity": float(self.alpha_T),
            "buoyancy": bool(self.buoyancy), "gravity": float(self.g_gravity),
            "beta": float(self.beta), "reference": float(self.T_ref),
        }

    def _scalar_field(self) -> np.ndarray:
        _, _, g = self._engine.get_state_device(want_prev=False, want_g=True)
        return g.sum(dim=0).cpu().numpy()

    def _macroscopic_host(self):
        """rho, u of the current state as host arrays: computed on the GPU from
        the population buffers (aero_get_macroscopic) and copied into the
        arrays run() prepared, or fresh ones."""
        t0 = time.perf_counter()
        dev = self._engine.macroscopic_device()
        buf = getattr(self, "_field_host", None)
        self._field_host = None
        host = buf.get() if buf is not None and buf.shape == tuple(dev.shape) else np.empty(tuple(dev.shape))
        copy_to_host(dev, host)
        self._last_readback_s = time.perf_counter() - t0
        return tuple(host[k] for k in range(host.shape[0]))


class _HostBuffer:
    """A float64 host array for run()'s result fields whose pages helper
    threads touch in the background while the GPU steps, 16 MiB chunks dealt
    round-robin to up to 8 threads (the page faults of a fresh array are the
    cost: one thread needs about 115 ms per GB).  get() stops the helpers
    after their current chunks and hands the array over however far they
    got; the read-back faults in the rest from torch's threads."""

    _CHUNK = 1 << 21  # float64 values (16 MiB)

    def __init__(self, shape):
        self.shape = tuple(shape)
        self._a = np.empty(self.shape)
        self._stop = threading.Event()
        n = max(1, min(8, (os.cpu_count() or 1) // 2))
        self._t = [threading.Thread(target=self._fill, args=(k, n), daemon=True) for k in range(n)]
        for t in self._t:
            t.start()

    def _fill(self, k, n):
        flat = self._a.reshape(-1)
        for off in range(k * self._CHUNK, flat.size, n * self._CHUNK):
            if self._stop.is_set():
                return
            flat[off:off + self._CHUNK:512] = 0.0  # one write per 4 KiB page

    def get(self):
        self._stop.set()
        for t in self._t:
            t.join()
        return self._a
