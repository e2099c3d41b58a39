"""D2Q9 wind-tunnel solver running on the B200 engine.

Drop-in for the reference ``aero.lbm.solver.Solver`` (aero/lbm/solver.py:74-
727): same constructor options and defaults, ``_step()`` returning (Cd, Cl),
``run()`` returning the same result dict, ``f`` / ``g`` / ``_f_outlet_prev``
as readable and writable host arrays, and .npz checkpoints with the same
keys.  Extra options: ``precision`` ("fp32" default, "fp64", "fp16s",
"bf16s": populations stored as deviations from the rest weights),
``scalar_lattice`` ("full" = the reference's D2Q9 scalar, "reduced" = D2Q5),
``device`` and ``hist_capacity`` (steps of force history kept on the GPU).
"""

from __future__ import annotations

from typing import Optional

import numpy as np

from ._base import LatticeSolverBase, _check_layout
from .diagnostics import FieldHealth, check_field_health, coefficient_spectrum


class Solver(LatticeSolverBase):
    dims = 2

    def __init__(self, Ny: int, Nx: int, solid: np.ndarray, omega: float, u0: float, D: float,
                 rho0: float = 1.0, wall_bc: str = "slip", inlet_bc: str = "velocity",
                 outlet_bc: str = "convective", rho_in: float = 1.0, rho_out: float = 1.0,
                 backend: str = "b200", collision: str = "bgk", inlet_perturbation: float = 0.0,
                 trt_lambda: float = 0.25, sponge_thickness: int = 0, sponge_strength: float = 0.1,
                 les: bool = False, les_cs: float = 0.16, les_model: str = "smagorinsky",
                 ibm_enabled: bool = False, phi: Optional[np.ndarray] = None, bouzidi: bool = False,
                 van_driest: bool = False, van_driest_A: float = 25.0,
                 wall_velocity_top: float = 0.0, wall_velocity_bottom: float = 0.0,
                 synthetic_inflow: bool = False, synthetic_inflow_intensity: float = 0.03,
                 synthetic_inflow_seed: int = 12345, thermal: bool = False, T_hot: float = 1.0,
                 T_cold: float = 0.0, alpha_T: float = 1e-3, buoyancy: bool = False,
                 g_gravity: float = 0.0, beta: float = 1e-3, T_ref: float = 0.5,
                 precision: str = "fp32", scalar_lattice: str = "full", device=None,
                 hist_capacity: int = 4096, layout: str = "ab"):
        _check_layout(layout)
        self.Ny, self.Nx = int(Ny), int(Nx)
        self._setup(
            shape=(self.Ny, self.Nx), solid=solid, omega=omega, u0=u0, D=D, rho0=rho0,
            wall_bc=wall_bc, inlet_bc=inlet_bc, outlet_bc=outlet_bc, streamwise_bc="open",
            backend=backend, collision=collision, inlet_perturbation=inlet_perturbation,
            trt_lambda=trt_lambda, sponge_thickness=sponge_thickness,
            sponge_strength=sponge_strength, les=les, les_cs=les_cs, les_model=les_model,
            ibm_enabled=ibm_enabled, phi=phi, bouzidi=bouzidi, van_driest=van_driest,
            van_driest_A=van_driest_A, body_force=(0.0, 0.0, 0.0),
            wall_velocity_top=wall_velocity_top, wall_velocity_bottom=wall_velocity_bottom,
            synthetic_inflow=synthetic_inflow, synthetic_inflow_intensity=synthetic_inflow_intensity,
            synthetic_inflow_seed=synthetic_inflow_seed, thermal=thermal, T_hot=T_hot,
            T_cold=T_cold, alpha_T=alpha_T, buoyancy=buoyancy, g_gravity=g_gravity, beta=beta,
            T_ref=T_ref, precision=precision, scalar_lattice=scalar_lattice, device=device,
            hist_capacity=hist_capacity, rho_in=rho_in, rho_out=rho_out, layout=layout)
        self._ref_center_x, self._ref_center_y = self._ref_center[0], self._ref_center[1]
        self.rho = self.ux = self.uy = None

    # -------------------------------------------------------------- histories
    def _init_histories(self):
        self.Cd_history, self.Cl_history, self.Cm_history = [], [], []
        self.Cd_p_history, self.Cd_v_history = [], []

    def _history_keys(self):
        return ("Cd_history", "Cl_history", "Cm_history")

    def _coefficients(self, raw: np.ndarray) -> dict:
        """forces.py:78-139: force / (0.5 rho0 u0^2 D), moment / (... D^2)."""
        fdyn = 0.5 * self.rho0 * self.u0 * self.u0 * self.D
        mdyn = fdyn * self.D
        if fdyn == 0.0:
            z = np.zeros(len(raw))
            return {"Cd": z, "Cl": z, "Cm": z, "Cd_p": z, "Cd_v": z}
        return {"Cd": raw[:, 0] / fdyn, "Cl": raw[:, 1] / fdyn, "Cm": raw[:, 11] / mdyn,
                "Cd_p": raw[:, 3] / fdyn, "Cd_v": raw[:, 6] / fdyn}

    def _append_histories(self, c: dict):
        self.Cd_history.extend(c["Cd"].tolist())
        self.Cl_history.extend(c["Cl"].tolist())
        self.Cm_history.extend(c["Cm"].tolist())
        self.Cd_p_history.extend(c["Cd_p"].tolist())
        self.Cd_v_history.extend(c["Cd_v"].tolist())

    def _set_last(self, raw_row: np.ndarray, profile: np.ndarray):
        c = self._coefficients(raw_row[None, :])
        self._last_cm = float(c["Cm"][0])
        self._last_cd_p = float(c["Cd_p"][0])
        self._last_cd_v = float(c["Cd_v"][0])
        self._last_force_profile = {"y": list(range(self.Ny)), "fx": profile[:, 0].tolist(),
                                    "fy": profile[:, 1].tolist()}

    def _step_return(self, c: dict, k: int):
        return float(c["Cd"][k]), float(c["Cl"][k])

    def _lift_history_for_stop(self, window):
        return self.Cl_history

    # -------------------------------------------------------------- run hooks
    def _print_banner(self):
        print(f"  Backend   : {self.backend} ({self.precision})")
        print(f"  Collision : {self.collision}")

    def _print_progress(self, step, steps, check_every, sps):
        w = min(check_every, len(self.Cd_history))
        print(f"  step {step:6d}/{steps}  Cd={float(np.mean(self.Cd_history[-w:])):+.4f}  "
              f"Cl={float(np.mean(self.Cl_history[-w:])):+.4f}  [{sps:.0f} steps/s]", flush=True)

    def _stability_check(self, step, want_fields=False):
        # solver.py:522-531 checks the whole field; the device reduces it
        check_field_health(FieldHealth.from_stats(self._engine.field_stats()), step)
        if not want_fields:
            return None
        m = self._engine.macroscopic_device().cpu().numpy()
        return m[0], m[1], m[2]

    def _callback(self, callback, step, macro):
        rho, ux, uy = macro
        callback(step, self.Cd_history[-1], self.Cl_history[-1], rho, ux, uy)

    def _checkpoint_name(self):
        return f"checkpoint_{self.step_count:08d}.npz"

    def _checkpoint_params(self):
        return dict(
            Ny=self.Ny, Nx=self.Nx, omega=self.omega, u0=self.u0, D=self.D, rho0=self.rho0,
            wall_bc=self.wall_bc, inlet_bc=self.inlet_bc, outlet_bc=self.outlet_bc,
            rho_in=self.rho_in, rho_out=self.rho_out, inlet_perturbation=self.inlet_perturbation,
            trt_lambda=self.trt_lambda, sponge_thickness=self.sponge_thickness,
            sponge_strength=self.sponge_strength, les=self.les, les_cs=self.les_cs,
            ibm_enabled=self.ibm_enabled, les_model=self.les_model, bouzidi=self.bouzidi,
            van_driest=self.van_driest, van_driest_A=self.van_driest_A,
            wall_velocity_top=self.wall_velocity_top, wall_velocity_bottom=self.wall_velocity_bottom,
            synthetic_inflow=self.synthetic_inflow,
            synthetic_inflow_intensity=self.synthetic_inflow_intensity, thermal=self.thermal,
            T_hot=self.T_hot, T_cold=self.T_cold, alpha_T=self.alpha_T, buoyancy=self.buoyancy,
            g_gravity=self.g_gravity, beta=self.beta, T_ref=self.T_ref, collision=self.collision,
            backend=self.backend,
        )

    def _result(self, avg_window, stop_reason, last_conv, last_st) -> dict:
        f = self.f
        rho, ux, uy = _macro2(f)
        self.rho, self.ux, self.uy = rho, ux, uy
        tail = lambda h: np.array(h[-avg_window:]) if h else np.zeros(1)
        Cd, Cl, Cm = tail(self.Cd_history), tail(self.Cl_history), tail(self.Cm_history)
        Cdp, Cdv = tail(self.Cd_p_history), tail(self.Cd_v_history)
        scalar, scalar_stats = self._scalar_stats()
        return {
            "Cd_mean": float(np.mean(Cd)), "Cl_mean": float(np.mean(Cl)), "Cm_mean": float(np.mean(Cm)),
            "Cd_std": float(np.std(Cd)), "Cl_std": float(np.std(Cl)), "Cm_std": float(np.std(Cm)),
            "Cd_p_mean": float(np.mean(Cdp)), "Cd_v_mean": float(np.mean(Cdv)),
            "Cd_history": self.Cd_history, "Cl_history": self.Cl_history,
            "Cm_history": self.Cm_history, "Cd_p_history": self.Cd_p_history,
            "Cd_v_history": self.Cd_v_history,
            "observables": {
                "cd_spectrum": coefficient_spectrum(self.Cd_history),
                "cl_spectrum": coefficient_spectrum(self.Cl_history),
                "cm_spectrum": coefficient_spectrum(self.Cm_history),
                "force_profile_last": getattr(self, "_last_force_profile", None),
            },
            "steps_completed": self.step_count, "stop_reason": stop_reason,
            "convergence_report": last_conv, "strouhal_report": last_st,
            "rho": rho, "ux": ux, "uy": uy, "scalar": scalar, "scalar_stats": scalar_stats,
        }


def _macro2(f: np.ndarray):
    from .lattice import macroscopic
    return macroscopic(f, 2)
