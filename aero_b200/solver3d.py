"""D3Q19 wind-tunnel solver running on the B200 engine.

Drop-in for the reference ``aero.lbm.solver3d.Solver3D``
(aero/lbm/solver3d.py:70-838): same constructor options and defaults,
``_step()`` returning (Cd, Cl_y, Cl_z), ``run()`` with the same result dict,
host-visible ``f`` / ``g`` / ``_f_outlet_prev`` and .npz checkpoints.  Extra
options as for the 2D Solver (``precision``, ``scalar_lattice`` with
"reduced" = D3Q7, ``device``, ``hist_capacity``).  Streamwise "recycling",
synthetic inflow and the SEM inlet run in the engine.
"""

from __future__ import annotations

from typing import Optional

import numpy as np

from ._base import LatticeSolverBase, _check_layout
from .diagnostics import FieldHealth, check_field_health, coefficient_spectrum


class Solver3D(LatticeSolverBase):
    dims = 3

    def __init__(self, Nz: int, Ny: int, Nx: int, solid: np.ndarray, omega: float, u0: float,
                 D: float, rho0: float = 1.0, wall_bc: str = "slip", inlet_bc: str = "velocity",
                 outlet_bc: str = "convective", streamwise_bc: str = "open", backend: str = "b200",
                 collision: str = "bgk", inlet_perturbation: float = 0.0, trt_lambda: float = 0.25,
                 sponge_thickness: int = 0, sponge_strength: float = 0.1, les: bool = False,
                 les_cs: float = 0.16, les_model: str = "smagorinsky", ibm_enabled: bool = False,
                 phi: Optional[np.ndarray] = None, bouzidi: bool = False, van_driest: bool = False,
                 van_driest_A: float = 25.0, body_force_x: float = 0.0, body_force_y: float = 0.0,
                 body_force_z: float = 0.0, wall_velocity_top: float = 0.0,
                 wall_velocity_bottom: float = 0.0, synthetic_inflow: bool = False,
                 synthetic_inflow_intensity: float = 0.03, synthetic_inflow_seed: int = 12345,
                 sem_inlet: bool = False, sem_Tu: float = 0.05, sem_L_int: float = 10.0,
                 sem_N: int = 200, thermal: bool = False, T_hot: float = 1.0, T_cold: float = 0.0,
                 alpha_T: float = 1e-3, buoyancy: bool = False, g_gravity: float = 0.0,
                 beta: float = 1e-3, T_ref: float = 0.5, precision: str = "fp32",
                 scalar_lattice: str = "full", device=None, hist_capacity: int = 4096,
                 layout: str = "ab"):
        _check_layout(layout)
        if streamwise_bc not in ("open", "periodic", "recycling"):
            raise ValueError(
                f"Unknown streamwise_bc '{streamwise_bc}'. Choose 'open', 'periodic', or 'recycling'.")
        self.Nz, self.Ny, self.Nx = int(Nz), int(Ny), int(Nx)
        self.sem_inlet = bool(sem_inlet)
        self.sem_Tu, self.sem_L_int, self.sem_N = float(sem_Tu), float(sem_L_int), int(sem_N)
        self._setup(
            shape=(self.Nz, self.Ny, self.Nx), solid=solid, omega=omega, u0=u0, D=D, rho0=rho0,
            wall_bc=wall_bc, inlet_bc=inlet_bc, outlet_bc=outlet_bc, streamwise_bc=streamwise_bc,
            backend=backend, collision=collision, inlet_perturbation=inlet_perturbation,
            trt_lambda=trt_lambda, sponge_thickness=sponge_thickness,
            sponge_strength=sponge_strength, les=les, les_cs=les_cs, les_model=les_model,
            ibm_enabled=ibm_enabled, phi=phi, bouzidi=bouzidi, van_driest=van_driest,
            van_driest_A=van_driest_A, body_force=(body_force_x, body_force_y, body_force_z),
            wall_velocity_top=wall_velocity_top, wall_velocity_bottom=wall_velocity_bottom,
            synthetic_inflow=synthetic_inflow, synthetic_inflow_intensity=synthetic_inflow_intensity,
            synthetic_inflow_seed=synthetic_inflow_seed, sem=(float(sem_Tu), float(sem_L_int), int(sem_N))
            if sem_inlet else None, thermal=thermal, T_hot=T_hot,
            T_cold=T_cold, alpha_T=alpha_T, buoyancy=buoyancy, g_gravity=g_gravity, beta=beta,
            T_ref=T_ref, precision=precision, scalar_lattice=scalar_lattice, device=device,
            hist_capacity=hist_capacity, layout=layout)
        self.body_force_x, self.body_force_y, self.body_force_z = self._body_force
        self._ref_center_x, self._ref_center_y, self._ref_center_z = self._ref_center

    # -------------------------------------------------------------- histories
    def _init_histories(self):
        self.Cd_history, self.Cly_history, self.Clz_history = [], [], []
        self.Cmx_history, self.Cmy_history, self.Cmz_history = [], [], []
        self.Cd_p_history, self.Cd_v_history = [], []

    def _history_keys(self):
        return ("Cd_history", "Cly_history", "Clz_history", "Cmx_history", "Cmy_history",
                "Cmz_history")

    def _coefficients(self, raw: np.ndarray) -> dict:
        """forces3d.py:70-145: force / (0.5 rho0 u0^2 D^2), moment / (... D^3)."""
        fdyn = 0.5 * self.rho0 * self.u0 * self.u0 * self.D * self.D
        mdyn = fdyn * self.D
        keys = ("Cd", "Cly", "Clz", "Cmx", "Cmy", "Cmz", "Cd_p", "Cd_v")
        if fdyn == 0.0:
            return {k: np.zeros(len(raw)) for k in keys}
        return {"Cd": raw[:, 0] / fdyn, "Cly": raw[:, 1] / fdyn, "Clz": raw[:, 2] / fdyn,
                "Cmx": raw[:, 9] / mdyn, "Cmy": raw[:, 10] / mdyn, "Cmz": raw[:, 11] / mdyn,
                "Cd_p": raw[:, 3] / fdyn, "Cd_v": raw[:, 6] / fdyn}

    def _append_histories(self, c: dict):
        for k in ("Cd", "Cly", "Clz", "Cmx", "Cmy", "Cmz", "Cd_p", "Cd_v"):
            getattr(self, f"{k}_history").extend(c[k].tolist())

    def _set_last(self, raw_row: np.ndarray, profile: np.ndarray):
        c = self._coefficients(raw_row[None, :])
        self._last_cd_p = float(c["Cd_p"][0])
        self._last_cd_v = float(c["Cd_v"][0])
        self._last_cmx = float(c["Cmx"][0])
        self._last_cmy = float(c["Cmy"][0])
        self._last_cmz = float(c["Cmz"][0])
        self._last_spanwise_profile = {"z": list(range(self.Nz)), "fx": profile[:, 0].tolist(),
                                       "fy": profile[:, 1].tolist(), "fz": profile[:, 2].tolist()}

    def _step_return(self, c: dict, k: int):
        return float(c["Cd"][k]), float(c["Cly"][k]), float(c["Clz"][k])

    def _lift_history_for_stop(self, window):
        # solver3d.py:634-639: the lift component with the larger recent variance
        w = lambda h: h[-min(len(h), window):]
        if np.std(w(self.Clz_history)) > np.std(w(self.Cly_history)):
            return self.Clz_history
        return self.Cly_history

    # -------------------------------------------------------------- run hooks
    def _print_banner(self):
        print(f"  Backend   : {self.backend} ({self.precision}, 3D D3Q19)")
        print(f"  Collision : {self.collision}")

    def _print_progress(self, step, steps, check_every, sps):
        w = min(check_every, len(self.Cd_history))
        print(f"  step {step:6d}/{steps}  Cd={float(np.mean(self.Cd_history[-w:])):+.4f}  "
              f"Cl_y={float(np.mean(self.Cly_history[-w:])):+.4f}  [{sps:.0f} steps/s]", flush=True)

    def _stability_check(self, step, want_fields=False):
        # solver3d.py:608-615 checks the mid z-plane only; the device reduces it
        check_field_health(FieldHealth.from_stats(self._engine.field_stats(self.Nz // 2, 1)), step)
        return None

    def _callback(self, callback, step, macro):
        callback(step, self.Cd_history[-1], self.Cly_history[-1], self.Clz_history[-1])

    def _checkpoint_name(self):
        return f"checkpoint3d_{self.step_count:08d}.npz"

    def _b200_options(self) -> dict:
        opts = super()._b200_options()
        if self.sem_inlet:
            opts.update(sem_inlet=True, sem_Tu=self.sem_Tu, sem_L_int=self.sem_L_int, sem_N=self.sem_N)
        return opts

    def _checkpoint_params(self):
        return dict(
            Nz=self.Nz, Ny=self.Ny, Nx=self.Nx, omega=self.omega, u0=self.u0, D=self.D,
            rho0=self.rho0, wall_bc=self.wall_bc, inlet_bc=self.inlet_bc,
            outlet_bc=self.outlet_bc, streamwise_bc=self.streamwise_bc, backend=self.backend,
            collision=self.collision, inlet_perturbation=self.inlet_perturbation,
            trt_lambda=self.trt_lambda, sponge_thickness=self.sponge_thickness,
            sponge_strength=self.sponge_strength, les=self.les, les_cs=self.les_cs,
            les_model=self.les_model, ibm_enabled=self.ibm_enabled, bouzidi=self.bouzidi,
            van_driest=self.van_driest, van_driest_A=self.van_driest_A,
            body_force_x=self.body_force_x, body_force_y=self.body_force_y,
            body_force_z=self.body_force_z, wall_velocity_top=self.wall_velocity_top,
            wall_velocity_bottom=self.wall_velocity_bottom, synthetic_inflow=self.synthetic_inflow,
            synthetic_inflow_intensity=self.synthetic_inflow_intensity, thermal=self.thermal,
            T_hot=self.T_hot, T_cold=self.T_cold, alpha_T=self.alpha_T, buoyancy=self.buoyancy,
            g_gravity=self.g_gravity, beta=self.beta, T_ref=self.T_ref,
        )

    def _result(self, avg_window, stop_reason, last_conv, last_st) -> dict:
        rho, ux, uy, uz = self._macroscopic_host()
        tail = lambda h: np.array(h[-avg_window:]) if h else np.zeros(1)
        r = {}
        for k in ("Cd", "Cly", "Clz", "Cmx", "Cmy", "Cmz"):
            a = tail(getattr(self, f"{k}_history"))
            r[f"{k}_mean"] = float(np.mean(a))
            r[f"{k}_std"] = float(np.std(a))
        r["Cd_p_mean"] = float(np.mean(tail(self.Cd_p_history)))
        r["Cd_v_mean"] = float(np.mean(tail(self.Cd_v_history)))
        for k in ("Cd", "Cly", "Clz", "Cmx", "Cmy", "Cmz", "Cd_p", "Cd_v"):
            r[f"{k}_history"] = getattr(self, f"{k}_history")
        scalar, scalar_stats = self._scalar_stats()
        r.update({
            "observables": {
                "cd_spectrum": coefficient_spectrum(self.Cd_history),
                "cly_spectrum": coefficient_spectrum(self.Cly_history),
                "clz_spectrum": coefficient_spectrum(self.Clz_history),
                "cmz_spectrum": coefficient_spectrum(self.Cmz_history),
                "spanwise_force_profile_last": getattr(self, "_last_spanwise_profile", None),
            },
            "steps_completed": self.step_count, "stop_reason": stop_reason,
            "convergence_report": last_conv, "strouhal_report": last_st,
            "rho": rho, "ux": ux, "uy": uy, "uz": uz, "scalar": scalar, "scalar_stats": scalar_stats,
        })
        return r
