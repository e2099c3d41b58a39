"""Health checks and coefficient-history statistics used by Solver.run.

What a caller sees follows the reference (aero/diagnostics.py:32-228,
aero/observables.py:10-43): the report dataclasses and their fields, the
thresholds, and the texts of the divergence error and of the two warnings.
How the figures are obtained is this engine's own:

* Stability is judged from FP64 statistics of the state that the GPU reduces
  in a fixed order (``aero_field_stats``: NaN populations, cells with
  rho <= 0, the largest |(ux, uy)|, the sum of rho), so no field crosses to
  the host for the check.
* Trailing-window statistics and spectra share two small helpers (a tail
  view of a history and a one-sided periodogram of the mean-removed signal).
"""

from __future__ import annotations

import math
import warnings
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

# Interface thresholds (the reference's values).
MACH_WARN_SPEED = 0.3        # |(ux, uy)| above which compressibility is flagged
MASS_DRIFT_WARN = 0.05       # |mean rho - 1| above which mass drift is flagged
ZERO_DRAG_LEVEL = 1e-12      # mean|C| below which a history counts as converged
MIN_STROUHAL_SAMPLES = 512
MIN_SHEDDING_AMPLITUDE = 1e-6


# ---------------------------------------------------------------------------
# reports
# ---------------------------------------------------------------------------
@dataclass
class ConvergenceReport:
    converged: bool
    window: int
    ratio: float
    mean_abs: float
    std: float
    threshold: float


@dataclass
class StrouhalReport:
    strouhal: Optional[float]
    peak_frequency: Optional[float]
    peak_amplitude: float
    sample_count: int
    window: int
    stationary: bool = False
    relative_drift: Optional[float] = None


@dataclass
class FieldHealth:
    """The device's FP64 statistics of a set of planes (aero_field_stats)."""

    nan_populations: int
    nonpositive_cells: int
    max_speed: float          # largest |(ux, uy)| over the cells
    mass: float               # sum of rho
    cells: int
    scalar_total: float       # sum of T = sum_i g_i (0 without a scalar)
    wall_flux: tuple          # (sum of -dT/dy at y = 0, columns, same at y = ny-1, columns)

    @classmethod
    def from_stats(cls, v: Sequence[float]) -> "FieldHealth":
        return cls(int(v[0]), int(v[1]), float(v[2]), float(v[3]), int(v[4]), float(v[5]),
                   (float(v[6]), int(v[7]), float(v[8]), int(v[9])))

    @property
    def mean_density(self) -> float:
        return self.mass / self.cells if self.cells else float("nan")

    def nusselt(self, height: float, delta_T: float) -> Optional[tuple]:
        """(bottom, top) Nusselt numbers: mean -dT/dy at each Dirichlet row times
        height / delta_T; None where no column was counted or delta_T = 0."""
        if delta_T == 0.0:
            return None
        s0, n0, s1, n1 = self.wall_flux
        nb = s0 / n0 * height / delta_T if n0 else None
        nt = s1 / n1 * height / delta_T if n1 else None
        return nb, nt


def check_field_health(h: FieldHealth, step: int) -> None:
    """Raises RuntimeError on a diverged state, warns on a fast flow or on a
    drifting mean density; the tests and texts of check_stability
    (diagnostics.py:32-71), applied to the device statistics."""
    if h.nan_populations:
        raise RuntimeError(
            f"[step {step}] NaN detected in f — simulation has diverged. "
            "Check tau (must be > 0.5), inlet velocity, and grid resolution.")
    if h.nonpositive_cells:
        raise RuntimeError(f"[step {step}] Non-positive density detected — simulation has diverged.")
    if h.max_speed > MACH_WARN_SPEED:
        warnings.warn(
            f"[step {step}] Max velocity = {h.max_speed:.4f} lattice units "
            f"(Ma ≈ {h.max_speed * math.sqrt(3.0):.3f}). "
            "Compressibility artifacts likely. Reduce u0 or increase grid size.",
            RuntimeWarning, stacklevel=2)
    if abs(h.mean_density - 1.0) > MASS_DRIFT_WARN:
        warnings.warn(
            f"[step {step}] Mean density drifted to {h.mean_density:.4f} (>5% from 1.0). "
            "Check outlet BC or total mass conservation.", RuntimeWarning, stacklevel=2)


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def _tail(history, n: Optional[int]) -> np.ndarray:
    """The last n samples (all when n is None or not positive) as float64."""
    a = np.asarray(history, dtype=np.float64)
    return a[-int(n):] if (n is not None and n > 0) else a


def _periodogram(signal: np.ndarray, spacing: float = 1.0):
    """Frequencies and magnitudes of the one-sided DFT of the mean-removed
    signal, with the peak |signal - mean| (the amplitude the reports use)."""
    centred = signal - float(signal.mean())
    amp = float(np.abs(centred).max()) if centred.size else 0.0
    return np.fft.rfftfreq(centred.size, d=spacing), np.abs(np.fft.rfft(centred)), amp


# ---------------------------------------------------------------------------
# convergence of a coefficient history
# ---------------------------------------------------------------------------
def analyze_convergence(history: List[float], window: int = 5000, tol: float = 0.01) -> ConvergenceReport:
    """Converged when std / mean|C| over the last `window` samples is below
    tol, or when mean|C| itself is below 1e-12 (population std)."""
    w = max(int(window), 1)
    x = _tail(history, w)
    if x.size < w:
        return ConvergenceReport(False, w, float("inf"), 0.0, 0.0, float(tol))
    level, spread = float(np.abs(x).mean()), float(x.std())
    ratio = 0.0 if level < ZERO_DRAG_LEVEL else spread / level
    return ConvergenceReport(level < ZERO_DRAG_LEVEL or ratio < tol, w, ratio, level, spread, float(tol))


def check_convergence(history: List[float], window: int = 5000, tol: float = 0.01) -> bool:
    return analyze_convergence(history, window=window, tol=tol).converged


# ---------------------------------------------------------------------------
# shedding frequency
# ---------------------------------------------------------------------------
def analyze_strouhal(Cl_history: List[float], D: float, u0: float, *, window: Optional[int] = None,
                     min_samples: int = MIN_STROUHAL_SAMPLES) -> StrouhalReport:
    """St = f_peak D / u0, f_peak the strongest non-zero frequency of the
    (windowed) lift history in cycles per step."""
    total = len(Cl_history)
    if not (u0 > 0.0 and D > 0.0):
        return StrouhalReport(None, None, 0.0, total, int(window or 0))
    x = _tail(Cl_history, window)
    if x.size < max(int(min_samples), 2):
        return StrouhalReport(None, None, 0.0, total, int(x.size))
    freqs, mags, amp = _periodogram(x)
    if amp < MIN_SHEDDING_AMPLITUDE or mags.size < 2:
        return StrouhalReport(None, None, amp, total, int(x.size))
    f_peak = float(freqs[1 + int(np.argmax(mags[1:]))])
    return StrouhalReport(f_peak * D / u0, f_peak, amp, total, int(x.size))


def compute_strouhal(Cl_history: List[float], D: float, u0: float) -> Optional[float]:
    return analyze_strouhal(Cl_history, D=D, u0=u0).strouhal


def detect_statistical_stationarity(Cd_history, Cl_history, D, u0, *, convergence_window=5000,
                                    convergence_tol=0.01, strouhal_window=4096, strouhal_tol=0.05):
    """(drag report, Strouhal report, stop): stop when the drag has converged
    and, once a full Strouhal window (at least 1024 samples) exists, the
    Strouhal numbers of its two halves agree within strouhal_tol."""
    cd = analyze_convergence(Cd_history, window=convergence_window, tol=convergence_tol)
    st = analyze_strouhal(Cl_history, D=D, u0=u0, window=strouhal_window)
    if st.strouhal is None or st.window < max(strouhal_window, 1024):
        return cd, st, cd.converged
    recent = _tail(Cl_history, st.window)
    cut = st.window - st.window // 2
    halves = [analyze_strouhal(part, D=D, u0=u0, min_samples=128).strouhal
              for part in (recent[:cut], recent[cut:])]
    if None in halves:
        return cd, st, cd.converged
    st.relative_drift = abs(halves[1] - halves[0]) / max(abs(halves[0]), 1e-12)
    st.stationary = st.relative_drift < strouhal_tol
    return cd, st, cd.converged and st.stationary


# ---------------------------------------------------------------------------
# spectrum summary of a history (run()'s "observables")
# ---------------------------------------------------------------------------
def coefficient_spectrum(history: List[float], *, sample_spacing: float = 1.0, min_samples: int = 128,
                         discard_fraction: float = 0.2, top_n: int = 8) -> Optional[Dict[str, object]]:
    """The top_n strongest non-zero frequencies of a history after its first
    discard_fraction is dropped (keeping at least min_samples), or None for a
    short or flat history."""
    x = _tail(history, None)
    if x.size < min_samples:
        return None
    skip = min(int(x.size * discard_fraction), max(0, x.size - min_samples))
    freqs, mags, amp = _periodogram(x[skip:], sample_spacing)
    if amp < ZERO_DRAG_LEVEL or mags.size < 2:
        return None
    order = 1 + np.argsort(mags[1:])[::-1][:top_n]
    return {
        "sample_count": int(x.size - skip),
        "dominant_frequency": float(freqs[order[0]]),
        "dominant_amplitude": float(mags[order[0]]),
        "frequencies": freqs[order].astype(float).tolist(),
        "amplitudes": mags[order].astype(float).tolist(),
    }
