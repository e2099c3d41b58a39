"""Run-time checks and history statistics used by Solver.run.

Same rules, thresholds and messages as the reference (aero/diagnostics.py:32-
228, aero/observables.py:10-43): divergence raises RuntimeError, a fast or
mass-drifting flow warns, convergence is std / mean|.| over a trailing
window, and the Strouhal number comes from the rFFT peak of the lift.
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np


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


def check_stability(f: np.ndarray, rho: np.ndarray, ux: np.ndarray, uy: np.ndarray, step: int) -> None:
    if np.isnan(f).any():
        raise RuntimeError(
            f"[step {step}] NaN detected in f — simulation has diverged. "
            "Check tau (must be > 0.5), inlet velocity, and grid resolution.")
    if (rho <= 0.0).any():
        raise RuntimeError(f"[step {step}] Non-positive density detected — simulation has diverged.")
    umag = float(np.sqrt(ux ** 2 + uy ** 2).max())
    if umag > 0.3:
        warnings.warn(
            f"[step {step}] Max velocity = {umag:.4f} lattice units (Ma ≈ {umag * 3 ** 0.5:.3f}). "
            "Compressibility artifacts likely. Reduce u0 or increase grid size.",
            RuntimeWarning, stacklevel=2)
    rho_mean = float(rho.mean())
    if abs(rho_mean - 1.0) > 0.05:
        warnings.warn(
            f"[step {step}] Mean density drifted to {rho_mean:.4f} (>5% from 1.0). "
            "Check outlet BC or total mass conservation.", RuntimeWarning, stacklevel=2)


def analyze_convergence(history: List[float], window: int = 5000, tol: float = 0.01) -> ConvergenceReport:
    window = max(int(window), 1)
    if len(history) < window:
        return ConvergenceReport(False, window, float("inf"), 0.0, 0.0, float(tol))
    recent = np.asarray(history[-window:], dtype=np.float64)
    mean_abs = float(np.mean(np.abs(recent)))
    std = float(np.std(recent))
    if mean_abs < 1e-12:
        return ConvergenceReport(True, window, 0.0, mean_abs, std, float(tol))
    ratio = std / mean_abs
    return ConvergenceReport(ratio < tol, window, ratio, mean_abs, std, float(tol))


def check_convergence(history: List[float], window: int = 5000, tol: float = 0.01) -> bool:
    return analyze_convergence(history, window=window, tol=tol).converged


def analyze_strouhal(Cl_history: List[float], D: float, u0: float, *, window: Optional[int] = None,
                     min_samples: int = 512) -> StrouhalReport:
    if u0 <= 0.0 or D <= 0.0:
        return StrouhalReport(None, None, 0.0, len(Cl_history), int(window or 0))
    x = np.asarray(Cl_history, dtype=np.float64)
    if window is not None and window > 0:
        x = x[-int(window):]
    used = int(x.size)
    if used < max(int(min_samples), 2):
        return StrouhalReport(None, None, 0.0, len(Cl_history), used)
    sig = x - float(np.mean(x))
    amp = float(np.max(np.abs(sig)))
    if amp < 1e-6:
        return StrouhalReport(None, None, amp, len(Cl_history), used)
    mag = np.abs(np.fft.rfft(sig))
    freqs = np.fft.rfftfreq(sig.size, d=1.0)
    if mag.size <= 1:
        return StrouhalReport(None, None, amp, len(Cl_history), used)
    k = int(np.argmax(mag[1:])) + 1
    fpk = float(freqs[k])
    return StrouhalReport(fpk * D / u0, fpk, amp, len(Cl_history), used)


def compute_strouhal(Cl_history: List[float], D: float, u0: float) -> Optional[float]:
    return analyze_strouhal(Cl_history, D=D, u0=u0).strouhal


def detect_statistical_stationarity(Cd_history, Cl_history, D, u0, *, convergence_window=5000,
                                    convergence_tol=0.01, strouhal_window=4096, strouhal_tol=0.05):
    cd = analyze_convergence(Cd_history, window=convergence_window, tol=convergence_tol)
    st = analyze_strouhal(Cl_history, D=D, u0=u0, window=strouhal_window)
    if st.strouhal is None or st.window < max(strouhal_window, 1024):
        return cd, st, cd.converged
    half = st.window // 2
    a = analyze_strouhal(Cl_history[-st.window:-half], D=D, u0=u0, min_samples=128)
    b = analyze_strouhal(Cl_history[-half:], D=D, u0=u0, min_samples=128)
    if a.strouhal is None or b.strouhal is None:
        return cd, st, cd.converged
    drift = abs(b.strouhal - a.strouhal) / max(abs(a.strouhal), 1e-12)
    st.stationary = drift < strouhal_tol
    st.relative_drift = drift
    return cd, st, cd.converged and st.stationary


def coefficient_spectrum(history: List[float], *, sample_spacing: float = 1.0, min_samples: int = 128,
                         discard_fraction: float = 0.2, top_n: int = 8) -> Optional[Dict[str, object]]:
    v = np.asarray(history, dtype=np.float64)
    if v.size < min_samples:
        return None
    discard = int(v.size * discard_fraction)
    if discard >= v.size - min_samples:
        discard = max(0, v.size - min_samples)
    v = v[discard:]
    sig = v - float(np.mean(v))
    if np.max(np.abs(sig)) < 1e-12:
        return None
    freqs = np.fft.rfftfreq(sig.size, d=sample_spacing)
    amps = np.abs(np.fft.rfft(sig))
    if amps.size <= 1:
        return None
    ranked = (np.argsort(amps[1:])[::-1] + 1)[:top_n]
    dom = int(ranked[0])
    return {
        "sample_count": int(sig.size),
        "dominant_frequency": float(freqs[dom]),
        "dominant_amplitude": float(amps[dom]),
        "frequencies": [float(freqs[k]) for k in ranked],
        "amplitudes": [float(amps[k]) for k in ranked],
    }
