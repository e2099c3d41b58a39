"""Host diagnostics of Solver.run (aero_b200.diagnostics) on synthetic
histories and device statistics: the reports, thresholds and messages of the
reference's aero/diagnostics.py:32-228 and aero/observables.py:10-43.  CPU
only."""

import math
import warnings

import numpy as np
import pytest

from aero_b200 import diagnostics as dg


def test_convergence_rule():
    rng = np.random.default_rng(3)
    h = list(2.0 + 1e-4 * rng.standard_normal(3000))
    r = dg.analyze_convergence(h, window=1000, tol=1e-3)
    tail = np.array(h[-1000:])
    assert r.window == 1000 and r.threshold == 1e-3
    assert math.isclose(r.mean_abs, np.abs(tail).mean(), rel_tol=1e-14)
    assert math.isclose(r.std, tail.std(), rel_tol=1e-12)
    assert math.isclose(r.ratio, tail.std() / np.abs(tail).mean(), rel_tol=1e-12)
    assert r.converged
    assert not dg.analyze_convergence(h, window=1000, tol=1e-5).converged
    short = dg.analyze_convergence(h[:999], window=1000)
    assert not short.converged and short.ratio == float("inf") and short.mean_abs == 0.0
    zero = dg.analyze_convergence([0.0] * 50, window=50, tol=1e-9)
    assert zero.converged and zero.ratio == 0.0
    assert dg.check_convergence(h, window=1000, tol=1e-3)


def test_strouhal_of_a_sine():
    n, period, D, u0 = 4096, 64.0, 40.0, 0.05
    t = np.arange(n)
    cl = list(0.3 * np.sin(2 * np.pi * t / period) + 0.01)
    r = dg.analyze_strouhal(cl, D=D, u0=u0)
    assert math.isclose(r.peak_frequency, 1.0 / period, rel_tol=1e-12)
    assert math.isclose(r.strouhal, D / (period * u0), rel_tol=1e-12)
    assert r.sample_count == n and r.window == n
    assert math.isclose(r.peak_amplitude, 0.3, rel_tol=1e-3)
    assert dg.compute_strouhal(cl, D, u0) == r.strouhal
    assert dg.analyze_strouhal(cl[:511], D, u0).strouhal is None          # too short
    assert dg.analyze_strouhal([1.0] * 600, D, u0).strouhal is None       # flat
    assert dg.analyze_strouhal(cl, D, 0.0).strouhal is None               # no flow
    w = dg.analyze_strouhal(cl, D, u0, window=1024)
    assert w.window == 1024 and w.sample_count == n


def test_stationarity_stop():
    n = 8192
    t = np.arange(n)
    cl = list(np.sin(2 * np.pi * t / 50.0))
    cd = list(1.5 + 1e-6 * np.cos(t))
    cdr, st, stop = dg.detect_statistical_stationarity(cd, cl, 20.0, 0.05, convergence_window=2000,
                                                         convergence_tol=1e-3, strouhal_window=4096)
    assert cdr.converged and st.stationary and stop
    assert st.relative_drift == 0.0
    # a shedding frequency that changes between the halves of the window
    chirp = list(np.sin(2 * np.pi * np.cumsum(np.linspace(1 / 80.0, 1 / 40.0, n))))
    _, st2, stop2 = dg.detect_statistical_stationarity(cd, chirp, 20.0, 0.05, convergence_window=2000,
                                                        convergence_tol=1e-3, strouhal_window=4096)
    assert not st2.stationary and not stop2 and st2.relative_drift > 0.05


def test_coefficient_spectrum_two_tones():
    n = 2000
    t = np.arange(n)
    h = list(0.5 * np.sin(2 * np.pi * t / 20.0) + 0.2 * np.sin(2 * np.pi * t / 100.0) + 3.0)
    r = dg.coefficient_spectrum(h)
    kept = n - int(n * 0.2)
    assert r["sample_count"] == kept
    assert math.isclose(r["dominant_frequency"], round(kept / 20.0) / kept, rel_tol=1e-12)
    assert len(r["frequencies"]) == 8 and len(r["amplitudes"]) == 8
    assert r["amplitudes"] == sorted(r["amplitudes"], reverse=True)
    assert dg.coefficient_spectrum(h[:100]) is None
    assert dg.coefficient_spectrum([2.0] * 500) is None
    # the discarded head never leaves fewer than min_samples
    assert dg.coefficient_spectrum(h[:140])["sample_count"] == 128


def _stats(nan=0, nonpos=0, umax=0.05, mass=1000.0, cells=1000):
    return [nan, nonpos, umax, mass, cells, 0.0, 0.0, 0, 0.0, 0]


def test_field_health_checks():
    dg.check_field_health(dg.FieldHealth.from_stats(_stats()), 10)
    with pytest.raises(RuntimeError, match=r"\[step 7\] NaN detected in f"):
        dg.check_field_health(dg.FieldHealth.from_stats(_stats(nan=3)), 7)
    with pytest.raises(RuntimeError, match="Non-positive density"):
        dg.check_field_health(dg.FieldHealth.from_stats(_stats(nonpos=1)), 7)
    with warnings.catch_warnings(record=True) as rec:
        warnings.simplefilter("always")
        dg.check_field_health(dg.FieldHealth.from_stats(_stats(umax=0.4)), 5)
        dg.check_field_health(dg.FieldHealth.from_stats(_stats(mass=1100.0)), 5)
    msgs = [str(r.message) for r in rec]
    assert any("Max velocity = 0.4000" in m and "Compressibility" in m for m in msgs)
    assert any("Mean density drifted to 1.1000" in m for m in msgs)


def test_nusselt_from_wall_sums():
    h = dg.FieldHealth.from_stats([0, 0, 0.0, 1.0, 1, 0.0, 2.0, 4, 3.0, 3, ])
    nb, nt = h.nusselt(height=10.0, delta_T=2.0)
    assert nb == 2.0 / 4 * 10.0 / 2.0 and nt == 3.0 / 3 * 10.0 / 2.0
    assert h.nusselt(10.0, 0.0) is None
