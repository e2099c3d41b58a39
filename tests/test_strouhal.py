"""Acceptance bound of the plain FP32 form on the 400x200 cylinder channel
(D2Q9 BGK, Re 100, tau 0.56, seeded +-1e-4 noise on the initial uy), run for
the configuration's 20000 steps with vortex shedding developed: mean Cd and
the Strouhal number within 1e-3 relative of the FP64 oracle.

The Strouhal number is taken as the reference takes it (analyze_strouhal,
diagnostics.py:123-194: the rFFT peak of Cl over the last 8192 steps), which
resolves frequency only to one FFT bin: here bin 2, the slow shedding mode
(about 4800 steps a period at St ~ 0.17).  The test therefore also compares
the mean interval between zero up-crossings of Cl (linearly interpolated),
which follows the faster oscillation riding on it (about 207 steps) and
resolves timing far more finely.  The oracle's 20000 FP64 steps take about
20 s on the host cores."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 20000
TAIL = 8192  # the last steps: the developed shedding


def _period(cl):
    """Mean interval (steps) between the interpolated zero up-crossings of
    cl - mean(cl)."""
    s = np.asarray(cl) - np.mean(cl)
    k = np.nonzero((s[:-1] < 0) & (s[1:] >= 0))[0]
    t = k + (-s[k]) / (s[k + 1] - s[k])
    assert len(t) >= 4, "Cl does not oscillate"
    return (t[-1] - t[0]) / (len(t) - 1)


def test_cylinder_channel_cd_and_strouhal_vs_oracle():
    from aero_b200 import Cylinder, Solver
    from aero_b200.diagnostics import analyze_strouhal
    from aero_b200.lattice import feq
    from oracle.oracle import OracleSolver
    ny, nx = 200, 400
    geo = Cylinder(radius=20, cx_frac=0.25, cy_frac=0.5)
    solid = geo.mark_solid(ny, nx)
    u0, D = 0.05, geo.reference_length()
    omega = 1.0 / (3.0 * u0 * D / 100.0 + 0.5)
    kw = dict(wall_bc="noslip", outlet_bc="zerogradient", inlet_bc="velocity", collision="bgk")
    rng = np.random.default_rng(11)
    f0 = feq(2, np.ones((ny, nx)), np.full((ny, nx), u0), rng.uniform(-1e-4, 1e-4, (ny, nx)))
    s = Solver(Ny=ny, Nx=nx, solid=solid, omega=omega, u0=u0, D=D, precision="fp32",
               hist_capacity=STEPS + 8, **kw)
    s.f = f0
    r = s.run(STEPS, check_every=5000, verbose=False)
    cd, cl = np.array(r["Cd_history"]), np.array(r["Cl_history"])
    o = OracleSolver(solid=solid, omega=omega, u0=u0, D=D, **kw)
    o.f = f0.copy()
    ocd, ocl = np.empty(STEPS), np.empty(STEPS)
    for k in range(STEPS):
        c = o.step()[0]
        ocd[k], ocl[k] = c["Cd"], c["Cl"]
    assert abs(cd[-TAIL:].mean() - ocd[-TAIL:].mean()) <= 1e-3 * abs(ocd[-TAIL:].mean())
    st = analyze_strouhal(list(cl), D=D, u0=u0, window=TAIL).strouhal
    ost = analyze_strouhal(list(ocl), D=D, u0=u0, window=TAIL).strouhal
    assert st is not None and ost is not None
    assert abs(st - ost) <= 1e-3 * abs(ost)
    assert abs(_period(cl[-TAIL:]) - _period(ocl[-TAIL:])) <= 1e-3 * _period(ocl[-TAIL:])
