"""Host-side inlet field generators (aero_b200.inflow) against the oracle
driver's independent restatement of the reference's generators
(aero/lbm/solver.py:259-270, aero/lbm/solver3d.py:297-321,
aero/lbm/sem_inlet.py:15-136): same seeded random streams, same fields,
step for step.  No GPU needed."""

import numpy as np

from aero_b200.inflow import SEMInflow, SyntheticInflow


def _oracle(dims, **kw):
    from oracle.oracle import OracleSolver
    shape = (14, 30) if dims == 2 else (9, 12, 20)
    solid = np.zeros(shape, dtype=bool)
    return OracleSolver(solid=solid, omega=1.6, u0=0.05, D=4.0, **kw)


def test_synthetic_inflow_2d_matches_oracle():
    o = _oracle(2, synthetic_inflow=True, synthetic_inflow_intensity=0.07, synthetic_inflow_seed=5)
    g = SyntheticInflow(2, 14, 1, 0.05, 0.07, 5)
    got = g.fields(25)
    for k in range(25):
        np.testing.assert_array_equal(got[k], o._next_inflow().reshape(1, -1))


def test_synthetic_inflow_3d_matches_oracle():
    o = _oracle(3, synthetic_inflow=True, synthetic_inflow_intensity=0.04, synthetic_inflow_seed=11)
    g = SyntheticInflow(3, 12, 9, 0.05, 0.04, 11)
    got = g.fields(10)
    for k in range(10):
        np.testing.assert_array_equal(got[k], o._next_inflow().reshape(2, -1))


def test_sem_matches_oracle_and_is_divergence_free():
    o = _oracle(3, sem_inlet=True, sem_Tu=0.05, sem_L_int=2.5, sem_N=30)
    g = SEMInflow(12, 9, 0.05, 0.05, 2.5, 30)
    got = g.fields(40)  # long enough for eddies to leave the box and be re-drawn
    for k in range(40):
        np.testing.assert_allclose(got[k], o._next_sem().reshape(3, -1), rtol=0, atol=1e-15)
    # (v', w') divergence-free in the plane up to the removed Nyquist modes
    v, w = got[-1][1].reshape(9, 12), got[-1][2].reshape(9, 12)
    ky = np.fft.fftfreq(12)[None, :] * 2 * np.pi
    kz = np.fft.fftfreq(9)[:, None] * 2 * np.pi
    div = ky * np.fft.fft2(v) + kz * np.fft.fft2(w)
    assert np.abs(div).max() < 1e-12 * max(np.abs(np.fft.fft2(v)).max(), 1e-30)
    # RMS of u' and the joint RMS of (v', w') are Tu u0
    assert abs(np.std(got[-1][0]) - 0.05 * 0.05) < 1e-15
