"""Failure detection without a GPU fault: the row-tiled kernel's waits on
its bulk-copy stages are bounded, so a stage that never completes makes the
step return with a status bit set instead of spinning, and the GPU context
stays usable afterwards."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sphere_solver():
    from aero_b200 import Solver3D, Sphere
    nz, ny, nx = 16, 16, 32
    sph = Sphere(radius=3, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
    return Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=sph.mark_solid(nz, ny, nx), omega=1 / 0.6, u0=0.05,
                    D=sph.reference_length(), collision="mrt", wall_bc="slip")


def test_tiled_stage_wait_gives_up_and_reports(monkeypatch):
    """AERO_B200_TEST_STALL_TILES=1 makes every stage announce more bytes than
    its copies deliver, so no stage of the row-tiled kernel ever completes.
    The bounded waits give up after about a second each, the step returns
    with status bit 1 ('a bounded device-side wait gave up'), and a lattice
    built afterwards steps normally on the same context."""
    monkeypatch.setenv("AERO_B200_TILES", "1")
    monkeypatch.setenv("AERO_B200_TEST_STALL_TILES", "1")
    s = _sphere_solver()
    assert s._engine.step_plan()["tiled"]
    t0 = time.perf_counter()
    s._engine.step(1)
    status = s._engine.status()  # synchronises the stream
    dt = time.perf_counter() - t0
    assert status & 2, status
    assert dt < 30.0, dt
    monkeypatch.delenv("AERO_B200_TEST_STALL_TILES")
    t = _sphere_solver()
    r = t.run(20, check_every=21, verbose=False)
    assert t.status() == 0
    assert np.isfinite(t.f).all() and np.isfinite(r["Cd_history"]).all()
    monkeypatch.delenv("AERO_B200_TILES")
    u = _sphere_solver()
    u.run(20, check_every=21, verbose=False)
    np.testing.assert_allclose(t.f, u.f, rtol=0, atol=1e-6 * np.abs(u.f).max())


def test_persistent_barrier_wait_gives_up_and_reports(monkeypatch):
    """AERO_B200_TEST_STALL_RUN=1 makes one cell block of the persistent
    runner leave before its first grid barrier, so that barrier never
    completes.  The other blocks' bounded waits give up after about a
    second, the call returns with status bit 1, and a lattice built
    afterwards steps normally on the same context."""
    monkeypatch.setenv("AERO_B200_TEST_STALL_RUN", "1")
    s = _sphere_solver()
    t0 = time.perf_counter()
    s._engine.step(4)
    status = s._engine.status()  # synchronises the stream
    dt = time.perf_counter() - t0
    assert status & 2, status
    assert dt < 30.0, dt
    monkeypatch.delenv("AERO_B200_TEST_STALL_RUN")
    t = _sphere_solver()
    r = t.run(20, check_every=21, verbose=False)
    assert t.status() == 0
    assert np.isfinite(t.f).all() and np.isfinite(r["Cd_history"]).all()
    u = _sphere_solver()
    u._engine.set_persistent(False)
    u.run(20, check_every=21, verbose=False)
    # MRT: the two kernels round their FMAs differently
    np.testing.assert_allclose(t.f, u.f, rtol=0, atol=1e-6 * np.abs(u.f).max())
