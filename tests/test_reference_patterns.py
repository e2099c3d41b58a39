"""The reference's own usage patterns with backend="b200" substituted.

* Backend selection (tests/test_phase3.py:190-208 of the reference): an
  unknown backend raises ValueError naming it.
* Numerical equivalence of backends (test_phase3.py:215-250): run() histories
  and the final f of the engine in FP64 against the FP64 oracle, at the
  reference's bounds between its own backends (rtol 1e-10, atol 1e-12).
* Checkpoint round trip and continuation (tests/test_phase2.py:356-420):
  f, histories and step count restored; 50 + checkpoint + 50 steps equal to
  100 steps.
* In-place edits of the host state (multiblock.py:143-153 and
  tests/test_sponge.py:41-44 write into s.f / s.g slices): an edit of the
  array s.f returned takes effect at the next step, exactly as the same edit
  made to the oracle's state.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _channel(backend="b200", Ny=30, Nx=60, **kw):
    from aero_b200 import Solver
    solid = np.zeros((Ny, Nx), dtype=bool)
    solid[Ny // 2 - 3:Ny // 2 + 3, Nx // 4 - 3:Nx // 4 + 3] = True
    return Solver(Ny=Ny, Nx=Nx, solid=solid, omega=1.2, u0=0.05, D=6.0, backend=backend, **kw)


def test_unknown_backend_raises():
    with pytest.raises(ValueError, match="Unknown backend"):
        _channel(backend="cuda")


def test_histories_and_f_match_oracle_like_backend_equivalence():
    from oracle.oracle import OracleSolver
    s = _channel(Ny=40, Nx=80, precision="fp64")
    o = OracleSolver(solid=s.solid, omega=1.2, u0=0.05, D=6.0)
    steps = 200
    s.run(steps=steps, check_every=steps + 1, verbose=False)
    cd, cl = [], []
    for _ in range(steps):
        c, _ = o.step()
        cd.append(c["Cd"])
        cl.append(c["Cl"])
    np.testing.assert_allclose(s.Cd_history, cd, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(s.Cl_history, cl, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(s.f, o.f, rtol=1e-10, atol=1e-12)


def test_checkpoint_round_trip_and_continuation(tmp_path):
    full = _channel(precision="fp64")
    full.run(steps=100, check_every=100, verbose=False)
    a = _channel(precision="fp64")
    a.run(steps=50, check_every=50, verbose=False)
    path = str(tmp_path / "mid.npz")
    a.save_checkpoint(path)
    b = _channel(precision="fp64")
    b.load_checkpoint(path)
    assert np.array_equal(a.f, b.f)
    assert a.Cd_history == b.Cd_history and a.Cl_history == b.Cl_history
    assert b.step_count == 50
    b.run(steps=50, check_every=50, verbose=False)
    # the reference bounds its own continuation at atol 1e-15 on O(1) values;
    # these drags are O(100), where one ulp is 1.4e-14: a few ulps
    np.testing.assert_allclose(full.Cd_history, b.Cd_history, rtol=1e-13, atol=0)
    np.testing.assert_allclose(full.f, b.f, rtol=0, atol=1e-14)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_in_place_edit_of_f_3d(precision):
    from oracle.oracle import OracleSolver

    from tests.golden_cases import load_case, make_oracle
    from tests.test_gpu_parity import _solver
    c = load_case("c3d_bgk_slip_convective")
    s = _solver(c, precision=precision)
    o = make_oracle(c)
    assert isinstance(o, OracleSolver)
    for _ in range(3):
        s._step()
        o.step()
    f = s.f                      # the host view ...
    f[:, 4, 5, 6] *= 1.01        # ... edited in place, as multiblock.py does
    f[3, 2, :, 9] += 1e-4
    s._f_outlet_prev[:, 2, 3] += 1e-4   # the convective outlet's state
    o.f[:, 4, 5, 6] *= 1.01
    o.f[3, 2, :, 9] += 1e-4
    o.f_outlet_prev[:, 2, 3] += 1e-4
    for _ in range(4):
        s._step()
        o.step()
    tol = 1e-10 if precision == "fp64" else 1e-6
    np.testing.assert_allclose(s.f, o.f, rtol=0, atol=tol * np.abs(o.f).max())


def test_in_place_edit_of_g_2d():
    from tests.golden_cases import load_case, make_oracle
    from tests.test_gpu_parity import _solver
    c = load_case("c2d_bgk_thermal")
    s = _solver(c, precision="fp64")
    o = make_oracle(c)
    for _ in range(2):
        s._step()
        o.step()
    s.g[:, 10, 20] *= 1.05
    o.g[:, 10, 20] *= 1.05
    for _ in range(3):
        s._step()
        o.step()
    np.testing.assert_allclose(s.f, o.f, rtol=0, atol=1e-10 * np.abs(o.f).max())
    np.testing.assert_allclose(s.g, o.g, rtol=0, atol=1e-10 * np.abs(o.g).max())
