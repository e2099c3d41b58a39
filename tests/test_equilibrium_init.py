"""set_equilibrium_state (aero_set_equilibrium): the equilibrium state built
on the device from macroscopic fields equals the state the reference's
assignment ``s.f = compute_feq(rho, ux, uy[, uz])`` sets (outlet state from
the last column, scalar w T), bit for bit in FP64 storage and to the
rounding of one conversion in FP32; the uniform default is the reference's
initial state (solver.py:218-227, solver3d.py:239-247)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fields(shape, dims, seed=5):
    rng = np.random.default_rng(seed)
    rho = 1.0 + 1e-3 * rng.uniform(-1, 1, shape)
    ux = 0.05 + 1e-2 * rng.uniform(-1, 1, shape)
    uy = 1e-2 * rng.uniform(-1, 1, shape)
    uz = 1e-2 * rng.uniform(-1, 1, shape) if dims == 3 else None
    T = 0.5 + 1e-3 * rng.uniform(-1, 1, shape)
    return rho, ux, uy, uz, T


def _pair(dims, precision, **kw):
    from aero_b200 import Solver, Solver3D, Sphere
    if dims == 2:
        shape = (20, 36)
        solid = np.zeros(shape, dtype=bool)
        solid[8:12, 8:12] = True
        mk = lambda: Solver(Ny=shape[0], Nx=shape[1], solid=solid, omega=1.4, u0=0.05, D=4.0,
                            precision=precision, **kw)
    else:
        shape = (8, 10, 18)
        sph = Sphere(radius=2.5, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
        solid = sph.mark_solid(*shape)
        mk = lambda: Solver3D(Nz=shape[0], Ny=shape[1], Nx=shape[2], solid=solid, omega=1.4, u0=0.05, D=5.0,
                              precision=precision, **kw)
    return mk(), mk(), shape


@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_device_equilibrium_equals_host_assignment(dims, precision):
    from aero_b200.lattice import feq, scalar_weights
    kw = dict(thermal=True, scalar_lattice="reduced") if dims == 3 else dict(thermal=True)
    a, b, shape = _pair(dims, precision, **kw)
    rho, ux, uy, uz, T = _fields(shape, dims)
    a.set_equilibrium_state(rho=rho, ux=ux, uy=uy, uz=uz, T=T)
    f = feq(dims, rho, ux, uy, uz)
    b.f = f
    b._f_outlet_prev = np.ascontiguousarray(f[..., -1])
    wg = scalar_weights(dims, b.scalar_lattice == "reduced")
    b.g = np.ascontiguousarray(wg.reshape((-1,) + (1,) * dims) * T[None])
    b._flush_host_state()  # b's arrays go to the device, so both sides are read back from it
    if precision == "fp64":
        assert np.array_equal(a.f, b.f)
        assert np.array_equal(a._f_outlet_prev, b._f_outlet_prev)
        assert np.array_equal(a.g, b.g)
    else:
        np.testing.assert_array_equal(a.f, b.f)
        np.testing.assert_array_equal(a._f_outlet_prev, b._f_outlet_prev)
        np.testing.assert_array_equal(a.g, b.g)
    for _ in range(3):
        a._step()
        b._step()
    if precision == "fp64":
        assert np.array_equal(a.f, b.f)
    else:
        np.testing.assert_allclose(a.f, b.f, rtol=0, atol=1e-6)


@pytest.mark.parametrize("dims", [2, 3])
def test_uniform_default_is_the_reference_initial_state(dims):
    from aero_b200.lattice import feq
    a, _, shape = _pair(dims, "fp64")
    ones = np.ones(shape)
    f = feq(dims, ones, 0.05 * ones, 0.0 * ones, 0.0 * ones if dims == 3 else None)
    assert np.array_equal(a.f, f)
    assert np.array_equal(a._f_outlet_prev, f[..., -1])
    a.run(4, check_every=5, verbose=False)
    a.set_equilibrium_state()
    assert np.array_equal(a.f, f) and a.step_count == 4


def test_field_arguments_are_checked():
    a, _, shape = _pair(2, "fp32")
    with pytest.raises(ValueError):
        a.set_equilibrium_state(uz=np.zeros(shape))
    with pytest.raises(ValueError):
        a.set_equilibrium_state(T=np.zeros(shape))
