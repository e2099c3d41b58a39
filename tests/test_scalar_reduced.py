"""The D2Q5 / D3Q7 passive scalar (scalar_lattice="reduced") against the FP64
oracle, and the device field statistics (mass, scalar total, Nusselt sums)
against the same figures computed on the host from the oracle's state.

The reduced scalar is this engine's speed mode: the reference runs its
scalar on the flow lattice (aero/lbm/thermal.py:31-203).  The oracle
restates the same scalar algorithm -- BGK collision toward
w_i T (1 + e_i.u / cs^2), periodic push, Dirichlet rows at y = 0 and
y = Ny-1, Boussinesq forcing of the flow (thermal.py:103-124, :206-222) --
on the D2Q5 (cs^2 = 1/3) and D3Q7 (cs^2 = 1/4) lattices.

Tolerances: FP64 storage |df| <= 1e-10 max|f|, |dg| <= 1e-10 max|g| (the
engine's association order differs from the oracle's); FP32 storage
relative L2 of rho, u and T <= 1e-5 (the bound of the plain FP32 form).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _box_channel_3d():
    from aero_b200 import Box
    nz, ny, nx = 12, 16, 32
    g = Box(width=6, height=5, depth=12, cx_frac=12 / 32, cy_frac=2 / 16, cz_frac=0.5)
    solid = g.mark_solid(nz, ny, nx)
    kw = dict(collision="trt", trt_lambda=3 / 16, les=True, les_model="wale", les_cs=0.5, wall_bc="noslip",
              streamwise_bc="periodic", body_force_x=1e-5, thermal=True, T_hot=1.0, T_cold=0.0, alpha_T=0.02,
              buoyancy=True, g_gravity=1e-3, beta=1.0, T_ref=0.5, scalar_lattice="reduced")
    return dict(dims=3, shape=(nz, ny, nx), solid=solid, omega=1.0 / 0.8, u0=0.05, D=g.reference_length(), kw=kw)


def _channel_2d():
    from aero_b200 import Cylinder
    ny, nx = 24, 48
    g = Cylinder(radius=4, cx_frac=0.3, cy_frac=0.5)
    solid = g.mark_solid(ny, nx)
    kw = dict(collision="bgk", wall_bc="noslip", outlet_bc="zerogradient", inlet_bc="velocity", thermal=True,
              T_hot=1.0, T_cold=0.0, alpha_T=0.02, buoyancy=True, g_gravity=1e-3, beta=1.0, T_ref=0.5,
              scalar_lattice="reduced")
    return dict(dims=2, shape=(ny, nx), solid=solid, omega=1.0 / 0.7, u0=0.04, D=g.reference_length(), kw=kw)


def _pair(case, precision, seed=7):
    """Engine and oracle from the same seeded state: f at equilibrium with a
    small seeded velocity perturbation, T = T_ref + U(-1e-3, 1e-3)."""
    from aero_b200 import Solver, Solver3D
    from oracle.oracle import OracleSolver
    rng = np.random.default_rng(seed)
    shape = case["shape"]
    kw = case["kw"]
    o = OracleSolver(solid=case["solid"], omega=case["omega"], u0=case["u0"], D=case["D"], **kw)
    ux = case["u0"] * (1.0 + 0.05 * rng.uniform(-1, 1, shape))
    uy = 0.01 * rng.uniform(-1, 1, shape)
    uz = 0.01 * rng.uniform(-1, 1, shape) if case["dims"] == 3 else None
    o.f = o.feq(np.ones(shape), ux, uy, uz)
    o.f_outlet_prev = np.ascontiguousarray(o.f[..., -1])
    T0 = kw["T_ref"] + 1e-3 * rng.uniform(-1, 1, shape)
    o.g = np.ascontiguousarray(o.Wg.reshape((-1,) + (1,) * case["dims"]) * T0)
    common = dict(solid=case["solid"], omega=case["omega"], u0=case["u0"], D=case["D"], precision=precision, **kw)
    if case["dims"] == 2:
        s = Solver(Ny=shape[0], Nx=shape[1], **common)
    else:
        s = Solver3D(Nz=shape[0], Ny=shape[1], Nx=shape[2], **common)
    s.f = o.f.copy()
    s._f_outlet_prev = o.f_outlet_prev.copy()
    s.g = o.g.copy()
    return s, o


def _rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def _macro(f, dims):
    from aero_b200.lattice import macroscopic
    return macroscopic(f, dims)


@pytest.mark.parametrize("which", ["3d", "2d"])
def test_reduced_scalar_fp64_matches_oracle(which):
    case = _box_channel_3d() if which == "3d" else _channel_2d()
    s, o = _pair(case, "fp64")
    steps = 60
    for _ in range(steps):
        s._step()
        o.step()
    assert s.g.shape[0] == (7 if which == "3d" else 5)
    np.testing.assert_allclose(s.f, o.f, rtol=0, atol=1e-10 * np.abs(o.f).max())
    np.testing.assert_allclose(s.g, o.g, rtol=0, atol=1e-10 * np.abs(o.g).max())


@pytest.mark.parametrize("which", ["3d", "2d"])
def test_reduced_scalar_fp32_close_to_oracle(which):
    case = _box_channel_3d() if which == "3d" else _channel_2d()
    s, o = _pair(case, "fp32")
    for _ in range(60):
        s._step()
        o.step()
    got, ref = _macro(s.f, case["dims"]), _macro(o.f, case["dims"])
    assert _rel_l2(got[0], ref[0]) <= 1e-5
    assert _rel_l2(np.stack(got[1:]), np.stack(ref[1:])) <= 1e-5
    assert _rel_l2(s.g.sum(axis=0), o.g.sum(axis=0)) <= 1e-5


def _host_stats(f, g, solid, dims, T_hot, T_cold):
    """The figures aero_field_stats reduces on the device, from host arrays."""
    rho, ux, uy = _macro(f, dims)[:3]
    T = g.sum(axis=0)
    ny = solid.shape[-2]
    if dims == 2:
        T, solid = T[None], solid[None]
    nu = []
    for y, s in ((0, 1), (ny - 1, -1)):
        fluid = ~solid[:, y + s, :] & ~solid[:, y + 2 * s, :]
        dn = 0.5 * (-3.0 * T[:, y, :] + 4.0 * T[:, y + s, :] - T[:, y + 2 * s, :])
        mdTdy = -dn if y == 0 else dn
        nu.append(mdTdy[fluid].mean() * (ny - 1) / (T_hot - T_cold))
    return dict(mass=rho.sum(), scalar_total=T.sum(), max_speed=np.sqrt(ux ** 2 + uy ** 2).max(),
                Nu_bottom=nu[0], Nu_top=nu[1])


@pytest.mark.parametrize("which", ["3d", "2d"])
def test_field_statistics_match_host(which):
    case = _box_channel_3d() if which == "3d" else _channel_2d()
    s, o = _pair(case, "fp64")
    for _ in range(25):
        s._step()
        o.step()
    got = s.field_statistics()
    ref = _host_stats(o.f, o.g, case["solid"], case["dims"], case["kw"]["T_hot"], case["kw"]["T_cold"])
    for k in ("mass", "scalar_total", "max_speed"):
        assert abs(got[k] - ref[k]) <= 1e-11 * abs(ref[k]), (k, got[k], ref[k])
    for k in ("Nu_bottom", "Nu_top"):
        assert abs(got[k] - ref[k]) <= 1e-8 * max(abs(ref[k]), 1e-3), (k, got[k], ref[k])
    assert got["nan_populations"] == 0 and got["nonpositive_cells"] == 0
    assert got["cells"] == case["solid"].size
    # the same reduction, twice: the fixed-order sums are reproducible
    again = s.field_statistics()
    assert again["mass"] == got["mass"] and again["scalar_total"] == got["scalar_total"]


def test_conduction_profile_has_unit_nusselt():
    """A linear T profile between the Dirichlet rows (pure conduction) gives
    Nu = 1 at both rows."""
    case = _channel_2d()
    case["kw"] = dict(case["kw"], buoyancy=False)
    s, o = _pair(case, "fp64")
    ny = case["shape"][0]
    T = np.linspace(1.0, 0.0, ny)[:, None] * np.ones(case["shape"])
    s.g = np.ascontiguousarray(o.Wg[:, None, None] * T)
    st = s.field_statistics()
    assert abs(st["Nu_bottom"] - 1.0) < 1e-12 and abs(st["Nu_top"] - 1.0) < 1e-12
