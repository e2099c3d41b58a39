"""Kernels compiled for one feature word and wall type: a lattice whose
features are exactly those of the thermal channel (D3Q19 TRT + WALE, uniform
body force, D3Q7 scalar with buoyancy, an obstacle with mid-link
bounce-back, no-slip walls, streamwise periodic) or of the open wind tunnel
(velocity inlet, outlet, obstacle, slip walls, with or without Smagorinsky
LES) steps with kernels in which every other feature's branch is removed at
compile time; every other lattice keeps the generic kernels.  Both compute
the same operations, so the states agree up to the FP rounding of the
compiled variant: FP32 1e-6, FP16 1e-4 and BF16 1e-3 of max|f| (and of
max|g|) after 40 steps, the drag histories to ten times that."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-6, "fp16s": 1e-4, "bf16s": 1e-3}


def _channel(precision, **extra):
    from aero_b200 import Box, Solver3D
    nz, ny, nx = 12, 16, 40
    box = Box(width=6, height=6, depth=12, cx_frac=0.3, cy_frac=3 / 16, cz_frac=0.5)
    solid = box.mark_solid(nz, ny, nx)
    kw = dict(omega=1 / 0.8, u0=0.05, D=6.0, collision="trt", trt_lambda=3 / 16, les=True, les_model="wale",
              les_cs=0.5, wall_bc="noslip", streamwise_bc="periodic", body_force_x=1e-5, thermal=True, T_hot=1.0,
              T_cold=0.0, alpha_T=0.02, buoyancy=True, g_gravity=1e-3, beta=1.0, T_ref=0.5,
              scalar_lattice="reduced", precision=precision)
    kw.update(extra)
    return Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, **kw)


def _run(s):
    rng = np.random.default_rng(3)
    shp = s.solid.shape
    s.set_equilibrium_state(ux=0.05 + 0.01 * rng.uniform(-1, 1, shp), uy=0.01 * rng.uniform(-1, 1, shp),
                            T=0.5 + 1e-3 * rng.uniform(-1, 1, shp))
    r = s.run(40, check_every=20, verbose=False)
    return np.array(r["Cd_history"])


@pytest.mark.parametrize("precision", ["fp32", "fp16s", "bf16s"])
def test_thermal_channel_kernels_equal_generic(precision, monkeypatch):
    monkeypatch.delenv("AERO_B200_GENERIC_KERNELS", raising=False)
    a = _channel(precision)
    assert a._engine.kernel_variant() == 1
    cda = _run(a)
    monkeypatch.setenv("AERO_B200_GENERIC_KERNELS", "1")
    b = _channel(precision)
    assert b._engine.kernel_variant() == 0
    cdb = _run(b)
    tol = TOL[precision]
    np.testing.assert_allclose(a.f, b.f, rtol=0, atol=tol * np.abs(b.f).max())
    np.testing.assert_allclose(a.g, b.g, rtol=0, atol=tol * np.abs(b.g).max())
    np.testing.assert_allclose(cda, cdb, rtol=0, atol=10 * tol * np.abs(cdb).max())
    assert a.status() == b.status() == 0


def _tunnel(dims, collision, les, precision="fp32", **extra):
    from aero_b200 import Cylinder, Solver, Solver3D, Sphere
    # TRT at tau 0.8: the reference's TRT parameters are unstable below about 0.77
    kw = dict(omega=1 / (0.8 if collision == "trt" else 0.6), u0=0.05, collision=collision, les=les, les_cs=0.16,
              wall_bc="slip",
              inlet_bc="velocity", outlet_bc="convective", precision=precision)
    kw.update(extra)
    if dims == 2:
        cyl = Cylinder(radius=5, cx_frac=0.25, cy_frac=0.5)
        return Solver(Ny=40, Nx=96, solid=cyl.mark_solid(40, 96), D=cyl.reference_length(), **kw)
    sph = Sphere(radius=4, cx_frac=0.25, cy_frac=0.5, cz_frac=0.5)
    return Solver3D(Nz=16, Ny=18, Nx=40, solid=sph.mark_solid(16, 18, 40), D=sph.reference_length(), **kw)


TUNNELS = [(2, "bgk", False, 2), (2, "trt", False, 2), (2, "mrt", False, 2), (3, "bgk", False, 3),
           (3, "trt", False, 3), (3, "mrt", False, 3), (2, "bgk", True, 4), (2, "trt", True, 4),
           (3, "bgk", True, 5), (3, "trt", True, 5)]


@pytest.mark.parametrize("dims,collision,les,variant", TUNNELS)
def test_wind_tunnel_kernels_equal_generic(dims, collision, les, variant, monkeypatch):
    """The open wind tunnel of the serving trace (velocity inlet, convective
    outlet, obstacle, slip walls; with and without Smagorinsky LES) takes the
    kernels compiled for its feature word: FP32 states within 1e-6 of max|f|
    of the generic kernels' after 40 steps, drag histories within 1e-5."""
    monkeypatch.delenv("AERO_B200_GENERIC_KERNELS", raising=False)
    a = _tunnel(dims, collision, les)
    assert a._engine.kernel_variant() == variant
    ra = a.run(40, check_every=20, verbose=False)
    monkeypatch.setenv("AERO_B200_GENERIC_KERNELS", "1")
    b = _tunnel(dims, collision, les)
    assert b._engine.kernel_variant() == 0
    rb = b.run(40, check_every=20, verbose=False)
    np.testing.assert_allclose(a.f, b.f, rtol=0, atol=1e-6 * np.abs(b.f).max())
    cdb = np.array(rb["Cd_history"])
    np.testing.assert_allclose(np.array(ra["Cd_history"]), cdb, rtol=0, atol=1e-5 * np.abs(cdb).max())


def test_batch_class_keeps_its_members_kernel_set(monkeypatch):
    """A batch puts lattices of different kernel sets in different classes:
    each member's populations equal those of the same lattice alone in a
    batch, bit for bit, with the tunnel (specialised) and a sponge variant
    (generic) of the same collision in one batch."""
    from aero_b200 import Batch
    monkeypatch.delenv("AERO_B200_GENERIC_KERNELS", raising=False)
    makes = [lambda: _tunnel(2, "trt", False), lambda: _tunnel(2, "trt", False, sponge_thickness=8)]
    alone = []
    for m in makes:
        s = m()
        b = Batch(max_members=1)
        b.add(s)
        b.step(25)
        alone.append(s._engine.get_state()[0])
        b.remove(s)
        b.close()
    mix = [m() for m in makes]
    assert [s._engine.kernel_variant() for s in mix] == [2, 0]
    b = Batch(max_members=2)
    for s in mix:
        b.add(s)
    b.step(25)
    for s, f in zip(mix, alone):
        np.testing.assert_array_equal(s._engine.get_state()[0], f)
    b.close()


def test_other_feature_words_take_the_generic_kernels(monkeypatch):
    monkeypatch.delenv("AERO_B200_GENERIC_KERNELS", raising=False)
    for extra in (dict(precision="fp64"), dict(collision="bgk"), dict(buoyancy=False),
                  dict(scalar_lattice="full"), dict(les_model="smagorinsky"), dict(wall_bc="slip")):
        kw = dict(precision="fp32")
        kw.update(extra)
        s = _channel(**kw)
        assert s._engine.kernel_variant() == 0, extra
