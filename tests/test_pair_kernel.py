"""The two-cells-per-thread D3Q19 step kernel (step kernel 4, packed FP32
arithmetic; MRT, BGK and TRT) against the per-cell kernel, the reference
fixtures and the FP64 oracle.

Tolerances: each lane runs the per-cell step's operations in the same order;
only the fusion of a product into a sum may differ, an FP32 rounding per
operation.  After 60 steps the states agree to 1e-6 of max|f| with FP32
storage, and to the storage's own resolution with 16-bit storage, where one
such rounding can move a value by one 16-bit step: 1e-4 (FP16, 11-bit
significand of the scaled deviation) and 1e-3 (BF16, 8 bits) of max|f|."""

import numpy as np
import pytest

from tests.golden_cases import load_case

pytestmark = pytest.mark.gpu

PAIR = 4
TOL = {"fp32": 1e-6, "fp16s": 1e-4, "bf16s": 1e-3}


# TRT runs at tau 0.8: with the reference's lambda semantics (trt2d.py:8-18)
# tau 0.6 gives s- = 10 and diverges.  BGK and TRT run with Smagorinsky LES,
# so each cell of a pair relaxes at its own rate.
COLL = {"mrt": dict(collision="mrt", omega=1 / 0.6),
        "bgk": dict(collision="bgk", omega=1 / 0.6, les=True, les_cs=0.15),
        "trt": dict(collision="trt", omega=1 / 0.8, les=True, les_cs=0.15, trt_lambda=0.25)}


def _sphere(precision, kernel, nz=20, ny=22, nx=64, steps=60, collision="mrt"):
    from aero_b200 import Solver3D, Sphere
    sph = Sphere(radius=4, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
    solid, phi = sph.mark_solid(nz, ny, nx), sph.sdf_field(nz, ny, nx)
    kw = dict(u0=0.05, D=sph.reference_length(), bouzidi=True, phi=phi, wall_bc="slip",
              outlet_bc="convective", sponge_thickness=6, inlet_perturbation=0.05, **COLL[collision])
    s = Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, precision=precision, **kw)
    s._engine.set_step_kernel(kernel)
    assert s._engine.get_step_kernel() == kernel
    r = s.run(steps, check_every=steps + 1, verbose=False)
    return s.f, np.array(r["Cd_history"])


@pytest.mark.parametrize("collision", ["mrt", "bgk", "trt"])
@pytest.mark.parametrize("precision", ["fp32", "fp16s", "bf16s"])
def test_pair_kernel_equals_per_cell_kernel(precision, collision):
    """3D Bouzidi sphere with slip walls (wall rows), sponge and convective
    outlet (per-cell edge columns), y and z wrap; MRT, and BGK / TRT with LES."""
    fa, cda = _sphere(precision, PAIR, collision=collision)
    fb, cdb = _sphere(precision, 0, collision=collision)
    np.testing.assert_allclose(fa, fb, rtol=0, atol=TOL[precision] * np.abs(fb).max())
    np.testing.assert_allclose(cda, cdb, rtol=0, atol=10 * TOL[precision] * np.abs(cdb).max())


@pytest.mark.parametrize("nx", [64, 200, 520])
@pytest.mark.parametrize("precision", ["fp16s", "bf16s"])
def test_pair_kernel_equals_batched_pair_kernel(precision, nx):
    """A 16-bit lattice alone in a batch runs the batched pair kernel (its
    parameters in shared memory, blocks found on the batch's work-list); the
    same lattice alone runs the single-lattice pair kernel.  Both do the same
    operations, so populations and drag agree bit for bit.  Rows of 30, 98
    and 258 pairs: one partial warp, several warps, and three blocks of which
    the last holds two pairs."""
    from aero_b200 import Batch, Solver3D, Sphere

    def make():
        nz, ny = 10, 12
        sph = Sphere(radius=3, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
        solid, phi = sph.mark_solid(nz, ny, nx), sph.sdf_field(nz, ny, nx)
        s = Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, omega=1 / 0.7, u0=0.05, D=6.0, collision="mrt",
                     bouzidi=True, phi=phi, wall_bc="slip", outlet_bc="convective", sponge_thickness=6,
                     precision=precision)
        rng = np.random.default_rng(5)
        s.set_equilibrium_state(ux=0.05 + 0.01 * rng.uniform(-1, 1, solid.shape),
                                uy=0.01 * rng.uniform(-1, 1, solid.shape), uz=0.01 * rng.uniform(-1, 1, solid.shape))
        return s

    a = make()
    a._engine.set_step_kernel(PAIR)
    assert a._engine.get_step_kernel() == PAIR
    r = a.run(30, check_every=31, verbose=False)
    b = make()
    bat = Batch(max_members=1)
    bat.add(b)
    bat.step(30)
    np.testing.assert_array_equal(a._engine.get_state()[0], b._engine.get_state()[0])
    cd = b._coefficients(b._engine.read_forces())["Cd"]
    np.testing.assert_array_equal(cd, np.array(r["Cd_history"]))
    bat.remove(b)
    bat.close()


def test_pair_kernel_sphere_matches_oracle_300_steps():
    """The acceptance bound of the plain FP32 form through the pair kernel:
    rel-L2(rho, u) <= 1e-5 after 300 steps against the FP64 oracle."""
    from aero_b200 import Solver3D, Sphere
    from oracle.oracle import OracleSolver
    from tests.test_gpu_parity import _macro, rel_l2
    nz, ny, nx = 40, 40, 96
    sph = Sphere(radius=6, cx_frac=0.25, cy_frac=0.5, cz_frac=0.5)
    solid, phi = sph.mark_solid(nz, ny, nx), sph.sdf_field(nz, ny, nx)
    kw = dict(omega=1 / 0.6, u0=0.05, D=sph.reference_length(), collision="mrt", bouzidi=True,
              phi=phi, wall_bc="slip", outlet_bc="convective", sponge_thickness=8)
    s = Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, precision="fp32", **kw)
    s._engine.set_step_kernel(PAIR)
    o = OracleSolver(solid=solid, **kw)
    s.run(300, check_every=301, verbose=False)
    for _ in range(300):
        o.step_raw()
    got, ref = _macro(s.f, 3), _macro(o.f, 3)
    assert rel_l2(got[0], ref[0]) <= 1e-5
    assert rel_l2(np.stack(got[1:]), np.stack(ref[1:])) <= 1e-5


@pytest.mark.parametrize("name", ["c3d_mrt_noslip_zerograd", "c3d_mrt_smag_bouzidi_sponge"])
def test_pair_kernel_close_to_reference_fixture(name):
    from tests.test_gpu_parity import _macro, _solver, rel_l2
    c = load_case(name)
    s = _solver(c, precision="fp32")
    s._engine.set_step_kernel(PAIR)
    cd = [s._step()[0] for _ in range(c["steps"])]
    got, ref = _macro(s.f, 3), _macro(c["f"], 3)
    assert rel_l2(got[0], ref[0]) <= 1e-5
    assert rel_l2(np.stack(got[1:]), np.stack(ref[1:])) <= 1e-5
    np.testing.assert_allclose(cd, c["hist"]["Cd"], rtol=0, atol=1e-4 * np.abs(c["hist"]["Cd"]).max())


def test_pair_kernel_nan_guard():
    """A NaN planted in plain fluid cells is caught by the divergence guard."""
    from tests.test_gpu_parity import _solver
    c = load_case("c3d_mrt_noslip_zerograd")
    s = _solver(c, precision="fp32")
    s._engine.set_step_kernel(PAIR)
    s._step()
    assert s.status() == 0
    f = s.f
    f[:, 4, 5, 8] = np.nan  # x = 8, an interior row
    s.f = f
    s._step()
    s._step()
    assert s.status() & 1


def test_pair_kernel_refused_outside_its_cover():
    from aero_b200 import Solver3D, Sphere
    from aero_b200._lib import AeroError

    def make(nx=32, **kw):
        sph = Sphere(radius=3, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
        solid = sph.mark_solid(12, 12, nx)
        args = dict(omega=1 / 0.6, u0=0.05, D=sph.reference_length(), collision="mrt")
        args.update(kw)
        return Solver3D(Nz=12, Ny=12, Nx=nx, solid=solid, **args)

    for s in (make(nx=33), make(precision="fp64"), make(body_force_x=1e-6, streamwise_bc="periodic")):
        with pytest.raises(AeroError, match="AERO_ERR_UNSUPPORTED"):
            s._engine.set_step_kernel(PAIR)
        assert s._engine.get_step_kernel() == 0


# ---------------------------------------------------------------------------
# The four-cells-per-thread kernel (step kernel 5, 16-bit storage)
# ---------------------------------------------------------------------------
QUAD = 5


@pytest.mark.parametrize("collision", ["mrt", "bgk", "trt"])
@pytest.mark.parametrize("precision", ["fp16s", "bf16s"])
def test_quad_kernel_equals_per_cell_and_pair_kernels(precision, collision):
    """Open sphere lattice (inlet / outlet edge columns per cell, slip-wall
    rows, Bouzidi link cells, sponge); nx = 64 leaves the row's last warp
    partly idle (14 quads), so the shuffles' edge lanes are exercised."""
    fq, cdq = _sphere(precision, QUAD, collision=collision)
    fc, cdc = _sphere(precision, 0, collision=collision)
    fp, _ = _sphere(precision, PAIR, collision=collision)
    np.testing.assert_allclose(fq, fc, rtol=0, atol=TOL[precision] * np.abs(fc).max())
    np.testing.assert_allclose(cdq, cdc, rtol=0, atol=10 * TOL[precision] * np.abs(cdc).max())
    np.testing.assert_allclose(fq, fp, rtol=0, atol=TOL[precision] * np.abs(fp).max())


@pytest.mark.parametrize("nx", [32, 136, 520])
@pytest.mark.parametrize("precision", ["fp16s", "bf16s"])
def test_quad_kernel_periodic_rows_wrap(precision, nx):
    """Streamwise periodic lattice: the quads cover whole rows, the x wrap of
    the first and last quad comes from the edge lanes' own loads; rows of 8,
    34 and 130 quads (one partial warp, several warps, several blocks)."""
    from aero_b200 import Solver3D, Sphere

    def run(kernel):
        nz, ny = 10, 12
        sph = Sphere(radius=3, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
        solid, phi = sph.mark_solid(nz, ny, nx), sph.sdf_field(nz, ny, nx)
        s = Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, omega=1 / 0.7, u0=0.05, D=6.0, collision="mrt",
                     bouzidi=True, phi=phi, wall_bc="noslip", streamwise_bc="periodic", precision=precision)
        rng = np.random.default_rng(3)
        s.set_equilibrium_state(ux=0.05 + 0.01 * rng.uniform(-1, 1, solid.shape),
                                uy=0.01 * rng.uniform(-1, 1, solid.shape), uz=0.01 * rng.uniform(-1, 1, solid.shape))
        s._engine.set_step_kernel(kernel)
        assert s._engine.get_step_kernel() == kernel
        s.run(40, check_every=41, verbose=False)
        return s.f

    fq, fc = run(QUAD), run(0)
    np.testing.assert_allclose(fq, fc, rtol=0, atol=TOL[precision] * np.abs(fc).max())


def test_quad_kernel_refuses_other_lattices():
    from aero_b200 import Solver3D
    from aero_b200._lib import AeroError
    solid = np.zeros((6, 6, 30), dtype=bool)
    for kw in (dict(precision="fp32"), dict(precision="fp16s", body_force_x=1e-5, streamwise_bc="periodic")):
        s = Solver3D(Nz=6, Ny=6, Nx=30, solid=solid, omega=1.5, u0=0.05, D=4.0, **kw)
        with pytest.raises(AeroError):
            s._engine.set_step_kernel(QUAD)
    s = Solver3D(Nz=6, Ny=6, Nx=30, solid=solid, omega=1.5, u0=0.05, D=4.0, precision="fp16s")
    with pytest.raises(AeroError):  # nx = 30 is not a multiple of 4
        s._engine.set_step_kernel(QUAD)
