"""The D3Q19 BGK / TRT step with the LES velocity stencil in shared memory
(step kernel 6, k_step_les) against the two-pass form (a moments pass, then
the per-cell step reading its velocity side output) and the reference
fixtures.

The fused kernel evaluates the same per-cell chain and the same velocity
arithmetic as the moments pass; only the compiler's fusion of a product
into a sum may differ between the two kernels, one rounding of the storage
arithmetic per operation: FP64 1e-12, FP32 1e-6, FP16 1e-4 of max|f| after
the steps below.  Against the reference fixtures the FP64 bound of the
golden parity tests holds (1e-10 max|f|, histories 1e-8).
"""

import numpy as np
import pytest

from tests.golden_cases import load_case

pytestmark = pytest.mark.gpu

LES = 6
TOL = {"fp64": 1e-12, "fp32": 1e-6, "fp16s": 1e-4, "bf16s": 1e-3}
CASES_3D_LES = ["c3d_trt_wale_periodic_bodyforce_thermal", "c3d_trt_moving_smag_vandriest",
                "c3d_bgk_smag_bodyforce_open"]


@pytest.mark.parametrize("name", CASES_3D_LES)
def test_fused_les_fp64_matches_reference_golden(name):
    from tests.test_gpu_parity import _solver
    c = load_case(name)
    s = _solver(c, precision="fp64")
    s._engine.set_step_kernel(LES)
    assert s._engine.get_step_kernel() == LES and s._engine.les_fused()
    cd = [s._step()[0] for _ in range(c["steps"])]
    scale = np.abs(c["f"]).max()
    np.testing.assert_allclose(s.f, c["f"], rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(s._f_outlet_prev, c["f_outlet_prev"], rtol=0, atol=1e-10 * scale)
    if "g" in c:
        np.testing.assert_allclose(s.g, c["g"], rtol=0, atol=1e-10 * np.abs(c["g"]).max())
    ref = c["hist"]["Cd"]
    np.testing.assert_allclose(cd, ref, rtol=0, atol=1e-8 * max(np.abs(ref).max(), 1e-3))


def _channel(precision, kernel, collision="trt", les_model="wale", thermal=True, steps=30,
             nz=20, ny=22, nx=70, streamwise_bc="open"):
    """A sphere in a channel spanning several tiles in x and y (partial ones
    too) and several z chunks: Bouzidi links, no-slip walls, sponge,
    convective outlet, WALE or Smagorinsky, D3Q7 scalar with buoyancy."""
    from aero_b200 import Solver3D, Sphere
    sph = Sphere(radius=4, cx_frac=0.3, cy_frac=0.45, cz_frac=0.5)
    solid, phi = sph.mark_solid(nz, ny, nx), sph.sdf_field(nz, ny, nx)
    kw = dict(omega=1 / 0.8, u0=0.05, D=sph.reference_length(), collision=collision, trt_lambda=0.25, les=True,
              les_model=les_model, les_cs=0.3, bouzidi=True, phi=phi, wall_bc="noslip", outlet_bc="convective",
              sponge_thickness=6, streamwise_bc=streamwise_bc, thermal=thermal, alpha_T=0.02, buoyancy=thermal,
              g_gravity=1e-3, beta=1.0, scalar_lattice="reduced")
    s = Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, precision=precision, **kw)
    rng = np.random.default_rng(11)
    shp = solid.shape
    s.set_equilibrium_state(ux=0.05 + 0.01 * rng.uniform(-1, 1, shp), uy=0.01 * rng.uniform(-1, 1, shp),
                            uz=0.01 * rng.uniform(-1, 1, shp),
                            T=(0.5 + 0.05 * rng.uniform(-1, 1, shp)) if thermal else None)
    s._engine.set_step_kernel(kernel)
    r = s.run(steps, check_every=steps + 1, verbose=False)
    return s, np.array(r["Cd_history"])


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16s"])
@pytest.mark.parametrize("collision,les_model", [("trt", "wale"), ("bgk", "smagorinsky")])
def test_fused_les_equals_two_pass(precision, collision, les_model):
    a, cda = _channel(precision, LES, collision, les_model)
    b, cdb = _channel(precision, 0, collision, les_model)
    tol = TOL[precision]
    np.testing.assert_allclose(a.f, b.f, rtol=0, atol=tol * np.abs(b.f).max())
    np.testing.assert_allclose(a.g, b.g, rtol=0, atol=tol * np.abs(b.g).max())
    np.testing.assert_allclose(a._f_outlet_prev, b._f_outlet_prev, rtol=0, atol=tol * np.abs(b.f).max())
    np.testing.assert_allclose(cda, cdb, rtol=0, atol=10 * tol * np.abs(cdb).max())


def test_fused_les_periodic_with_body_force():
    """Streamwise periodic with a body force (the configuration-3 form)."""
    from aero_b200 import Solver3D, Box

    def run(kernel):
        nz, ny, nx = 18, 20, 64
        box = Box(width=8, height=6, depth=18, cx_frac=0.3, cy_frac=3 / 20, cz_frac=0.5)
        solid = box.mark_solid(nz, ny, nx)
        s = Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, omega=1 / 0.8, u0=0.05, D=6.0, collision="trt",
                     trt_lambda=3 / 16, les=True, les_model="wale", les_cs=0.5, wall_bc="noslip",
                     streamwise_bc="periodic", body_force_x=1e-5, thermal=True, alpha_T=0.01, buoyancy=True,
                     g_gravity=1e-3, beta=1.0, scalar_lattice="reduced", precision="fp32")
        s._engine.set_step_kernel(kernel)
        s.run(40, check_every=41, verbose=False)
        return s

    a, b = run(LES), run(0)
    np.testing.assert_allclose(a.f, b.f, rtol=0, atol=1e-6 * np.abs(b.f).max())
    np.testing.assert_allclose(a.g, b.g, rtol=0, atol=1e-6 * np.abs(b.g).max())


def test_fused_les_refuses_other_lattices():
    from aero_b200 import Solver3D
    from aero_b200._lib import AeroError
    solid = np.zeros((6, 6, 16), dtype=bool)
    for kw in (dict(collision="mrt", les=True), dict(collision="bgk", les=False)):
        s = Solver3D(Nz=6, Ny=6, Nx=16, solid=solid, omega=1.5, u0=0.05, D=4.0, **kw)
        with pytest.raises(AeroError):
            s._engine.set_step_kernel(LES)
