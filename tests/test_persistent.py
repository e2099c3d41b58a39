"""Persistent runs of small lattices (k_run_small): one cooperative launch
takes all steps of a call, cell blocks stepping the lattice and one block
finalising each step's forces while the next step runs.  The per-cell code
and the finalisation order are those of the per-step launches, so
populations, outlet and scalar state, force histories and the force profile
agree with the same lattice stepped by per-step launches
(aero_set_persistent(0)) over calls of several lengths: bit for bit for
BGK / TRT; for MRT up to the rounding of the compiled variant (the two
kernels contract the adapted-basis products into FMAs differently), FP64
1e-13, FP32 1e-6 and FP16 1e-4 of max|f| after 39 steps."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _channel(**kw):
    from aero_b200 import Cylinder, Solver
    ny, nx = 60, 120
    cyl = Cylinder(radius=6, cx_frac=0.25, cy_frac=0.5)
    solid, phi = cyl.mark_solid(ny, nx), cyl.sdf_field(ny, nx)
    base = dict(omega=1 / 0.56, u0=0.05, D=cyl.reference_length(), wall_bc="noslip", outlet_bc="zerogradient",
                bouzidi=True, phi=phi)
    base.update(kw)
    return Solver(Ny=ny, Nx=nx, solid=solid, **base)


def _sphere(**kw):
    from aero_b200 import Solver3D, Sphere
    nz, ny, nx = 20, 22, 48
    sph = Sphere(radius=4, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
    solid, phi = sph.mark_solid(nz, ny, nx), sph.sdf_field(nz, ny, nx)
    base = dict(omega=1 / 0.7, u0=0.05, D=sph.reference_length(), collision="mrt", les=True, bouzidi=True,
                phi=phi, wall_bc="slip", outlet_bc="convective", sponge_thickness=6, inlet_perturbation=0.05)
    base.update(kw)
    return Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, **base)


CASES = {
    "channel_2d_bgk_bouzidi_zerograd": lambda p: _channel(precision=p),
    "channel_2d_trt_thermal_convective": lambda p: _channel(precision=p, collision="trt", omega=1 / 0.8,
                                                            outlet_bc="convective", thermal=True, alpha_T=0.02,
                                                            buoyancy=True, g_gravity=1e-3, beta=1.0),
    "channel_2d_synthetic_inflow": lambda p: _channel(precision=p, synthetic_inflow=True,
                                                      synthetic_inflow_intensity=0.02),
    "sphere_3d_mrt_les_bouzidi_sponge": lambda p: _sphere(precision=p),
    "sphere_3d_mrt_body_force_periodic": lambda p: _sphere(precision=p, streamwise_bc="periodic",
                                                           body_force_x=1e-5, sponge_thickness=0),
}


@pytest.mark.parametrize("precision", ["fp32", "fp64", "fp16s"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_persistent_run_equals_per_step_launches(case, precision):
    runs = {}
    for persistent in (True, False):
        s = CASES[case](precision)
        s._engine.set_persistent(persistent)
        rng = np.random.default_rng(7)
        shp = s.solid.shape
        s.set_equilibrium_state(ux=0.05 + 0.01 * rng.uniform(-1, 1, shp), uy=0.01 * rng.uniform(-1, 1, shp))
        # calls of 10, 10, 10 and 7 steps, then single steps
        r = s.run(37, check_every=10, verbose=False)
        s._step()
        s._step()
        runs[persistent] = (s, r)
    (a, ra), (b, rb) = runs[True], runs[False]
    tol = 0.0 if b.collision != "mrt" else {"fp64": 1e-13, "fp32": 1e-6, "fp16s": 1e-4}[precision]
    np.testing.assert_allclose(a.f, b.f, rtol=0, atol=tol * np.abs(b.f).max())
    np.testing.assert_allclose(a._f_outlet_prev, b._f_outlet_prev, rtol=0, atol=tol * np.abs(b.f).max())
    if b.thermal:
        np.testing.assert_array_equal(a.g, b.g)
    for k in ("Cd_history", "Cd_p_history", "Cd_v_history"):
        ref = np.array(rb[k])
        np.testing.assert_allclose(np.array(ra[k]), ref, rtol=0, atol=10 * tol * np.abs(ref).max())
    pa, pb = a._engine.read_profile(), b._engine.read_profile()
    np.testing.assert_allclose(pa, pb, rtol=0, atol=10 * tol * np.abs(pb).max())
    assert a.status() == b.status() == 0
    assert a.step_count == b.step_count == 39


def test_persistent_run_long_call_wraps_the_history_ring():
    """A call longer than the force-history ring: the ring is read in chunks
    by run(); the persistent runner writes its slots as the per-step path
    does, and the drag histories agree bit for bit."""
    out = []
    for persistent in (True, False):
        s = _channel(precision="fp32", hist_capacity=64)
        s._engine.set_persistent(persistent)
        r = s.run(200, check_every=201, verbose=False)
        out.append((np.array(r["Cd_history"]), s.f))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    assert len(out[0][0]) == 200
