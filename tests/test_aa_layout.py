"""The AA layout (layout="aa"): one population buffer updated in place.

A step reads each cell's pulled populations from the slots it then
overwrites (alternating between two slot layouts), so no second buffer is
needed; the reads that cross cells inside a step (the pre-stream values of
link cells, the pulled populations of the plane x = nx-2 that the outlet and
recycling cells re-evaluate) are staged before the step, except that an
outlet cell whose x = nx-2 neighbour runs in its own warp takes that state by
warp shuffles (nx-1 not a multiple of 32; both forms are covered below).  Between aero_step
calls the buffer holds the post-boundary state itself (the call's last step
stores it; the next call collides it in place), so the state read back is
the reference's self.f as with two buffers.

Checked: every reference fixture in FP64 with one step per call (each call
ends with the state-storing step) at the bound of the golden parity tests
(1e-10 max|f|, histories 1e-8); the AA and A/B layouts against each other
over multi-step calls (FP64 1e-12, FP32 1e-6, FP16 1e-4 of max|f|: the same
arithmetic, the set state collided by the from-state kernel instead of
inside the step kernel); the halved population memory; the kernels and
batches the layout does not take.
"""

import numpy as np
import pytest

from tests.golden_cases import CASES, load_case

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-6, "fp16s": 1e-4}


@pytest.mark.parametrize("name", CASES)
def test_aa_fp64_matches_reference_golden(name):
    from tests.test_gpu_parity import _solver
    c = load_case(name)
    s = _solver(c, precision="fp64", layout="aa")
    assert s.layout == "aa"
    cd = [s._step()[0] for _ in range(c["steps"])]
    scale = np.abs(c["f"]).max()
    np.testing.assert_allclose(s.f, c["f"], rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(s._f_outlet_prev, c["f_outlet_prev"], rtol=0, atol=1e-10 * scale)
    if "g" in c:
        np.testing.assert_allclose(s.g, c["g"], rtol=0, atol=1e-10 * np.abs(c["g"]).max())
    ref = c["hist"]["Cd"]
    np.testing.assert_allclose(cd, ref, rtol=0, atol=1e-8 * max(np.abs(ref).max(), 1e-3))


def _sphere(precision, layout, nx=48, **extra):
    from aero_b200 import Solver3D, Sphere
    nz, ny = 18, 20
    sph = Sphere(radius=4, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
    solid, phi = sph.mark_solid(nz, ny, nx), sph.sdf_field(nz, ny, nx)
    kw = dict(omega=1 / 0.7, u0=0.05, D=sph.reference_length(), collision="mrt", bouzidi=True, phi=phi,
              wall_bc="slip", outlet_bc="convective", sponge_thickness=6, inlet_perturbation=0.05)
    kw.update(extra)
    return Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, precision=precision, layout=layout, **kw)


def _thermal_box(precision, layout):
    from aero_b200 import Box, Solver3D
    nz, ny, nx = 14, 16, 40
    box = Box(width=6, height=5, depth=14, cx_frac=0.3, cy_frac=2.5 / 16, cz_frac=0.5)
    solid, phi = box.mark_solid(nz, ny, nx), box.sdf_field(nz, ny, nx)
    return Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, omega=1 / 0.8, u0=0.05, D=5.0, collision="trt",
                    trt_lambda=0.25, les=True, les_model="wale", les_cs=0.3, bouzidi=True, phi=phi,
                    wall_bc="noslip", streamwise_bc="periodic", body_force_x=1e-5, thermal=True, alpha_T=0.02,
                    buoyancy=True, g_gravity=1e-3, beta=1.0, scalar_lattice="reduced", precision=precision,
                    layout=layout)


def _cylinder(precision, layout):
    from aero_b200 import Cylinder, Solver
    ny, nx = 40, 90
    cyl = Cylinder(radius=5, cx_frac=0.3, cy_frac=0.5)
    solid, phi = cyl.mark_solid(ny, nx), cyl.sdf_field(ny, nx)
    return Solver(Ny=ny, Nx=nx, solid=solid, omega=1 / 0.6, u0=0.05, D=cyl.reference_length(), collision="bgk",
                  bouzidi=True, phi=phi, wall_bc="noslip", outlet_bc="zerogradient", les=True,
                  precision=precision, layout=layout)


MAKERS = {
    "sphere_mrt_bouzidi_convective": lambda prec, lay: _sphere(prec, lay),
    # nx - 1 = 64: the x = nx-2 and nx-1 cells run in different warps, so the
    # outlet reads the staged plane instead of shuffling
    "sphere_mrt_bouzidi_convective_staged_outlet": lambda prec, lay: _sphere(prec, lay, nx=65),
    "sphere_bgk_les_recycling": lambda prec, lay: _sphere(prec, lay, collision="bgk", les=True,
                                                           streamwise_bc="recycling", outlet_bc="zerogradient",
                                                           body_force_x=1e-5),
    "box_trt_wale_thermal_periodic": _thermal_box,
    "cylinder_2d_bgk_les_zerograd": _cylinder,
}


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16s"])
@pytest.mark.parametrize("case", sorted(MAKERS))
def test_aa_equals_ab_over_multistep_calls(case, precision):
    if precision == "fp16s" and case.startswith("cylinder"):
        pytest.skip("16-bit storage is compared on the 3D cases")
    runs = {}
    for layout in ("ab", "aa"):
        s = MAKERS[case](precision, layout)
        rng = np.random.default_rng(2)
        shp = s.solid.shape
        s.set_equilibrium_state(ux=0.05 + 0.01 * rng.uniform(-1, 1, shp), uy=0.01 * rng.uniform(-1, 1, shp))
        # calls of 10, 10, 10 and 7 steps (graphs inside, the state stored at each call's end)
        r = s.run(37, check_every=10, verbose=False)
        s._step()
        runs[layout] = (s, np.array(r["Cd_history"]))
    (a, cda), (b, cdb) = runs["aa"], runs["ab"]
    tol = TOL[precision]
    np.testing.assert_allclose(a.f, b.f, rtol=0, atol=tol * np.abs(b.f).max())
    np.testing.assert_allclose(a._f_outlet_prev, b._f_outlet_prev, rtol=0, atol=tol * np.abs(b.f).max())
    if b.thermal:
        np.testing.assert_allclose(a.g, b.g, rtol=0, atol=tol * np.abs(b.g).max())
    np.testing.assert_allclose(cda, cdb, rtol=0, atol=10 * tol * max(np.abs(cdb).max(), 1e-3))
    fa, fb = a.field_statistics(), b.field_statistics()
    assert abs(fa["mass"] - fb["mass"]) <= 10 * tol * fb["mass"]


def test_auto_layout_takes_ab_when_it_fits_else_aa(monkeypatch):
    """layout="auto" keeps the faster two-buffer layout when its workspace
    fits the device's free memory with headroom, and otherwise builds the
    lattice in the AA layout, which then steps exactly as layout="aa"."""
    from aero_b200.engine import Engine
    s = _sphere("fp32", "auto")
    assert s.layout == "ab" and s._b200_options()["layout"] == "ab"
    monkeypatch.setattr(Engine, "AUTO_LAYOUT_FREE_SHARE", 0.0)
    a, b = _sphere("fp32", "auto"), _sphere("fp32", "aa")
    assert a.layout == "aa" and a._engine.workspace_bytes == b._engine.workspace_bytes
    ra, rb = a.run(12, check_every=13, verbose=False), b.run(12, check_every=13, verbose=False)
    np.testing.assert_array_equal(a.f, b.f)
    np.testing.assert_array_equal(ra["Cd_history"], rb["Cd_history"])


def test_aa_halves_population_memory():
    a, b = _sphere("fp32", "aa"), _sphere("fp32", "ab")
    one_buffer = 19 * 4 * ((18 * 20 * 48 + 63) // 64 * 64)
    assert b._engine.workspace_bytes - a._engine.workspace_bytes >= 0.9 * one_buffer


def test_aa_refuses_other_kernels_and_small_batch_members():
    """The AA layout takes the per-cell step kernel only, and joins a batch
    only with at least 2^20 cells (tests/test_batch.py covers that case)."""
    from aero_b200 import Batch
    from aero_b200._lib import AeroError
    s = _sphere("fp16s", "aa")
    for k in (1, 2, 3, 4, 5):
        with pytest.raises(AeroError):
            s._engine.set_step_kernel(k)
    s._engine.set_step_kernel(0)
    b = Batch(max_members=2, device=s._engine.device)
    with pytest.raises(AeroError):
        b.add(s)
    b.close()
    with pytest.raises(ValueError):
        _sphere("fp32", "ba")
