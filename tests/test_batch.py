"""Batched stepping (aero_batch_*): members of mixed class advance in the
batch exactly as they do alone, join and leave between steps, and the
device convergence detector follows analyze_convergence
(aero/diagnostics.py:87-120).  The CPU tests cover argument checking of
the C ABI without a GPU."""

import ctypes

import numpy as np
import pytest


def _lib():
    from aero_b200 import _lib
    return _lib.load(build_if_missing=False)


def test_batch_create_checks_arguments():
    lib = _lib()
    h = ctypes.c_void_p()
    assert lib.aero_batch_create(0, ctypes.byref(h)) != 0
    assert lib.aero_batch_create(4, ctypes.byref(h)) == 0
    n = ctypes.c_uint64()
    assert lib.aero_batch_workspace_size(h, ctypes.byref(n)) == 0 and n.value > 0
    assert lib.aero_batch_bind_workspace(h, None, n.value) != 0
    out = np.zeros(7)
    assert lib.aero_batch_converge(h, 10, 1e-3, out.ctypes.data, None) != 0  # not bound
    assert lib.aero_batch_step(h, 1, None) != 0  # not bound
    size = ctypes.c_int32(-1)
    assert lib.aero_batch_size(h, ctypes.byref(size)) == 0 and size.value == 0
    assert lib.aero_batch_destroy(h) == 0


def _cases():
    """Solver constructors of mixed class: 2D/3D, BGK/TRT/MRT, LES (moments
    pass), thermal scalar, fp32/fp64/fp16s/bf16s, Bouzidi, uneven sizes.  The
    16-bit 3D members without body force or scalar and with even nx run in
    the two-cells-per-thread batch kernel."""
    from aero_b200 import Box, Cylinder, Rectangle, Solver, Solver3D, Sphere

    def c2d(ny, nx, geo, **kw):
        solid = geo.mark_solid(ny, nx)
        phi = geo.sdf_field(ny, nx) if kw.get("bouzidi") else None
        return lambda: Solver(Ny=ny, Nx=nx, solid=solid, D=geo.reference_length(), phi=phi, **kw)

    def c3d(nz, ny, nx, geo, **kw):
        solid = geo.mark_solid(nz, ny, nx)
        phi = geo.sdf_field(nz, ny, nx) if kw.get("bouzidi") else None
        return lambda: Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, D=geo.reference_length(), phi=phi, **kw)

    return [
        c2d(40, 96, Cylinder(radius=6, cx_frac=0.3, cy_frac=0.5), omega=1 / 0.56, u0=0.05,
            wall_bc="noslip", outlet_bc="zerogradient", bouzidi=True, precision="fp32"),
        c2d(34, 70, Rectangle(width=10, height=8, cx_frac=0.3, cy_frac=0.5), omega=1 / 0.8, u0=0.05,
            collision="trt", wall_bc="slip", outlet_bc="convective", les=True, les_cs=0.15, precision="fp32"),
        c2d(30, 64, Cylinder(radius=4, cx_frac=0.3, cy_frac=0.5), omega=1 / 0.6, u0=0.04,
            collision="mrt", wall_bc="noslip", sponge_thickness=8, precision="fp64"),
        c3d(16, 18, 40, Sphere(radius=4, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5), omega=1 / 0.6, u0=0.05,
            collision="mrt", bouzidi=True, wall_bc="slip", outlet_bc="convective", sponge_thickness=6,
            precision="fp32"),
        c3d(12, 14, 30, Sphere(radius=3, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5), omega=1 / 0.7, u0=0.05,
            collision="bgk", les=True, les_cs=0.1, wall_bc="noslip", precision="fp16s"),
        c3d(14, 12, 36, Sphere(radius=3, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5), omega=1 / 0.8, u0=0.05,
            collision="trt", trt_lambda=0.25, les=True, les_cs=0.12, wall_bc="slip", sponge_thickness=5,
            precision="fp16s"),
        c3d(12, 16, 24, Box(width=4, height=4, depth=12, cx_frac=0.3, cy_frac=0.25, cz_frac=0.5),
            omega=1 / 0.8, u0=0.05, collision="trt", trt_lambda=0.25, wall_bc="noslip", streamwise_bc="periodic",
            body_force_x=1e-6, thermal=True, alpha_T=0.02, buoyancy=True, g_gravity=1e-4, beta=1.0,
            T_ref=0.5, precision="bf16s"),
    ]


def _alone(make, steps):
    s = make()
    r = s.run(steps, check_every=steps + 1, verbose=False)
    return s.f, np.array(r["Cd_history"])


# The batch kernels run the per-cell code of the single-lattice kernels, but
# they are separate compilations, so floating-point contraction may differ in
# the last bit: the batch agrees with the single-lattice API to these
# fractions of max|f| (and of max|Cd|) per storage format.
TOL = {"fp64": 1e-12, "fp32": 1e-6, "fp16s": 2e-3, "bf16s": 2e-3}


def _close(s, f, f_ref, cd=None, cd_ref=None):
    tol = TOL[s.precision]
    np.testing.assert_allclose(f, f_ref, rtol=0, atol=tol * np.abs(f_ref).max())
    if cd is not None:
        np.testing.assert_allclose(cd, cd_ref, rtol=0, atol=tol * max(np.abs(cd_ref).max(), 1e-3))


@pytest.mark.gpu
def test_batch_members_match_alone():
    from aero_b200 import Batch
    makes = _cases()
    steps = 31  # odd: the batch ends on the other buffer parity
    ref = [_alone(m, steps) for m in makes]
    b = Batch(max_members=8)
    solvers = [m() for m in makes]
    for s in solvers:
        b.add(s)
    b.step(steps)
    for s, (f_ref, cd_ref) in zip(solvers, ref):
        cd = s._coefficients(s._engine.read_forces())["Cd"]
        b.remove(s)
        _close(s, s.f, f_ref, cd, cd_ref)
    b.close()


@pytest.mark.gpu
def test_batch_result_same_alone_and_in_the_mix():
    """Each case gives bit-identical populations and forces whether it runs
    alone in a batch or in a batch with every other case: the members of a
    batch share launches but no data."""
    from aero_b200 import Batch
    makes = _cases()
    steps = 24
    alone = []
    for m in makes:
        b = Batch(max_members=1)
        s = m()
        b.add(s)
        b.step(steps)
        alone.append((s._engine.read_forces(), s._engine.get_state()[0]))
        b.remove(s)
        b.close()
    b = Batch(max_members=8)
    mix = [m() for m in makes]
    for s in mix:
        b.add(s)
    b.step(10)
    b.step(steps - 10)
    for s, (raw, f) in zip(mix, alone):
        np.testing.assert_array_equal(s._engine.read_forces(), raw)
        np.testing.assert_array_equal(s._engine.get_state()[0], f)
    b.close()


@pytest.mark.gpu
def test_batch_join_and_leave_between_steps():
    """Continuous batching: members join and leave at different steps and
    end in the same state as when run alone for the same number of steps."""
    from aero_b200 import Batch
    makes = _cases()[:4]
    b = Batch(max_members=4)
    s = [m() for m in makes]
    b.add(s[0])
    b.step(7)
    b.add(s[1])
    b.add(s[2])
    b.step(10)
    b.remove(s[0])      # 17 steps
    b.add(s[3])
    b.step(5)
    b.remove(s[2])      # 15 steps
    b.step(4)           # s[1]: 19, s[3]: 9
    done = {0: 17, 1: 19, 2: 15, 3: 9}
    b.remove(s[1])
    b.remove(s[3])
    for k, n in done.items():
        f_ref, _ = _alone(makes[k], n)
        assert s[k].step_count == n
        _close(s[k], s[k].f, f_ref)
    # a solver that left the batch steps on its own again
    s[0].run(3, check_every=10, verbose=False)
    f_ref, _ = _alone(makes[0], 20)
    _close(s[0], s[0].f, f_ref)
    b.close()


@pytest.mark.gpu
def test_member_cannot_step_alone():
    from aero_b200 import Batch
    from aero_b200._lib import AeroError
    s = _cases()[0]()
    b = Batch(max_members=2)
    b.add(s)
    with pytest.raises(AeroError, match="batch member"):
        s._engine.step(1)
    b.remove(s)
    s._engine.step(1)
    b.close()


@pytest.mark.gpu
def test_device_convergence_matches_analyze_convergence():
    from aero_b200 import Batch
    from aero_b200.diagnostics import analyze_convergence
    makes = _cases()
    b = Batch(max_members=8)
    solvers = [makes[0](), makes[3]()]
    for s in solvers:
        b.add(s)
    W = 60
    out = b.converge(W, 1e-3)
    assert np.all(out[:, 3] == 0) and np.all(np.isinf(out[:, 0]))  # too few steps yet
    b.step(100)
    out = b.converge(W, 0.05)
    for s, row in zip(solvers, out):
        raw = s._engine.read_forces()
        cd = s._coefficients(raw)["Cd"]
        assert len(cd) == 100
        rep = analyze_convergence(list(cd), window=W, tol=0.05)
        np.testing.assert_allclose(row[0], rep.ratio, rtol=1e-9, atol=1e-15)
        np.testing.assert_allclose(row[1], rep.mean_abs, rtol=1e-12)
        np.testing.assert_allclose(row[2], rep.std, rtol=1e-9, atol=1e-15)
        assert bool(row[3]) == rep.converged
        assert row[4] == 100 and row[5] == 0
        np.testing.assert_allclose(row[6], np.mean(cd[-W:]), rtol=1e-12)
    b.close()


@pytest.mark.gpu
def test_large_members_step_on_their_own_kernels():
    """A member of at least 2^20 cells steps in the batch through its own
    single-lattice kernels (its autotuned step kernel and its finalisation),
    as a branch beside the class kernels of the small members: its populations
    and forces equal those of the same lattice stepped alone through
    Solver3D.run, bit for bit, over calls of even and odd lengths."""
    from aero_b200 import Batch, Solver3D, Sphere
    makes = _cases()[:4]

    def big(precision):
        nz, ny, nx = 96, 96, 128  # 1,179,648 cells
        sph = Sphere(radius=8, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
        solid, phi = sph.mark_solid(nz, ny, nx), sph.sdf_field(nz, ny, nx)
        return Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, omega=1 / 0.6, u0=0.05, D=16.0, collision="mrt",
                        bouzidi=True, phi=phi, wall_bc="slip", outlet_bc="convective", sponge_thickness=8,
                        precision=precision)

    for precision, kernel in (("fp32", 0), ("fp16s", 4)):
        alone = big(precision)
        alone._engine.set_step_kernel(kernel)
        r = alone.run(25, check_every=26, verbose=False)
        b = Batch(max_members=8)
        mix = [m() for m in makes]
        s = big(precision)
        s._engine.set_step_kernel(kernel)
        for x in mix[:2] + [s] + mix[2:]:
            b.add(x)
        b.step(10)
        b.step(15)
        cd = s._coefficients(s._engine.read_forces())["Cd"]
        np.testing.assert_array_equal(cd, np.array(r["Cd_history"]))
        b.remove(s)
        np.testing.assert_array_equal(s.f, alone.f)
        b.close()


@pytest.mark.gpu
def test_large_aa_member_steps_in_the_batch_as_alone():
    """A lattice in the AA layout joins a batch when it has at least 2^20
    cells, and then steps on its own kernels as a branch of the batch step.
    Each batch call first collides the state the member's previous call
    stored and ends on a state-storing step, as a call of its own does, so
    populations and drag equal those of the same lattice stepped alone in
    the AA layout with calls of the same lengths (10, 15 and 1 steps), bit
    for bit.  A smaller AA lattice is refused."""
    from aero_b200 import Batch, Solver3D, Sphere
    from aero_b200._lib import AeroError
    makes = _cases()[:3]

    def big():
        nz, ny, nx = 96, 96, 128  # 1,179,648 cells
        sph = Sphere(radius=8, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
        solid, phi = sph.mark_solid(nz, ny, nx), sph.sdf_field(nz, ny, nx)
        return Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, omega=1 / 0.6, u0=0.05, D=16.0, collision="mrt",
                        bouzidi=True, phi=phi, wall_bc="slip", outlet_bc="convective", sponge_thickness=8,
                        precision="fp32", layout="aa")

    calls = (10, 15, 1)
    alone = big()
    for n in calls:
        r = alone.run(n, check_every=n + 1, verbose=False)
    b = Batch(max_members=8)
    mix = [m() for m in makes]
    s = big()
    for x in mix[:1] + [s] + mix[1:]:
        b.add(x)
    for n in calls:
        b.step(n)
    cd = s._coefficients(s._engine.read_forces())["Cd"]
    np.testing.assert_array_equal(cd, np.array(r["Cd_history"]))
    b.remove(s)
    np.testing.assert_array_equal(s.f, alone.f)
    b.close()
    small = Solver3D(Nz=16, Ny=18, Nx=40, solid=np.zeros((16, 18, 40), bool), omega=1 / 0.6, u0=0.05, D=4.0,
                     layout="aa")
    b = Batch(max_members=2)
    with pytest.raises(AeroError):
        b.add(small)
    b.close()


def _inflow_cases():
    from aero_b200 import Cylinder, Solver, Solver3D, Sphere

    def c2d():
        cyl = Cylinder(radius=4, cx_frac=0.3, cy_frac=0.5)
        return Solver(Ny=30, Nx=80, solid=cyl.mark_solid(30, 80), omega=1 / 0.6, u0=0.05,
                      D=cyl.reference_length(), collision="bgk", synthetic_inflow=True,
                      synthetic_inflow_intensity=0.02, synthetic_inflow_seed=11, precision="fp32")

    def c3d(precision, **kw):
        sph = Sphere(radius=3, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
        nz, ny, nx = 12, 14, 32
        return Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=sph.mark_solid(nz, ny, nx), omega=1 / 0.7, u0=0.05,
                        D=sph.reference_length(), collision="mrt", wall_bc="slip", outlet_bc="convective",
                        precision=precision, **kw)

    return [c2d,
            lambda: c3d("fp32", sem_inlet=True, sem_Tu=0.05, sem_L_int=3.0, sem_N=40),
            lambda: c3d("fp16s", synthetic_inflow=True, synthetic_inflow_intensity=0.03, synthetic_inflow_seed=5)]


@pytest.mark.gpu
def test_inflow_field_members_step_in_the_batch():
    """Lattices with synthetic inflow (2D, 3D) or an SEM inlet join a batch:
    Batch.step uploads each one's fields ahead of every chunk of at most its
    ring's 64 steps, and the members match the same lattices run alone
    (Solver.run) to the batch tolerances over 150 steps, and are bit-identical
    alone in a batch and beside a plain member."""
    from aero_b200 import Batch
    makes = _inflow_cases()
    plain = _cases()[0]
    steps = 150
    ref = [_alone(m, steps) for m in makes]
    b = Batch(max_members=4)
    mix = [m() for m in makes] + [plain()]
    for s in mix:
        b.add(s)
    b.step(steps)
    for s, (f_ref, cd_ref) in zip(mix, ref):
        cd = s._coefficients(s._engine.read_forces())["Cd"]
        assert s.status() == 0
        _close(s, s.f, f_ref, cd, cd_ref)
    for m, s in zip(makes, mix):
        b1 = Batch(max_members=1)
        t = m()
        b1.add(t)
        b1.step(steps)
        np.testing.assert_array_equal(t._engine.get_state()[0], s._engine.get_state()[0])
        b1.remove(t)
        b1.close()
    b.close()


@pytest.mark.gpu
def test_batch_step_needs_the_inflow_fields():
    """aero_batch_step refuses (AERO_ERR_STATE) while a member's inflow
    fields for the call's steps are not on the device, and steps once they
    are."""
    from aero_b200 import Batch
    s = _inflow_cases()[0]()
    b = Batch(max_members=2)
    b.add(s)
    rc = b.lib.aero_batch_step(b.h, 5, b._stream())
    assert rc == -3, rc
    assert b"aero_set_inflow" in b.lib.aero_last_error()
    s._engine.set_inflow(s._inflow.fields(5), s.step_count)
    assert b.lib.aero_batch_step(b.h, 5, b._stream()) == 0
    b.close()


@pytest.mark.gpu
def test_recycling_members_step_in_the_batch():
    """Lattices with the 3D recycling inlet join a batch: each batch step
    launches their plane-mean pass before the class kernels (the per-cell
    classes in FP64 and FP32, the pair class in BF16), and they match the same
    lattices run alone to the batch tolerances, bit-identical alone in a
    batch and beside a plain member."""
    from aero_b200 import Batch, Solver3D, Sphere

    def rec(precision):
        sph = Sphere(radius=3, cx_frac=0.4, cy_frac=0.5, cz_frac=0.5)
        nz, ny, nx = 12, 14, 40
        return lambda: Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=sph.mark_solid(nz, ny, nx), omega=1 / 0.7, u0=0.05,
                                D=sph.reference_length(), collision="mrt", wall_bc="noslip",
                                streamwise_bc="recycling", precision=precision)

    makes = [rec("fp64"), rec("fp32"), rec("bf16s")]
    steps = 41
    ref = [_alone(m, steps) for m in makes]
    b = Batch(max_members=4)
    mix = [m() for m in makes] + [_cases()[0]()]
    for s in mix:
        b.add(s)
    b.step(20)
    b.step(steps - 20)
    for s, (f_ref, cd_ref) in zip(mix, ref):
        cd = s._coefficients(s._engine.read_forces())["Cd"]
        assert s.status() == 0
        _close(s, s.f, f_ref, cd, cd_ref)
    for m, s in zip(makes, mix):
        b1 = Batch(max_members=1)
        t = m()
        b1.add(t)
        b1.step(steps)
        np.testing.assert_array_equal(t._engine.get_state()[0], s._engine.get_state()[0])
        b1.remove(t)
        b1.close()
    b.close()
