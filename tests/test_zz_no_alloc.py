"""GPU test of aero_link_forces_static, the force entry point that allocates
nothing (its per-link scratch is a fixed array inside the library).

It is meant for callers that cannot call cudaMalloc -- loops with device
memory fixed in advance, host frameworks that only lend out their own
buffers.  The test gives it the pre-stream and
post-boundary populations of two consecutive engine steps, calls it twice in
a row through the C ABI, and checks each result against the forces the
engine's own per-step path (aero_step + aero_read_forces) reported for the
same step, to 1e-10 of the largest value (the FP64 tolerance of the parity
tests).  This file is named so that pytest collects it last.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_forces_match_engine_two_calls_in_a_row():
    import torch

    from aero_b200 import Solver3D, Sphere, _lib

    lib = _lib.load()
    nz, ny, nx = 16, 20, 40
    sph = Sphere(radius=4, cx_frac=0.3, cy_frac=0.5, cz_frac=0.5)
    solid, phi = sph.mark_solid(nz, ny, nx), sph.sdf_field(nz, ny, nx)
    s = Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, omega=1 / 0.7, u0=0.05, D=sph.reference_length(),
                 collision="mrt", bouzidi=True, phi=phi, wall_bc="slip", outlet_bc="convective",
                 precision="fp64")
    for _ in range(5):
        s._step()
    dev = s._engine.device
    links = torch.from_numpy(np.ascontiguousarray(s.surface_links, dtype=np.int32)).to(dev)
    center = np.ascontiguousarray(s._ref_center, dtype=np.float64)
    solid_u8 = np.ascontiguousarray(solid.astype(np.uint8))  # kept alive across the ctypes calls
    Q = 19
    for call in range(2):
        # post-collision (pre-stream) populations of the next step: the
        # engine's own collision applied to the current state, on the host
        f_state = s.f.copy()
        f_pre = np.empty_like(f_state)
        rc = lib.aero_collide_host(ctypes.byref(s._params), f_state.ctypes.data, f_pre.ctypes.data,
                                   solid_u8.ctypes.data, solid.size)
        assert rc == 0, lib.aero_last_error()
        raw = s._advance(1)[0]                      # engine forces of that step
        prof_engine = np.array([s._last_spanwise_profile[k] for k in ("fx", "fy", "fz")]).T
        f_post = s.f.copy()
        fp = torch.from_numpy(f_pre.reshape(Q, -1)).to(dev)
        fq = torch.from_numpy(f_post.reshape(Q, -1)).to(dev)
        out = torch.full((12,), float("nan"), dtype=torch.float64, device=dev)
        prof = torch.full((nz, 3), float("nan"), dtype=torch.float64, device=dev)
        with torch.cuda.device(dev):
            rc = lib.aero_link_forces_static(3, nx, ny, nz, fp.data_ptr(), fq.data_ptr(), links.data_ptr(),
                                             links.shape[0], center.ctypes.data, out.data_ptr(),
                                             prof.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
            torch.cuda.synchronize(dev)
        assert rc == 0, lib.aero_last_error()
        got = out.cpu().numpy()
        scale = np.abs(raw).max()
        np.testing.assert_allclose(got, raw, rtol=0, atol=1e-10 * scale, err_msg=f"call {call}")
        np.testing.assert_allclose(prof.cpu().numpy(), prof_engine, rtol=0, atol=1e-10 * scale)


def test_static_forces_match_engine_2d_two_calls_in_a_row():
    """The 2D path: link rows [i, y, x], the D2Q9 tables, z = 0 with nz = 1,
    and the profile binned by y over ny rows."""
    import torch

    from aero_b200 import Cylinder, Solver, _lib

    lib = _lib.load()
    ny, nx = 36, 90
    cyl = Cylinder(radius=6, cx_frac=0.3, cy_frac=0.5)
    solid, phi = cyl.mark_solid(ny, nx), cyl.sdf_field(ny, nx)
    s = Solver(Ny=ny, Nx=nx, solid=solid, omega=1 / 0.6, u0=0.05, D=cyl.reference_length(), collision="bgk",
               bouzidi=True, phi=phi, wall_bc="noslip", outlet_bc="zerogradient", precision="fp64")
    for _ in range(5):
        s._step()
    dev = s._engine.device
    links = torch.from_numpy(np.ascontiguousarray(s.surface_links, dtype=np.int32)).to(dev)
    assert links.shape[1] == 3
    center = np.ascontiguousarray(s._ref_center, dtype=np.float64)
    solid_u8 = np.ascontiguousarray(solid.astype(np.uint8))
    Q = 9
    for call in range(2):
        f_state = s.f.copy()
        f_pre = np.empty_like(f_state)
        rc = lib.aero_collide_host(ctypes.byref(s._params), f_state.ctypes.data, f_pre.ctypes.data,
                                   solid_u8.ctypes.data, solid.size)
        assert rc == 0, lib.aero_last_error()
        raw = s._advance(1)[0]
        prof_engine = np.array([s._last_force_profile["fx"], s._last_force_profile["fy"]]).T
        f_post = s.f.copy()
        fp = torch.from_numpy(f_pre.reshape(Q, -1)).to(dev)
        fq = torch.from_numpy(f_post.reshape(Q, -1)).to(dev)
        out = torch.full((12,), float("nan"), dtype=torch.float64, device=dev)
        prof = torch.full((ny, 3), float("nan"), dtype=torch.float64, device=dev)
        with torch.cuda.device(dev):
            rc = lib.aero_link_forces_static(2, nx, ny, 1, fp.data_ptr(), fq.data_ptr(), links.data_ptr(),
                                             links.shape[0], center.ctypes.data, out.data_ptr(),
                                             prof.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
            torch.cuda.synchronize(dev)
        assert rc == 0, lib.aero_last_error()
        got = out.cpu().numpy()
        scale = np.abs(raw).max()
        np.testing.assert_allclose(got, raw, rtol=0, atol=1e-10 * scale, err_msg=f"call {call}")
        pr = prof.cpu().numpy()
        np.testing.assert_allclose(pr[:, :2], prof_engine, rtol=0, atol=1e-10 * scale)
        assert np.all(pr[:, 2] == 0.0)


def test_static_forces_malformed_rows_give_nan():
    """A row with direction 0 or a cell outside the grid (both caught by the
    kernel's own range check before any access) turns every output NaN."""
    import torch

    from aero_b200 import _lib

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    nz, ny, nx = 4, 5, 6
    f = torch.ones((19, nz * ny * nx), dtype=torch.float64, device=dev)
    center = np.zeros(3)
    for bad in ([0, 1, 1, 1], [3, 1, 1, nx]):
        links = torch.tensor([[1, 1, 2, 2], bad], dtype=torch.int32, device=dev)
        out = torch.zeros(12, dtype=torch.float64, device=dev)
        prof = torch.zeros((nz, 3), dtype=torch.float64, device=dev)
        with torch.cuda.device(dev):
            rc = lib.aero_link_forces_static(3, nx, ny, nz, f.data_ptr(), f.data_ptr(), links.data_ptr(), 2,
                                             center.ctypes.data, out.data_ptr(), prof.data_ptr(),
                                             torch.cuda.current_stream(dev).cuda_stream)
            torch.cuda.synchronize(dev)
        assert rc == 0, lib.aero_last_error()
        assert torch.isnan(out).all() and torch.isnan(prof).all()


def test_static_forces_reject_oversized_link_lists():
    from aero_b200 import _lib
    lib = _lib.load()
    center = np.zeros(3)
    rc = lib.aero_link_forces_static(3, 8, 8, 8, 1, 1, 1, 40000, center.ctypes.data, 1, None, None)
    assert rc == -5
    assert b"capacity" in lib.aero_last_error()
