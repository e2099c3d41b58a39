"""CPU tests of the host side: geometry and link tables bit-exact against the
reference fixtures, the C ABI library (loads, exports every declared symbol,
validates options without touching a GPU), and the MRT operator."""

import ctypes
import hashlib
import json
import re

import numpy as np
import pytest

from aero_b200 import Box, Cylinder, Rectangle, Sphere, build_surface_links
from tests.golden_cases import CASES, GOLDEN, load_case


def _digest(a):
    a = np.ascontiguousarray(a)
    h = hashlib.sha256()
    h.update(str(a.dtype).encode())
    h.update(str(a.shape).encode())
    h.update(a.tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def geom():
    return np.load(GOLDEN / "geometry.npz")


def test_channel_cylinder_mask_links_q_bit_exact(geom):
    cyl = Cylinder(radius=20, cx_frac=0.25, cy_frac=0.5)
    solid = cyl.mark_solid(200, 400)
    assert np.array_equal(np.packbits(solid), geom["c1_solid"])
    phi = cyl.sdf_field(200, 400)
    assert _digest(phi) == str(geom["c1_phi_digest"])
    links, q = build_surface_links(solid, phi)
    assert np.array_equal(links, geom["c1_links"]) and links.dtype == np.int32
    assert np.array_equal(q, geom["c1_q"]) and q.dtype == np.float32


def test_box_channel_digests(geom):
    box = Box(width=24, height=24, depth=128, cx_frac=76 / 256, cy_frac=12 / 128, cz_frac=0.5)
    solid = box.mark_solid(128, 128, 256)
    assert _digest(solid) == str(geom["c3_solid_digest"])
    links, q = build_surface_links(solid, None)
    assert len(links) == int(geom["c3_n_links"])
    assert _digest(links) == str(geom["c3_links_digest"])
    assert _digest(q) == str(geom["c3_q_digest"])


def test_sphere_512_digests(geom):
    sph = Sphere(radius=16, cx_frac=96 / 512, cy_frac=0.5, cz_frac=0.5)
    solid = sph.mark_solid(256, 256, 512)
    assert _digest(solid) == str(geom["c2_solid_digest"])
    phi = sph.sdf_field(256, 256, 512)
    links, q = build_surface_links(solid, phi)
    assert _digest(links) == str(geom["c2_links_digest"])
    assert _digest(q) == str(geom["c2_q_digest"])


def test_small_shapes_bit_exact(geom):
    meta = json.loads(str(geom["small_meta"]))
    k2 = k3 = 0
    for m in meta:
        kind, p = m["kind"], m["params"]
        if kind in ("cyl", "rect"):
            g = Cylinder(*p) if kind == "cyl" else Rectangle(*p)
            s, phi = g.mark_solid(m["ny"], m["nx"]), g.sdf_field(m["ny"], m["nx"])
            key = f"s2_{k2}"
            k2 += 1
        else:
            g = Sphere(*p) if kind == "sph" else Box(*p)
            s = g.mark_solid(m["nz"], m["ny"], m["nx"])
            phi = g.sdf_field(m["nz"], m["ny"], m["nx"])
            key = f"s3_{k3}"
            k3 += 1
        assert np.array_equal(np.packbits(s), geom[f"{key}_solid"]), key
        links, q = build_surface_links(s, phi)
        assert np.array_equal(links, geom[f"{key}_links"]), key
        assert np.array_equal(q, geom[f"{key}_q"]), key


@pytest.mark.parametrize("name", CASES)
def test_case_links_bit_exact(name):
    c = load_case(name)
    links, q = build_surface_links(c["solid"], c["phi"] if c["kwargs"].get("bouzidi") else None)
    assert np.array_equal(links, c["links"]) and np.array_equal(q, c["q_vals"])


def test_empty_domain_has_no_links():
    links, q = build_surface_links(np.zeros((8, 12), bool))
    assert links.shape == (0, 3) and q.shape == (0,)
    links, q = build_surface_links(np.zeros((4, 8, 12), bool))
    assert links.shape == (0, 4)


# --------------------------------------------------------------------- C ABI
def _declared_symbols():
    hdr = (GOLDEN.parent.parent / "include" / "aero_b200.h").read_text()
    return sorted(set(re.findall(r"AERO_API\s+[^;(]*?\b(aero_\w+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    from aero_b200 import _lib
    lib = _lib.load()
    names = _declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert lib.aero_abi_version() == _lib.ABI_VERSION
    assert lib.aero_params_size() == ctypes.sizeof(_lib.AeroParams)


def _params(**kw):
    from aero_b200 import _lib
    p = _lib.AeroParams()
    p.abi_version = _lib.ABI_VERSION
    p.dims, p.nx, p.ny, p.nz = 2, 40, 20, 1
    p.omega, p.u0, p.rho0 = 1.6, 0.05, 1.0
    p.inlet_bc, p.outlet_bc, p.wall_bc = 1, 2, 2
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def test_create_validates_options_without_gpu():
    from aero_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.aero_create(ctypes.byref(_params(dims=4)), ctypes.byref(h)) == -1
    assert b"dims" in lib.aero_last_error()
    assert lib.aero_create(ctypes.byref(_params(nz=3)), ctypes.byref(h)) == -1
    assert lib.aero_create(ctypes.byref(_params(abi_version=99)), ctypes.byref(h)) == -1
    assert lib.aero_create(ctypes.byref(_params(omega=-1.0)), ctypes.byref(h)) == -1
    assert lib.aero_create(ctypes.byref(_params(dims=3, nz=4, inlet_bc=2)), ctypes.byref(h)) == -4
    assert lib.aero_create(ctypes.byref(_params()), ctypes.byref(h)) == 0
    solid = np.zeros((20, 40), np.uint8)
    solid[8:12, 10:14] = 1
    links, q = build_surface_links(solid.astype(bool))
    links = np.ascontiguousarray(links)
    assert lib.aero_step(h, 1, None) == -3  # no workspace / state yet
    rc = lib.aero_set_geometry(h, solid.ctypes.data, links.ctypes.data, q.ctypes.data, len(links), None)
    assert rc == 0
    nbytes = ctypes.c_uint64()
    assert lib.aero_workspace_size(h, ctypes.byref(nbytes)) == 0
    assert nbytes.value > 2 * 9 * 4 * 20 * 40
    bad = links.copy()
    bad[0, 1] = 99
    h2 = ctypes.c_void_p()
    assert lib.aero_create(ctypes.byref(_params()), ctypes.byref(h2)) == 0
    assert lib.aero_set_geometry(h2, solid.ctypes.data, bad.ctypes.data, q.ctypes.data, len(bad), None) == -1
    lib.aero_destroy(h2)
    lib.aero_destroy(h)


@pytest.mark.parametrize("dims", [2, 3])
def test_mrt_operator_matches_reference_basis(dims):
    """A = Minv (I - S) M, B = Minv S M with the reference matrices (tables.npz)."""
    from aero_b200 import _lib
    t = np.load(GOLDEN / "tables.npz")
    M = t["M9"] if dims == 2 else t["M19"]
    Minv = t["M9_inv"] if dims == 2 else t["M19_inv"]
    Q = M.shape[0]
    lib = _lib.load()
    for k, om in enumerate(t["omegas"]):
        s = t["s9"][k] if dims == 2 else t["s19"][k]
        A = np.empty((Q, Q))
        B = np.empty((Q, Q))
        assert lib.aero_mrt_operator(dims, float(om), A.ctypes.data, B.ctypes.data) == 0
        A_ref = Minv @ np.diag(1 - s) @ M
        B_ref = Minv @ np.diag(s) @ M
        np.testing.assert_allclose(A, A_ref, rtol=0, atol=1e-13)
        np.testing.assert_allclose(B, B_ref, rtol=0, atol=1e-13)


def test_corrupt_checkpoint_is_rejected_before_gpu_work(tmp_path):
    """A truncated or incomplete checkpoint raises ValueError when it is
    opened, before any solver (or device memory) is created."""
    from aero_b200.solver import Solver
    from aero_b200.solver3d import Solver3D
    good = tmp_path / "ok.npz"
    np.savez(good, f=np.zeros((9, 4, 6)), f_outlet_prev=np.zeros((9, 4)), step_count=np.array(3),
             solid=np.zeros((4, 6), bool), params_json=np.array('{"omega": 1.0}'))
    raw = good.read_bytes()
    trunc = tmp_path / "trunc.npz"
    trunc.write_bytes(raw[: len(raw) // 2])
    for cls in (Solver, Solver3D):
        with pytest.raises(ValueError, match="corrupt or unreadable checkpoint"):
            cls.from_checkpoint(str(trunc))
    nokeys = tmp_path / "nokeys.npz"
    np.savez(nokeys, f=np.zeros(3))
    with pytest.raises(ValueError, match="no 'params_json' entry"):
        Solver.from_checkpoint(str(nokeys))
    badjson = tmp_path / "badjson.npz"
    np.savez(badjson, solid=np.zeros((4, 6), bool), params_json=np.array("{not json"))
    with pytest.raises(ValueError, match="unreadable params_json"):
        Solver.from_checkpoint(str(badjson))


def test_layout_option():
    """layout is 'ab' (two buffers), 'aa' (one buffer in place) or 'auto'
    (chosen by the memory the lattice needs); anything else is refused before
    any device work, and the C ABI takes the layout field of AeroParams."""
    from aero_b200 import _lib
    from aero_b200._base import LAYOUTS, _check_layout
    from aero_b200.solver import Solver
    solid = np.zeros((8, 16), bool)
    for name in ("ab", "aa", "auto"):
        _check_layout(name)
    assert LAYOUTS == {"ab": 0, "aa": 1}
    with pytest.raises(ValueError, match="Unknown layout"):
        Solver(Ny=8, Nx=16, solid=solid, omega=1.0, u0=0.05, D=4.0, layout="soa")
    assert "layout" in dict(_lib.AeroParams._fields_)


def test_batch_step_uploads_inflow_fields_in_ring_chunks():
    """Batch.step (host logic, no GPU): with a member whose inflow ring holds
    64 steps, 150 steps go to aero_batch_step as 64 + 64 + 22, each chunk's
    fields uploaded first for that member (starting at its step count) and
    none for the plain member; without inflow members one call takes all
    steps."""
    import contextlib
    import types

    from aero_b200.batch import Batch

    calls = []

    class Lib:
        def aero_batch_step(self, h, n, stream):
            calls.append(("step", n))
            return 0

    class Eng:
        def __init__(self, name):
            self.name = name

        def set_inflow(self, fields, first):
            calls.append(("inflow", self.name, len(fields), first))

    class Gen:
        def fields(self, k):
            return np.zeros((k, 2, 4))

    def member(name, inflow):
        m = types.SimpleNamespace(step_count=10, _engine=Eng(name), _flush_host_state=lambda: None,
                                  _params=types.SimpleNamespace(inflow_ring=64))
        m._inflow = Gen() if inflow else None
        return m

    fake_torch = types.SimpleNamespace(cuda=types.SimpleNamespace(device=lambda d: contextlib.nullcontext()))
    b = Batch.__new__(Batch)
    b.torch, b.lib, b.h, b.device = fake_torch, Lib(), None, None
    b._stream = lambda: 0
    a, p = member("a", True), member("p", False)
    b.members = [a, p]
    b.step(150)
    assert calls == [("inflow", "a", 64, 10), ("step", 64), ("inflow", "a", 64, 74), ("step", 64),
                     ("inflow", "a", 22, 138), ("step", 22)]
    assert a.step_count == p.step_count == 160
    calls.clear()
    b.members = [p]
    b.step(150)
    assert calls == [("step", 150)] and p.step_count == 310
    b.members = []  # nothing for __del__ to release
