"""The surface link list built on the device (aero_surface_links_device)
against the reference's lists: the geometry fixtures generated from
build_surface_links / build_surface_links_3d (boundary.py:232-280,
boundary3d.py:279-329) and, for random and edge-case solids, the host
builder that those fixtures pin.  Entry for entry, bit for bit."""

import ctypes
import hashlib
import json

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


# ------------------------------------------------------------------ host side
def test_scratch_size_and_argument_checks_without_gpu():
    from aero_b200 import _lib
    lib = _lib.load()
    b = ctypes.c_uint64()
    assert lib.aero_surface_links_scratch_size(2, 40, 20, 1, ctypes.byref(b)) == 0
    # 800 cells: the box (32 bytes), one unit per direction, 8 CTAs of one
    # unit, plus the total
    assert b.value == 32 + 8 * (8 + 1)
    assert lib.aero_surface_links_scratch_size(3, 512, 256, 256, ctypes.byref(b)) == 0
    assert b.value % 8 == 0 and b.value <= 32 + 8 * (148 * 16 + 1)
    assert lib.aero_surface_links_scratch_size(2, 40, 20, 3, ctypes.byref(b)) == -1
    assert lib.aero_surface_links_scratch_size(4, 40, 20, 1, ctypes.byref(b)) == -1
    assert lib.aero_surface_links_scratch_size(3, 0, 20, 4, ctypes.byref(b)) == -1
    assert lib.aero_surface_links_scratch_size(3, 1 << 12, 1 << 12, 1 << 8, ctypes.byref(b)) == -4
    n = ctypes.c_int64()
    # NULL inputs and short scratch are refused before any device work
    assert lib.aero_surface_links_device(2, 40, 20, 1, None, None, 8, 72, None, None, 0,
                                         ctypes.byref(n), None) == -1
    assert lib.aero_surface_links_device(2, 40, 20, 1, 8, None, 8, 64, None, None, 0,
                                         ctypes.byref(n), None) == -1
    assert b"scratch" in lib.aero_last_error()
    assert lib.aero_surface_links_device(2, 40, 20, 1, 8, None, 12, 104, None, None, 0,
                                         ctypes.byref(n), None) == -1
    assert b"aligned" in lib.aero_last_error()


def test_device_builder_refuses_host_arrays():
    from aero_b200 import build_surface_links_device
    with pytest.raises(ValueError, match="CUDA tensor"):
        build_surface_links_device(np.zeros((8, 8), bool))
    torch = pytest.importorskip("torch")
    with pytest.raises(ValueError, match="CUDA tensor"):
        build_surface_links_device(torch.zeros((8, 8), dtype=torch.bool))


# ------------------------------------------------------------------ device
def _dev(solid, phi=None, **kw):
    import torch
    from aero_b200 import build_surface_links_device
    s = torch.from_numpy(np.ascontiguousarray(solid)).cuda()
    p = None if phi is None else torch.from_numpy(np.ascontiguousarray(phi, dtype=np.float64)).cuda()
    links, q = build_surface_links_device(s, p, **kw)
    return links.cpu().numpy(), q.cpu().numpy()


def _same(solid, phi=None, **kw):
    links, q = _dev(solid, phi, **kw)
    ref_links, ref_q = build_surface_links(solid, phi)
    assert links.dtype == np.int32 and q.dtype == np.float32
    assert links.shape == ref_links.shape
    assert np.array_equal(links, ref_links)
    assert np.array_equal(q.view(np.uint32), ref_q.view(np.uint32))
    return len(links)


@pytest.fixture(scope="module")
def geom():
    return np.load(GOLDEN / "geometry.npz")


@pytest.mark.gpu
def test_cylinder_channel_against_reference_fixture(geom):
    cyl = Cylinder(radius=20, cx_frac=0.25, cy_frac=0.5)
    links, q = _dev(cyl.mark_solid(200, 400), cyl.sdf_field(200, 400))
    assert np.array_equal(links, geom["c1_links"])
    assert np.array_equal(q, geom["c1_q"])


@pytest.mark.gpu
def test_sphere_512_against_reference_digests(geom):
    """The full-size sphere workload, 512x256x256: 33.5M cells."""
    sph = Sphere(radius=16, cx_frac=96 / 512, cy_frac=0.5, cz_frac=0.5)
    links, q = _dev(sph.mark_solid(256, 256, 512), sph.sdf_field(256, 256, 512))
    assert len(links) == int(geom["c2_n_links"])
    assert _digest(links) == str(geom["c2_links_digest"])
    assert _digest(q) == str(geom["c2_q_digest"])


@pytest.mark.gpu
def test_box_channel_against_reference_digests(geom):
    box = Box(width=24, height=24, depth=128, cx_frac=76 / 256, cy_frac=12 / 128, cz_frac=0.5)
    links, q = _dev(box.mark_solid(128, 128, 256))
    assert len(links) == int(geom["c3_n_links"])
    assert _digest(links) == str(geom["c3_links_digest"])
    assert _digest(q) == str(geom["c3_q_digest"])


@pytest.mark.gpu
def test_small_shapes_against_reference_fixtures(geom):
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
        links, q = _dev(s, phi)
        assert np.array_equal(links, geom[f"{key}_links"]), key
        assert np.array_equal(q, geom[f"{key}_q"]), key


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_case_fixtures(name):
    c = load_case(name)
    links, q = _dev(c["solid"], c["phi"] if c["kwargs"].get("bouzidi") else None)
    assert np.array_equal(links, c["links"]) and np.array_equal(q, c["q_vals"])


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(37, 53), (3, 1031), (1, 1), (5, 17, 29), (64, 96, 200), (2, 1, 3000)])
@pytest.mark.parametrize("density", [0.02, 0.4])
def test_random_solids_equal_the_host_builder(shape, density):
    """Scattered solids with links at every grid edge (clipped neighbours),
    ragged sizes (not multiples of the 1024-cell unit), many CTA groups."""
    rng = np.random.default_rng(hash((shape, density)) % (1 << 32))
    solid = rng.random(shape) < density
    phi = rng.normal(0.5, 0.7, shape)  # values below 1e-4 and above 1
    _same(solid, phi)
    _same(solid, None)


@pytest.mark.gpu
def test_edge_cases():
    # no solid, all solid: no links
    for shape in [(8, 12), (4, 8, 12)]:
        assert _same(np.zeros(shape, bool)) == 0
        assert _same(np.ones(shape, bool)) == 0
    # one fluid cell inside solid: a link in every direction
    s = np.ones((5, 5, 5), bool)
    s[2, 2, 2] = False
    assert _same(s) == 18
    # solid slabs on the grid faces: clipped neighbours of edge cells
    s = np.zeros((6, 7, 9), bool)
    s[:, :, 0] = s[:, 0, :] = s[-1, :, :] = True
    _same(s, np.linspace(-1, 2, s.size).reshape(s.shape))
    # non-finite phi: NaN stays NaN, +-inf clips, as np.clip
    s = np.zeros((6, 10), bool)
    s[2:4, 3:6] = True
    phi = np.full(s.shape, np.nan)
    phi[::2] = np.inf
    phi[1::4] = -np.inf
    links, q = _dev(s, phi)
    ref_links, ref_q = build_surface_links(s, phi)
    assert np.array_equal(links, ref_links)
    assert np.array_equal(q, ref_q, equal_nan=True)


@pytest.mark.gpu
def test_capacity_guess_too_small_takes_a_second_pass():
    sph = Sphere(radius=6, cx_frac=0.5, cy_frac=0.5, cz_frac=0.5)
    s, phi = sph.mark_solid(24, 24, 24), sph.sdf_field(24, 24, 24)
    n = _same(s, phi, capacity=1)
    assert n > 1


@pytest.mark.gpu
def test_capacity_refusal_reports_the_count():
    import torch
    from aero_b200 import _lib
    lib = _lib.load()
    s = torch.zeros((16, 16), dtype=torch.uint8, device="cuda")
    s[5:9, 5:9] = 1
    b = ctypes.c_uint64()
    assert lib.aero_surface_links_scratch_size(2, 16, 16, 1, ctypes.byref(b)) == 0
    scratch = torch.empty(b.value // 8, dtype=torch.int64, device="cuda")
    n = ctypes.c_int64()
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.aero_surface_links_device(2, 16, 16, 1, s.data_ptr(), None, scratch.data_ptr(), b.value,
                                       None, None, 0, ctypes.byref(n), st)
    assert rc == -5
    ref, _ = build_surface_links(s.cpu().numpy().astype(bool))
    assert n.value == len(ref)
