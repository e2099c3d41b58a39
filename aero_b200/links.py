"""Surface link lists for obstacle bounce-back.

Restates build_surface_links / build_surface_links_3d
(aero/lbm/boundary.py:232-280, aero/lbm/boundary3d.py:279-329) with whole-
array operations: a link (i, [z,] y, x) joins a fluid cell to the solid cell
in direction e_i, the neighbour index is CLIPPED to the grid (not wrapped),
the list is direction-major and C-ordered within a direction, and
q = clip(float32(phi[cell]), 1e-4, 1) when phi is given (else 0.5).
"""

from __future__ import annotations

from typing import Optional, Tuple

import numpy as np

from .lattice import E, E3


def build_surface_links(solid: np.ndarray, phi: Optional[np.ndarray] = None
                        ) -> Tuple[np.ndarray, np.ndarray]:
    """Links are only possible in the solid's bounding box grown by one cell,
    so the search runs on that box: padded by one more cell on every side,
    with the edge value repeated where the box meets the grid edge (the
    reference's clipped neighbour) and fluid elsewhere (no solid lies outside
    the box).  Within one direction the C order of the box's cells is the C
    order of the grid's, so the list is the reference's, entry for entry."""
    solid = np.asarray(solid, dtype=bool)
    dims = solid.ndim
    e = E if dims == 2 else E3
    empty = (np.empty((0, dims + 1), dtype=np.int32), np.empty(0, dtype=np.float32))
    idx = np.nonzero(solid)
    if idx[0].size == 0:
        return empty
    lo = [max(int(a.min()) - 1, 0) for a in idx]
    hi = [min(int(a.max()) + 2, n) for a, n in zip(idx, solid.shape)]
    box = solid[tuple(slice(l, h) for l, h in zip(lo, hi))]
    # pad by one: repeat the edge at the grid boundary, fluid inside the grid
    pad = np.pad(box, 1, mode="constant", constant_values=False)
    for ax in range(dims):
        n = solid.shape[ax]
        if lo[ax] == 0:
            src = [slice(None)] * dims
            dst = [slice(None)] * dims
            src[ax], dst[ax] = slice(1, 2), slice(0, 1)
            pad[tuple(dst)] = pad[tuple(src)]
        if hi[ax] == n:
            src = [slice(None)] * dims
            dst = [slice(None)] * dims
            src[ax], dst[ax] = slice(-2, -1), slice(-1, None)
            pad[tuple(dst)] = pad[tuple(src)]
    fluid = ~box
    shape = box.shape
    parts = []
    for i in range(1, len(e)):
        # array axes are ([z,] y, x); e is (ex, ey[, ez])
        sl = tuple(slice(1 + int(e[i, dims - 1 - ax]), 1 + int(e[i, dims - 1 - ax]) + shape[ax])
                   for ax in range(dims))
        hit = np.nonzero(fluid & pad[sl])
        if hit[0].size:
            parts.append(np.stack([np.full(hit[0].size, i, dtype=np.int64)] +
                                  [h + l for h, l in zip(hit, lo)], axis=1))
    if not parts:
        return empty
    links = np.concatenate(parts).astype(np.int32)
    if phi is not None:
        cells = tuple(links[:, 1 + a] for a in range(dims))
        q = np.clip(np.asarray(phi)[cells].astype(np.float32), 1e-4, 1.0)
    else:
        q = np.full(len(links), 0.5, dtype=np.float32)
    return links, q


def build_surface_links_3d(solid: np.ndarray, phi: Optional[np.ndarray] = None
                           ) -> Tuple[np.ndarray, np.ndarray]:
    return build_surface_links(solid, phi)


def build_surface_links_device(solid, phi=None, stream=None, capacity: int = 1 << 16):
    """The same list built on the GPU (aero_surface_links_device in
    libaero_b200.so): solid is a ([nz,] ny, nx) torch CUDA tensor (bool or
    uint8) and phi an optional float64 tensor of the same shape; returns
    (links int32 (n, dims+1), q float32 (n,)) as CUDA tensors, equal entry for
    entry to build_surface_links(solid, phi).  `capacity` is the first guess
    of the list length; a longer list costs one more counting pass."""
    import ctypes

    import torch

    from . import _lib
    from ._lib import AeroError, check

    if not isinstance(solid, torch.Tensor) or solid.device.type != "cuda":
        raise ValueError("build_surface_links_device takes a CUDA tensor; use build_surface_links for host arrays")
    dims = solid.dim()
    if dims not in (2, 3):
        raise ValueError(f"solid must be 2D or 3D, got shape {tuple(solid.shape)}")
    dev = solid.device
    s = solid.to(torch.uint8).contiguous()
    p = None
    if phi is not None:
        if tuple(phi.shape) != tuple(solid.shape):
            raise ValueError("phi must have the shape of solid")
        p = phi.to(device=dev, dtype=torch.float64).contiguous()
    nz, ny, nx = (1,) + tuple(s.shape) if dims == 2 else tuple(s.shape)
    lib = _lib.load()
    nbytes = ctypes.c_uint64()
    check("aero_surface_links_scratch_size",
          lib.aero_surface_links_scratch_size(dims, nx, ny, nz, ctypes.byref(nbytes)))
    with torch.cuda.device(dev):
        st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        scratch = torch.empty((int(nbytes.value) + 7) // 8, dtype=torch.int64, device=dev)
        n = ctypes.c_int64()
        cap = max(int(capacity), 1)
        for _ in range(2):
            links = torch.empty((cap, dims + 1), dtype=torch.int32, device=dev)
            q = torch.empty(cap, dtype=torch.float32, device=dev)
            rc = lib.aero_surface_links_device(
                dims, nx, ny, nz, s.data_ptr(), None if p is None else p.data_ptr(), scratch.data_ptr(),
                nbytes.value, links.data_ptr(), q.data_ptr(), cap, ctypes.byref(n), st)
            if rc == _lib.ERRORS_BY_NAME["AERO_ERR_CAPACITY"] and n.value > cap:
                cap = int(n.value)
                continue
            check("aero_surface_links_device", rc)
            if stream is not None:
                # the kernels ran on a stream the allocator does not order with
                # the current one: keep the inputs and scratch alive until they end
                torch.cuda.ExternalStream(st).synchronize()
            return links[: n.value], q[: n.value]
    raise AeroError("aero_surface_links_device", -5, "link count changed between passes")
