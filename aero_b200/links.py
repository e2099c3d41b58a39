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


def _shift_clipped(a: np.ndarray, axis: int, step: int) -> np.ndarray:
    """b[..., k, ...] = a[..., clip(k + step), ...] along one axis (step in -1, 0, 1)."""
    if step == 0:
        return a
    n = a.shape[axis]
    if step > 0:
        idx = np.concatenate([np.arange(1, n), [n - 1]])
    else:
        idx = np.concatenate([[0], np.arange(0, n - 1)])
    return np.take(a, idx, axis=axis)


def build_surface_links(solid: np.ndarray, phi: Optional[np.ndarray] = None
                        ) -> Tuple[np.ndarray, np.ndarray]:
    solid = np.asarray(solid, dtype=bool)
    dims = solid.ndim
    e = E if dims == 2 else E3
    fluid = ~solid
    parts = []
    for i in range(1, len(e)):
        nb = solid
        # array axes are ([z,] y, x); e is (ex, ey[, ez])
        for comp in range(dims):
            nb = _shift_clipped(nb, dims - 1 - comp, int(e[i, comp]))
        idx = np.nonzero(fluid & nb)
        if idx[0].size:
            parts.append(np.stack([np.full(idx[0].size, i, dtype=np.int64), *idx], axis=1))
    if not parts:
        return np.empty((0, dims + 1), dtype=np.int32), np.empty(0, dtype=np.float32)
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
