"""Host-side lattice tables and the equilibrium, for set-up and diagnostics.

Direction order, weights and opposites are the reference's
(aero/lbm/d2q9.py:18-38, aero/lbm/d3q19.py:37-73): population arrays keep the
reference layout (Q, [Nz,] Ny, Nx), so states and checkpoints interchange.
"""

from __future__ import annotations

import numpy as np

Q = 9
E = np.array([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, 1], [-1, -1], [1, -1]],
             dtype=np.int8)
W = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4, dtype=np.float64)
OPP = np.array([0, 3, 4, 1, 2, 7, 8, 5, 6], dtype=np.int8)

Q3 = 19
E3 = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
               [1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1],
               [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]], dtype=np.int8)
W3 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float64)
OPP3 = np.array([0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15], dtype=np.int8)
Y_MIR3 = np.array([0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 11, 12, 13, 14, 16, 15, 18, 17], dtype=np.int8)

# Reduced scalar lattices (D2Q5 cs^2 = 1/3, D3Q7 cs^2 = 1/4).
W_Q5 = np.array([1 / 3] + [1 / 6] * 4)
W_Q7 = np.array([1 / 4] + [1 / 8] * 6)


def tables(dims: int):
    return (E, W, OPP) if dims == 2 else (E3, W3, OPP3)


def scalar_weights(dims: int, reduced: bool) -> np.ndarray:
    if not reduced:
        return tables(dims)[1]
    return W_Q5 if dims == 2 else W_Q7


def feq(dims: int, rho, ux, uy, uz=None, xp=np):
    """w_i rho (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u.u) for every direction.

    ``xp`` may be numpy or torch (arrays on the GPU for large set-ups).
    """
    e, w, _ = tables(dims)
    uz = 0.0 * ux if uz is None else uz
    usq = ux * ux + uy * uy + uz * uz
    out = []
    for i in range(len(w)):
        eu = float(e[i, 0]) * ux + float(e[i, 1]) * uy + (float(e[i, 2]) * uz if dims == 3 else 0.0)
        out.append(float(w[i]) * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * usq))
    return xp.stack(out)


def macroscopic(f: np.ndarray, dims: int):
    """rho and velocity of populations f (Q, ...); u = 0 where rho <= 0."""
    e, _, _ = tables(dims)
    rho = f.sum(axis=0)
    inv = np.where(rho > 0, 1.0 / np.where(rho > 0, rho, 1.0), 0.0)
    u = [inv * np.tensordot(e[:, a].astype(np.float64), f, axes=(0, 0)) for a in range(dims)]
    return (rho, *u)
