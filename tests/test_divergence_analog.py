"""The sphere benchmark configuration diverges in the reference algorithm.

tau 0.5048 (nu 0.0016) with D3Q19 MRT (rank-16 basis, pseudo-inverse,
mrt3d.py:46-135), Bouzidi links, slip walls, convective outlet and a sponge
(solver3d.py:325-541) loses positivity after about a hundred steps.  A
64x32x32 analogue (sphere r6) shows it in a second: the FP64 oracle, which
matches the reference's own step to 1e-11 on the golden cases, first has a
non-finite or non-positive density at step 98.  The GPU test checks that the
engine's device-side divergence flag names the same step.
"""

import numpy as np
import pytest

from oracle.oracle import OracleSolver

NZ, NY, NX = 32, 32, 64
KW = dict(collision="mrt", les=True, les_cs=0.1, bouzidi=True, wall_bc="slip", inlet_bc="velocity",
          outlet_bc="convective", streamwise_bc="open", sponge_thickness=4, sponge_strength=0.1)
OMEGA = 1.0 / (3.0 * 0.0016 + 0.5)


def _geometry():
    from aero_b200 import Sphere
    sph = Sphere(radius=6, cx_frac=12 / 64, cy_frac=0.5, cz_frac=0.5)
    return sph.mark_solid(NZ, NY, NX), sph.sdf_field(NZ, NY, NX), sph.reference_length()


def _oracle_first_bad(max_steps=200):
    solid, phi, D = _geometry()
    o = OracleSolver(solid=solid, omega=OMEGA, u0=0.05, D=D, phi=phi, **KW)
    for k in range(1, max_steps + 1):
        o.step()
        rho = o.f.sum(axis=0)
        if not np.isfinite(rho).all() or (rho <= 0).any():
            return k
    return None


def test_oracle_diverges_on_sphere_analogue():
    assert _oracle_first_bad() == 98


@pytest.mark.gpu
def test_engine_flags_the_same_first_bad_step():
    from aero_b200 import Solver3D
    solid, phi, D = _geometry()
    s = Solver3D(Nz=NZ, Ny=NY, Nx=NX, solid=solid, omega=OMEGA, u0=0.05, D=D, phi=phi,
                 precision="fp64", **KW)
    s._advance(120)
    assert s._engine.first_bad_step() == 98
    assert s._engine.status() & 1
