"""CPU check of the engine's collision arithmetic.

aero_collide_host runs the kernels' collide() (the same device source,
compiled for the host, FP64) on random near-equilibrium states; the result
must match the FP64 oracle's restatement of the reference collision
(kernels.py:42-92, kernels_trt.py:125-174, kernels_mrt.py:190-241,
kernels3d_mrt.py:24-82) to 1e-13.  This covers the pair-form BGK/TRT and the
symmetry-adapted D3Q19 MRT, solid cells included.
"""

import ctypes

import numpy as np
import pytest

from oracle.oracle import OracleSolver


def _params(dims, collision, omega, lam=0.25):
    from aero_b200 import _lib
    p = _lib.AeroParams()
    p.abi_version = _lib.ABI_VERSION
    p.dims = dims
    p.nx, p.ny, p.nz = (8, 6, 1) if dims == 2 else (6, 5, 4)
    p.collision = _lib.COLLISION[collision]
    p.omega, p.u0, p.rho0, p.trt_lambda = omega, 0.05, 1.0, lam
    return p


@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("collision", ["bgk", "trt", "mrt"])
@pytest.mark.parametrize("omega", [1 / 0.5048, 1 / 0.56, 1.0, 1 / 0.8])
def test_collide_matches_oracle(dims, collision, omega):
    from aero_b200 import _lib
    lib = _lib.load()
    shape = (6, 8) if dims == 2 else (4, 5, 6)
    rng = np.random.default_rng(5)
    solid = rng.random(shape) < 0.15
    o = OracleSolver(solid=solid, omega=omega, u0=0.05, D=4.0, collision=collision,
                     trt_lambda=3 / 16)
    rho = 1.0 + 0.02 * rng.uniform(-1, 1, shape)
    u = [0.08 * rng.uniform(-1, 1, shape) for _ in range(dims)]
    f = o.feq(rho, *u) * (1.0 + 0.01 * rng.uniform(-1, 1, (o.Q,) + shape))
    o.f = np.ascontiguousarray(f)
    ref = o.collide_only()
    n = solid.size
    out = np.empty_like(f)
    sol = np.ascontiguousarray(solid.astype(np.uint8))
    p = _params(dims, collision, omega, lam=3 / 16)
    p.nx, p.ny, p.nz = (shape[1], shape[0], 1) if dims == 2 else (shape[2], shape[1], shape[0])
    rc = lib.aero_collide_host(ctypes.byref(p), np.ascontiguousarray(f).ctypes.data, out.ctypes.data,
                               sol.ctypes.data, n)
    assert rc == 0, lib.aero_last_error()
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-13)


def test_mrt3_adapted_blocks_accepted_over_omega_range():
    """aero_create derives and checks the symmetry-adapted D3Q19 MRT blocks."""
    from aero_b200 import _lib
    lib = _lib.load()
    for om in np.linspace(0.2, 1.98, 25):
        h = ctypes.c_void_p()
        assert lib.aero_create(ctypes.byref(_params(3, "mrt", float(om))), ctypes.byref(h)) == 0, \
            lib.aero_last_error()
        lib.aero_destroy(h)
