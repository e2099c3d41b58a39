"""Kernels compiled for one feature word: a lattice whose features are exactly
the thermal channel's (D3Q19 TRT + WALE, uniform body force, D3Q7 scalar with
buoyancy, an obstacle with mid-link bounce-back, no-slip walls, streamwise
periodic) steps
with kernels in which every other feature's branch is removed at compile
time; every other lattice keeps the generic kernels.  Both compute the same
operations, so the states agree up to the FP rounding of the compiled
variant: FP32 1e-6, FP16 1e-4 and BF16 1e-3 of max|f| (and of max|g|)
after 40 steps, the drag histories to ten times that."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-6, "fp16s": 1e-4, "bf16s": 1e-3}


def _channel(precision, **extra):
    from aero_b200 import Box, Solver3D
    nz, ny, nx = 12, 16, 40
    box = Box(width=6, height=6, depth=12, cx_frac=0.3, cy_frac=3 / 16, cz_frac=0.5)
    solid = box.mark_solid(nz, ny, nx)
    kw = dict(omega=1 / 0.8, u0=0.05, D=6.0, collision="trt", trt_lambda=3 / 16, les=True, les_model="wale",
              les_cs=0.5, wall_bc="noslip", streamwise_bc="periodic", body_force_x=1e-5, thermal=True, T_hot=1.0,
              T_cold=0.0, alpha_T=0.02, buoyancy=True, g_gravity=1e-3, beta=1.0, T_ref=0.5,
              scalar_lattice="reduced", precision=precision)
    kw.update(extra)
    return Solver3D(Nz=nz, Ny=ny, Nx=nx, solid=solid, **kw)


def _run(s):
    rng = np.random.default_rng(3)
    shp = s.solid.shape
    s.set_equilibrium_state(ux=0.05 + 0.01 * rng.uniform(-1, 1, shp), uy=0.01 * rng.uniform(-1, 1, shp),
                            T=0.5 + 1e-3 * rng.uniform(-1, 1, shp))
    r = s.run(40, check_every=20, verbose=False)
    return np.array(r["Cd_history"])


@pytest.mark.parametrize("precision", ["fp32", "fp16s", "bf16s"])
def test_thermal_channel_kernels_equal_generic(precision, monkeypatch):
    monkeypatch.delenv("AERO_B200_GENERIC_KERNELS", raising=False)
    a = _channel(precision)
    assert a._engine.kernel_variant() == 1
    cda = _run(a)
    monkeypatch.setenv("AERO_B200_GENERIC_KERNELS", "1")
    b = _channel(precision)
    assert b._engine.kernel_variant() == 0
    cdb = _run(b)
    tol = TOL[precision]
    np.testing.assert_allclose(a.f, b.f, rtol=0, atol=tol * np.abs(b.f).max())
    np.testing.assert_allclose(a.g, b.g, rtol=0, atol=tol * np.abs(b.g).max())
    np.testing.assert_allclose(cda, cdb, rtol=0, atol=10 * tol * np.abs(cdb).max())
    assert a.status() == b.status() == 0


def test_other_feature_words_take_the_generic_kernels(monkeypatch):
    monkeypatch.delenv("AERO_B200_GENERIC_KERNELS", raising=False)
    for extra in (dict(precision="fp64"), dict(collision="bgk"), dict(buoyancy=False),
                  dict(scalar_lattice="full"), dict(les_model="smagorinsky"), dict(wall_bc="slip")):
        kw = dict(precision="fp32")
        kw.update(extra)
        s = _channel(**kw)
        assert s._engine.kernel_variant() == 0, extra
