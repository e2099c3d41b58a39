"""Density and velocity computed on the device (aero_get_macroscopic) against
compute_macroscopic(_3d) (d2q9.py:44-63, d3q19.py:80-102) applied on the host
to the state the engine hands out (self.f).  Both sum f_i = w_i + d_i over
the directions and scale by 1 / rho; the host's velocity sums go through
BLAS (tensordot) in an order of its own, so FP64 agrees to the round-off of
19 terms of size ~0.1: a few 1e-16 absolute, within 1e-12 of max|.|."""

import numpy as np
import pytest

from tests.golden_cases import load_case

pytestmark = pytest.mark.gpu


def _check(s, dims):
    from aero_b200.lattice import macroscopic
    s._flush_host_state()  # a state assigned to s.f reaches the device at the next step
    got = s._engine.macroscopic_device().cpu().numpy()
    ref = macroscopic(s.f, dims)
    assert got.shape == (1 + dims,) + s.f.shape[1:]
    for k in range(1 + dims):
        np.testing.assert_allclose(got[k], ref[k], rtol=0, atol=1e-12 * max(np.abs(ref[k]).max(), 1e-30))


@pytest.mark.parametrize("name", ["c2d_bgk_slip_convective_pert", "c3d_mrt_smag_bouzidi_sponge",
                                  "c3d_trt_wale_periodic_bodyforce_thermal", "c3d_bgk_sem_inlet"])
@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16s"])
def test_device_moments_equal_host_moments_of_the_state(name, precision):
    from tests.test_gpu_parity import _solver
    c = load_case(name)
    s = _solver(c, precision=precision)
    _check(s, c["dims"])           # the state as set, before any step
    for _ in range(c["steps"]):
        s._step()
    _check(s, c["dims"])           # the post-boundary state after steps


def test_run_result_fields_are_the_moments_of_the_state():
    from aero_b200.lattice import macroscopic
    from tests.test_gpu_parity import _solver
    c = load_case("c3d_mrt_smag_bouzidi_sponge")
    s = _solver(c, precision="fp32")
    r = s.run(c["steps"], check_every=c["steps"] + 1, verbose=False)
    ref = macroscopic(s.f, 3)
    for k, name in enumerate(("rho", "ux", "uy", "uz")):
        assert r[name].dtype == np.float64 and r[name].shape == s.f.shape[1:]
        np.testing.assert_allclose(r[name], ref[k], rtol=0, atol=1e-12 * np.abs(ref[k]).max())
    # a second run hands out new arrays, not the first run's
    r2 = s.run(3, check_every=10, verbose=False)
    assert not np.shares_memory(r["rho"], r2["rho"])


@pytest.mark.parametrize("n", [1000, (32 << 20) // 8, (32 << 20) // 8 + 1, 9_000_001])
def test_copy_to_host_through_bounce_buffers(n):
    """Results larger than one pinned bounce buffer (32 MiB) reach the host
    chunk by chunk; the bytes equal those of a plain copy, whether the size
    is below, at, just above or several buffers and a remainder above it,
    into a fresh array or a given one, FP64 or FP32."""
    import torch
    from aero_b200.engine import copy_to_host
    g = torch.Generator(device="cuda").manual_seed(n)
    for dt in (torch.float64, torch.float32):
        src = torch.rand((n,), generator=g, device="cuda", dtype=torch.float64).to(dt)
        ref = src.cpu().numpy()
        got = copy_to_host(src)
        assert got.dtype == ref.dtype and got.shape == ref.shape
        np.testing.assert_array_equal(got, ref)
        out = np.full(ref.shape, -1.0, dtype=ref.dtype)
        assert copy_to_host(src.reshape(1, -1), out.reshape(1, -1)) is not None
        np.testing.assert_array_equal(out, ref)
