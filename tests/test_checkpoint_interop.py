"""Checkpoints exchanged with the reference.

The fixtures ckpt_ref_{2d,3d}.npz are files written by the reference's own
save_checkpoint (aero/lbm/solver.py:638-686, aero/lbm/solver3d.py:727-780)
after a seeded run, and ckpt_cont_{2d,3d}.npz hold the state and histories
the reference reached n2 steps later, with the names of the reference
constructors' keyword arguments (tests/golden/make_golden.py).

* A reference checkpoint loads through from_checkpoint and continues to the
  reference's state: FP64 storage |df| <= 1e-10 max|f| (as the golden parity
  tests), FP32 relative L2 of rho and u <= 1e-5.
* A checkpoint this engine writes has exactly the reference's keys and
  dtypes (plus b200_options, which the reference's loader ignores), and its
  params_json has exactly the keys of the reference's, all of them keyword
  arguments of the reference constructor.
"""

import json

import numpy as np
import pytest

from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = ("2d", "3d")


def _cls(tag):
    from aero_b200 import Solver, Solver3D
    return Solver if tag == "2d" else Solver3D


def _macro(f, dims):
    from aero_b200.lattice import macroscopic
    return macroscopic(f, dims)


def _rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("tag", CASES)
def test_reference_checkpoint_continues_fp64(tag):
    ref_path = GOLDEN / f"ckpt_ref_{tag}.npz"
    cont = np.load(GOLDEN / f"ckpt_cont_{tag}.npz")
    s = _cls(tag).from_checkpoint(str(ref_path), precision="fp64")
    ck = np.load(ref_path)
    assert s.step_count == int(ck["step_count"])
    assert np.array_equal(s.surface_links, ck["surface_links"]) and np.array_equal(s.q_vals, ck["q_vals"])
    np.testing.assert_array_equal(np.array(s.Cd_history), ck["Cd_history"])
    s.run(int(cont["n2"]), check_every=int(cont["n2"]) + 1, verbose=False)
    assert s.step_count == int(cont["step_count"])
    scale = np.abs(cont["f"]).max()
    np.testing.assert_allclose(s.f, cont["f"], rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(s._f_outlet_prev, cont["f_outlet_prev"], rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(s.g, cont["g"], rtol=0, atol=1e-10 * np.abs(cont["g"]).max())
    cd = cont["Cd_history"]
    np.testing.assert_allclose(np.array(s.Cd_history), cd, rtol=0, atol=1e-8 * np.abs(cd).max())


@pytest.mark.parametrize("tag", CASES)
def test_reference_checkpoint_continues_fp32(tag):
    cont = np.load(GOLDEN / f"ckpt_cont_{tag}.npz")
    s = _cls(tag).from_checkpoint(str(GOLDEN / f"ckpt_ref_{tag}.npz"))
    assert s.precision == "fp32"
    s.run(int(cont["n2"]), check_every=int(cont["n2"]) + 1, verbose=False)
    dims = 2 if tag == "2d" else 3
    got, ref = _macro(s.f, dims), _macro(cont["f"], dims)
    assert _rel_l2(got[0], ref[0]) <= 1e-5
    assert _rel_l2(np.stack(got[1:]), np.stack(ref[1:])) <= 1e-5


@pytest.mark.parametrize("tag", CASES)
def test_engine_checkpoint_has_the_reference_layout(tag, tmp_path):
    ref = np.load(GOLDEN / f"ckpt_ref_{tag}.npz")
    cont = np.load(GOLDEN / f"ckpt_cont_{tag}.npz")
    s = _cls(tag).from_checkpoint(str(GOLDEN / f"ckpt_ref_{tag}.npz"), precision="fp64")
    s.run(3, check_every=4, verbose=False)
    path = tmp_path / "ours.npz"
    s.save_checkpoint(str(path))
    ours = np.load(path)
    assert set(ours.files) == set(ref.files) | {"b200_options"}
    for k in ref.files:
        assert ours[k].dtype.kind == ref[k].dtype.kind and ours[k].dtype.itemsize == ref[k].dtype.itemsize \
            or k == "params_json", (k, ours[k].dtype, ref[k].dtype)
        assert ours[k].ndim == ref[k].ndim, k
    p_ours, p_ref = json.loads(str(ours["params_json"])), json.loads(str(ref["params_json"]))
    assert set(p_ours) == set(p_ref)
    assert set(p_ours) <= set(json.loads(str(cont["ctor_params"])))
    assert p_ours["backend"] in ("numpy", "numba", "auto")
    assert json.loads(str(ours["b200_options"]))["precision"] == "fp64"
    # and it round-trips through this engine: the same state and step count
    t = _cls(tag).from_checkpoint(str(path))
    assert t.precision == "fp64" and t.step_count == s.step_count
    np.testing.assert_array_equal(t.f, s.f)
    np.testing.assert_array_equal(t.g, s.g)


def test_checkpoint_link_table_is_adopted(tmp_path):
    """The reference's load_checkpoint adopts the checkpoint's surface links
    and q values (solver.py:705-709): a table with different q values is
    uploaded to the engine and changes the next step exactly as the oracle
    stepping with that table."""
    from oracle.oracle import OracleSolver
    ref = np.load(GOLDEN / "ckpt_ref_2d.npz")
    d = {k: ref[k] for k in ref.files}
    d["q_vals"] = np.clip(d["q_vals"] * np.float32(0.9), np.float32(1e-4), np.float32(1.0)).astype(np.float32)
    path = tmp_path / "q.npz"
    np.savez_compressed(path, **d)
    s = _cls("2d").from_checkpoint(str(path), precision="fp64")
    assert np.array_equal(s.q_vals, d["q_vals"])
    params = json.loads(str(d["params_json"]))
    o = OracleSolver(solid=d["solid"], phi=d["phi"], omega=params["omega"], u0=params["u0"], D=params["D"],
                     **{k: params[k] for k in ("collision", "wall_bc", "outlet_bc", "bouzidi", "thermal", "alpha_T",
                                               "buoyancy", "g_gravity", "beta", "T_ref")})
    o.q = np.ascontiguousarray(d["q_vals"])
    o.f, o.f_outlet_prev, o.g = d["f"].copy(), d["f_outlet_prev"].copy(), d["g"].copy()
    for _ in range(5):
        s._step()
        o.step()
    np.testing.assert_allclose(s.f, o.f, rtol=0, atol=1e-10 * np.abs(o.f).max())
