"""Continuous-batching server (aero_b200.serve): trace generation and the
footprint bound on CPU; on the GPU, served results equal sequential plain
solves with the same stopping rule, each case gives the same result alone
and in the mix, and requests that arrive while others run are admitted
before those finish."""

import ctypes
import math

import numpy as np
import pytest

from aero_b200 import serve


def test_trace_is_seeded_and_respects_the_rules():
    a = serve.trace(200, seed=3, rate=5.0)
    b = serve.trace(200, seed=3, rate=5.0)
    assert [serve.case_dict(c) for c in a] == [serve.case_dict(c) for c in b]
    arr = [c.arrival for c in a]
    assert all(x < y for x, y in zip(arr, arr[1:]))
    n2 = sum(c.dims == 2 for c in a)
    assert 0.55 < n2 / len(a) < 0.85
    for c in a:
        assert c.ny == c.nx // 2 and (c.nz == (c.ny if c.dims == 3 else 1))
        assert (256 <= c.nx <= 1024) if c.dims == 2 else (96 <= c.nx <= 320)
        D = serve.geometry(c).reference_length()
        tau = 1.0 / serve.omega_of(c, D)
        assert tau >= 0.51 - 1e-12 and c.u0 <= 0.1 + 1e-12
        assert c.les == (c.Re > 200.0)
        assert c.collision in ("bgk", "trt", "mrt")


def test_trace_cases_do_not_depend_on_the_arrival_rate():
    a = serve.trace(50, seed=9, rate=0.0)
    b = serve.trace(50, seed=9, rate=7.0)
    strip = lambda c: {k: v for k, v in serve.case_dict(c).items() if k != "arrival"}
    assert [strip(c) for c in a] == [strip(c) for c in b]
    assert all(c.arrival == 0.0 for c in a) and b[-1].arrival > 0.0


def test_footprint_bounds_the_workspace():
    """footprint() is at least the workspace aero_workspace_size reports
    (computed through the C ABI, no GPU needed)."""
    from aero_b200 import _lib
    from aero_b200.links import build_surface_links
    lib = _lib.load(build_if_missing=False)
    for c in serve.trace(12, seed=5, rate=0.0, nx2=(64, 192), nx3=(32, 64)):
        c.les = True
        geo = serve.geometry(c)
        shape = (c.ny, c.nx) if c.dims == 2 else (c.nz, c.ny, c.nx)
        solid = geo.mark_solid(*shape)
        links, q = build_surface_links(solid, None)
        P = _lib.AeroParams()
        P.abi_version, P.dims = _lib.ABI_VERSION, c.dims
        P.nx, P.ny, P.nz = c.nx, c.ny, c.nz
        P.storage = _lib.STORE[c.precision]
        P.collision = _lib.COLLISION["bgk"]
        P.inlet_bc, P.outlet_bc, P.wall_bc = 1, 1, 1
        P.streamwise_open, P.les = 1, 1
        P.omega, P.u0, P.rho0 = 1.0 / 0.6, c.u0, 1.0
        h = ctypes.c_void_p()
        assert lib.aero_create(ctypes.byref(P), ctypes.byref(h)) == 0
        s8 = np.ascontiguousarray(solid, dtype=np.uint8)
        links = np.ascontiguousarray(links, dtype=np.int32)
        q = np.ascontiguousarray(q, dtype=np.float32)
        assert lib.aero_set_geometry(h, s8.ctypes.data, links.ctypes.data if len(links) else None,
                                     q.ctypes.data if len(q) else None, len(links), None) == 0
        nb = ctypes.c_uint64()
        assert lib.aero_workspace_size(h, ctypes.byref(nb)) == 0
        assert serve.footprint(c) >= nb.value
        lib.aero_destroy(h)
        # the same lattice in the AA layout: one population buffer plus staging
        P.layout = 1
        assert lib.aero_create(ctypes.byref(P), ctypes.byref(h)) == 0
        assert lib.aero_set_geometry(h, s8.ctypes.data, links.ctypes.data if len(links) else None,
                                     q.ctypes.data if len(q) else None, len(links), None) == 0
        na = ctypes.c_uint64()
        assert lib.aero_workspace_size(h, ctypes.byref(na)) == 0
        assert na.value < nb.value
        assert serve.footprint(c) > serve.footprint(c, layout="aa") >= na.value
        lib.aero_destroy(h)


def _small_cases():
    """Mixed 2D/3D cases at stable relaxation times (tau 0.55; TRT at tau
    0.86, where the reference's TRT parameters are stable), so that no
    verdict depends on when a divergence is detected."""
    cs = [
        serve.Case(0, 2, 96, 48, shape="cylinder", size=5, Re=30, collision="bgk", arrival=0.0),
        serve.Case(1, 2, 80, 40, shape="rectangle", size=4, Re=24, collision="mrt", arrival=0.0),
        serve.Case(2, 3, 48, 24, 24, shape="sphere", size=3, Re=18, collision="mrt", arrival=0.0),
        serve.Case(3, 2, 64, 32, shape="cylinder", size=4, Re=24, collision="bgk", les=True, arrival=0.0),
        serve.Case(4, 3, 40, 20, 20, shape="box", size=3, Re=18, collision="bgk", arrival=0.0),
        serve.Case(5, 2, 128, 64, shape="cylinder", size=6, Re=5, collision="trt", arrival=0.0),
    ]
    for c in cs:
        c.max_steps = 600
    return cs


KW = dict(chunk=50, window=100, tol=2e-3)


@pytest.mark.gpu
def test_served_results_equal_plain_sequential_solves():
    plain = {r.id: r for r in serve.run_plain(_small_cases(), **KW)}
    srv = serve.Server(hbm_cap=8e9, max_members=8, **KW)
    served = {r.id: r for r in srv.run(_small_cases())}
    srv.close()
    assert set(plain) == set(served)
    for k, p in plain.items():
        s = served[k]
        assert s.status == p.status and s.steps == p.steps, (k, s, p)
        if p.status in ("converged", "max_steps") and math.isfinite(p.cd_mean) and p.cd_mean != 0.0:
            # batch and single-lattice kernels differ only in FP32 rounding
            assert abs(s.cd_mean - p.cd_mean) <= 1e-5 * abs(p.cd_mean), (k, s.cd_mean, p.cd_mean)


@pytest.mark.gpu
def test_each_result_same_alone_and_in_the_mix():
    mix = serve.Server(hbm_cap=8e9, max_members=8, **KW)
    together = {r.id: r for r in mix.run(_small_cases())}
    mix.close()
    for c in _small_cases():
        one = serve.Server(hbm_cap=8e9, max_members=1, **KW)
        (r,) = one.run([c])
        one.close()
        t = together[c.id]
        assert (r.status, r.steps) == (t.status, t.steps)
        assert r.cd_mean == t.cd_mean or (math.isnan(r.cd_mean) and math.isnan(t.cd_mean))


@pytest.mark.gpu
def test_late_requests_join_while_others_run():
    cs = _small_cases()
    for c in cs:
        c.max_steps = 2000
    # half the requests arrive after the first ones are running
    for c in cs[3:]:
        c.arrival = 0.3
    # simulated clock: every reading advances 10 ms, so the late requests
    # arrive after a few rounds whatever the speed of the GPU
    t = [0.0]

    def clock():
        t[0] += 0.01
        return t[0]

    def sleep(dt):
        t[0] += dt

    srv = serve.Server(hbm_cap=8e9, max_members=8, chunk=50, window=2000, tol=0.0)
    res = {r.id: r for r in srv.run(cs, clock=clock, sleep=sleep)}
    srv.close()
    first_done = min(res[c.id].done for c in cs[:3])
    late_admitted = max(res[c.id].admitted for c in cs[3:])
    assert late_admitted < first_done        # admitted while the first cases were still running
    assert all(r.status == "max_steps" and r.steps == 2000 for r in res.values())


def test_oversized_request_is_rejected_without_gpu_work(monkeypatch):
    """A request larger than the HBM cap is rejected at admission."""
    class FakeBatch:
        def __init__(self, *a, **k):
            self.device = None
        def close(self):
            pass
    monkeypatch.setattr(serve, "Batch", FakeBatch)
    import sys, types
    fake_torch = types.SimpleNamespace(cuda=types.SimpleNamespace(synchronize=lambda d=None: None,
                                                                  Stream=lambda d=None: None))
    monkeypatch.setitem(sys.modules, "torch", fake_torch)
    srv = serve.Server(hbm_cap=1e6, max_members=4, chunk=10, window=10)
    (r,) = srv.run([serve.Case(0, 3, 128, 64, 64)])
    assert r.status == "rejected" and r.steps == 0


def test_admission_takes_the_aa_layout_when_two_buffers_do_not_fit(monkeypatch):
    """layout="auto": a request of at least 2^20 cells whose two-buffer
    footprint does not fit beside the running requests, while its one-buffer
    footprint does, is built in the AA layout; smaller requests and requests
    that fit keep two buffers; layout="aa" builds every large request in it.
    Checked with a fake batch and fake solvers, no GPU."""
    import sys
    import types
    built = []

    class FakeBatch:
        def __init__(self, *a, **k):
            self.device = None
            self.members = []

        def add(self, s):
            self.members.append(s)

        def remove(self, s):
            self.members.remove(s)

        def step(self, n):
            pass

        def converge(self, window, tol):
            rows = np.zeros((len(self.members), len(serve.CONVERGE_FIELDS)))
            rows[:, serve._F["converged"]] = 1.0
            return rows

        def close(self):
            pass

    monkeypatch.setattr(serve, "Batch", FakeBatch)
    monkeypatch.setattr(serve, "make_solver", lambda c, dev, hist, layout="ab": built.append((c.id, layout)) or object())
    fake_torch = types.SimpleNamespace(cuda=types.SimpleNamespace(
        synchronize=lambda d=None: None, Stream=lambda d=None: None, stream=lambda st: _Null()))
    monkeypatch.setitem(sys.modules, "torch", fake_torch)
    big = serve.Case(0, 3, 128, 96, 96, shape="sphere", size=8)      # 1,179,648 cells
    small = serve.Case(1, 3, 64, 32, 32, shape="sphere", size=4)     # 65,536 cells
    ab, aa = serve.footprint(big), serve.footprint(big, layout="aa")
    assert aa < ab
    for layout, cap, want in (("auto", 10 * ab, "ab"), ("auto", (ab + aa) / 2, "aa"), ("aa", 10 * ab, "aa"),
                              ("ab", (ab + aa) / 2, None)):
        built.clear()
        srv = serve.Server(hbm_cap=cap, max_members=4, chunk=10, window=10, layout=layout)
        res = {r.id: r for r in srv.run([big, small])}
        assert dict(built).get(1) == "ab"
        if want is None:
            assert res[0].status == "rejected" and 0 not in dict(built)
        else:
            assert dict(built)[0] == want and res[0].status == "converged"
            assert srv.stats["aa_admitted"] == (want == "aa")
    with pytest.raises(ValueError):
        serve.Server(layout="ba")


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


@pytest.mark.gpu
def test_aa_requests_serve_like_two_buffer_ones():
    """A large request served in the AA layout (in the batch beside small
    two-buffer requests) reaches the verdict and step count of the same
    request served with two buffers, drag within FP32 rounding."""
    cases = lambda: [serve.Case(0, 3, 128, 96, 96, shape="sphere", size=8, Re=40, collision="mrt", max_steps=150),
                     serve.Case(1, 2, 96, 48, shape="cylinder", size=5, Re=30, collision="bgk", max_steps=150)]
    out = {}
    for layout in ("ab", "aa"):
        srv = serve.Server(hbm_cap=8e9, max_members=4, chunk=50, window=100, tol=2e-3, layout=layout)
        out[layout] = {r.id: r for r in srv.run(cases())}
        assert srv.stats["aa_admitted"] == (layout == "aa")
        srv.close()
    for k, a in out["ab"].items():
        b = out["aa"][k]
        assert (a.status, a.steps) == (b.status, b.steps)
        if math.isfinite(a.cd_mean) and a.cd_mean != 0.0:
            assert abs(a.cd_mean - b.cd_mean) <= 1e-5 * abs(a.cd_mean)


@pytest.mark.gpu
def test_diverged_request_is_retired_and_others_finish():
    """A request whose state goes bad (a NaN injected into its initial state
    on the host) is retired as 'diverged' after its first round, from the
    device status word; the other requests in the same batch run to their
    normal end with the same results as without the faulty one."""
    def poison(case, solver):
        if case.id == 1:
            f = solver.f
            f[:, 3, 5] = np.nan
            solver.f = f

    srv = serve.Server(hbm_cap=8e9, max_members=8, on_admit=poison, **KW)
    res = {r.id: r for r in srv.run(_small_cases())}
    srv.close()
    clean = serve.Server(hbm_cap=8e9, max_members=8, **KW)
    ref = {r.id: r for r in clean.run(_small_cases())}
    clean.close()
    assert res[1].status == "diverged" and res[1].steps == KW["chunk"]
    for k in ref:
        if k == 1:
            continue
        assert (res[k].status, res[k].steps) == (ref[k].status, ref[k].steps)
        assert res[k].cd_mean == ref[k].cd_mean or (math.isnan(res[k].cd_mean) and math.isnan(ref[k].cd_mean))


@pytest.mark.gpu
def test_cancelled_requests_leave_and_others_finish():
    """A running request cancelled after two rounds leaves the batch with
    status 'cancelled'; a queued one is dropped before it starts; the rest
    finish as they would without them."""
    cs = _small_cases()
    cs[4].arrival = 1e9  # never arrives before it is cancelled

    def on_round(srv, k):
        if k == 2:
            srv.cancel(1)
            srv.cancel(4)

    srv = serve.Server(hbm_cap=8e9, max_members=8, on_round=on_round, **KW)
    res = {r.id: r for r in srv.run(cs)}
    srv.close()
    assert res[1].status == "cancelled" and res[1].steps == 3 * KW["chunk"]
    assert res[4].status == "cancelled" and res[4].steps == 0
    clean = serve.Server(hbm_cap=8e9, max_members=8, **KW)
    ref = {r.id: r for r in clean.run(_small_cases())}
    clean.close()
    for k in (0, 2, 3, 5):
        assert (res[k].status, res[k].steps, res[k].cd_mean) == (ref[k].status, ref[k].steps, ref[k].cd_mean)


def test_admission_is_budgeted_by_the_chunk_time(monkeypatch):
    """While a chunk runs, requests are set up until one more set-up would
    outlast the previous chunk's GPU time: with a 50 ms chunk and 4 ms per
    set-up, 12 a round once the chunk is timed; 8 (admit_idle) before that.
    Simulated clock, fake batch and solvers: no GPU."""
    import contextlib
    import sys
    import types

    t = [0.0]
    clock = lambda: t[0]

    def sleep(dt):
        t[0] += dt

    class FakeBatch:
        chunk_time = 0.05

        def __init__(self, *a, **k):
            self.device = None
            self.members = []
            self.steps = {}
            self.joins = [0]       # joins after each round's admissions
            self.launched = None

        def step(self, n):
            self.launched = t[0]
            for s in self.members:
                self.steps[id(s)] += n

        def converge(self, window, tol):
            t[0] = max(t[0], self.launched + self.chunk_time)  # waits for the chunk
            self.joins.append(0)
            rows = np.zeros((len(self.members), len(serve.CONVERGE_FIELDS)))
            for k, s in enumerate(self.members):
                rows[k, serve._F["steps"]] = self.steps[id(s)]
                rows[k, serve._F["ratio"]] = math.inf
            return rows

        def add(self, s):
            self.members.append(s)
            self.steps[id(s)] = 0
            self.joins[-1] += 1

        def remove(self, s):
            self.members.remove(s)

        def close(self):
            pass

    def fake_solver(case, device=None, hist_capacity=4096, layout="ab"):
        t[0] += 0.004  # set-up time of one request
        return types.SimpleNamespace(case=case)

    monkeypatch.setattr(serve, "Batch", FakeBatch)
    monkeypatch.setattr(serve, "make_solver", fake_solver)
    fake_torch = types.SimpleNamespace(cuda=types.SimpleNamespace(
        synchronize=lambda d=None: None, Stream=lambda d=None: None, stream=lambda s: contextlib.nullcontext()))
    monkeypatch.setitem(sys.modules, "torch", fake_torch)
    cases = [serve.Case(i, 2, 64, 32, max_steps=40) for i in range(60)]
    srv = serve.Server(hbm_cap=1e12, max_members=256, chunk=10, window=10, tol=0.0)
    res = srv.run(cases, clock=clock, sleep=sleep)
    joins = srv.batch.joins
    srv.close()
    assert joins[:3] == [8, 8, 12]
    assert all(j <= 12 for j in joins)
    assert sorted(r.id for r in res) == list(range(60))
    assert all(r.status == "max_steps" and r.steps == 40 for r in res)
