"""Continuous-batching request loop for wind-tunnel cases on one GPU.

Requests (``Case``) arrive over time.  The server admits each one as soon as
its device footprint fits under an HBM cap and a batch slot is free, builds
its solver (geometry, links, initial equilibrium state on the device) and
adds it to the running ``Batch``; every member then advances with the
others in ``chunk``-step rounds.  After each round the batch evaluates the
reference's drag-convergence rule (``analyze_convergence``,
aero/diagnostics.py:87-120: std / mean|Cd| over a trailing window) for all
members on the device, and the server retires the members that converged,
reached their step limit or diverged (the device status word, the test of
``check_stability``, aero/diagnostics.py:32-71), freeing their memory for
waiting requests.  Populations and force histories stay on the device for
the whole life of a case; per round the host reads only the convergence
table.

``run_plain`` solves the same cases one after another through the plain
single-solver API with the same stopping rule (checked at the same step
counts), which is the sequential baseline the serving throughput is
compared with.

Case construction follows the reference CLI defaults (cli.py:43-170,
cli3d.py:36-174: velocity inlet, convective outlet, slip walls, LES
constant 0.16) and derives nu = u0 D / Re, omega = 1 / (3 nu + 1/2)
(cli.py:191-204).  There is no serving loop in the reference.
"""

from __future__ import annotations

import math
import time
from dataclasses import asdict, dataclass, field
from typing import Dict, List, Optional

import numpy as np

from .batch import CONVERGE_FIELDS, Batch

_F = {k: i for i, k in enumerate(CONVERGE_FIELDS)}
STATUS_DIVERGED = 1  # bit 0 of the device status word


@dataclass
class Case:
    """One wind-tunnel request."""
    id: int
    dims: int
    nx: int
    ny: int
    nz: int = 1
    shape: str = "cylinder"     # cylinder | rectangle (2D), sphere | box (3D)
    size: float = 8.0           # radius, or half-width, in cells
    Re: float = 100.0
    u0: float = 0.05
    collision: str = "bgk"
    les: bool = False
    precision: str = "fp32"
    arrival: float = 0.0        # seconds after the start of the trace
    max_steps: int = 50000


@dataclass
class Result:
    id: int
    status: str                 # converged | max_steps | diverged | rejected | cancelled
    steps: int
    cd_mean: float
    ratio: float
    arrival: float
    admitted: float
    done: float
    cells: int
    footprint: int

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def geometry(case: Case):
    from .geometry import Box, Cylinder, Rectangle, Sphere
    h = float(case.size)
    if case.dims == 2:
        if case.shape == "rectangle":
            return Rectangle(width=2 * h, height=2 * h, cx_frac=0.25, cy_frac=0.5)
        return Cylinder(radius=h, cx_frac=0.25, cy_frac=0.5)
    if case.shape == "box":
        return Box(width=2 * h, height=2 * h, depth=2 * h, cx_frac=0.25, cy_frac=0.5, cz_frac=0.5)
    return Sphere(radius=h, cx_frac=0.25, cy_frac=0.5, cz_frac=0.5)


def omega_of(case: Case, D: float) -> float:
    nu = case.u0 * D / case.Re
    return 1.0 / (3.0 * nu + 0.5)


def make_solver(case: Case, device=None, hist_capacity: int = 4096, layout: str = "ab"):
    """The solver of a case, with the reference CLI's boundary conditions, in
    population layout `layout` ("ab" or "aa")."""
    from .solver import Solver
    from .solver3d import Solver3D
    geo = geometry(case)
    D = geo.reference_length()
    kw = dict(omega=omega_of(case, D), u0=case.u0, D=D, wall_bc="slip", inlet_bc="velocity",
              outlet_bc="convective", collision=case.collision, les=case.les, les_cs=0.16,
              precision=case.precision, device=device, hist_capacity=hist_capacity, layout=layout)
    if case.dims == 2:
        solid = geo.mark_solid(case.ny, case.nx)
        return Solver(Ny=case.ny, Nx=case.nx, solid=solid, **kw)
    solid = geo.mark_solid(case.nz, case.ny, case.nx)
    return Solver3D(Nz=case.nz, Ny=case.ny, Nx=case.nx, solid=solid, **kw)


def footprint(case: Case, hist_capacity: int = 4096, layout: str = "ab") -> int:
    """Upper bound of the device bytes a case holds while admitted: the
    population buffers (two, or one in the AA layout plus its staging of
    link cells and the outlet plane), flags, LES velocities and outlet state
    of its workspace, the force ring, plus the FP64 initial state built
    during set-up."""
    Q = 9 if case.dims == 2 else 19
    cells = case.nx * case.ny * case.nz
    cs = (cells + 63) // 64 * 64
    sb = {"fp32": 4, "fp64": 8, "fp16s": 2, "bf16s": 2}[case.precision]
    rb = 8 if case.precision == "fp64" else 4
    nbuf = 1 if layout == "aa" else 2
    ws = nbuf * Q * cs * sb + cs + 32 + 8 * (cs // 32 + 64)
    if layout == "aa":
        # link-cell staging (an upper bound: every cell of the obstacle's
        # bounding box a link cell) and the outlet plane
        box = int(2 * case.size + 4) ** case.dims
        ws += 2 * Q * rb * min(box, cells) + Q * rb * case.ny * case.nz
    ws += (3 * cs * rb if case.les and case.collision != "mrt" else 0)
    ws += 2 * 20 * case.ny * case.nz * rb + 96 * hist_capacity + (1 << 20)
    staging = Q * cells * 8 * 2
    return int(ws + staging)


def _cells(case: Case) -> int:
    return case.nx * case.ny * case.nz


# Requests of at least this many cells step in the batch on their own
# kernels, which is what lets them take the AA layout there.
AA_MIN_CELLS = 1 << 20


class Server:
    """Continuous batching of wind-tunnel cases on one device."""

    def __init__(self, hbm_cap: float = 150e9, max_members: int = 256, chunk: int = 200,
                 window: int = 2000, tol: float = 1e-3, device=None, hist_capacity: int = 4096,
                 on_admit=None, admit_per_round: int = 64, on_round=None, admit_idle: int = 8,
                 layout: str = "auto"):
        if window > hist_capacity:
            raise ValueError("the convergence window must fit the force history ring")
        if layout not in ("ab", "aa", "auto"):
            raise ValueError(f"Unknown layout '{layout}'. Choose 'ab', 'aa' or 'auto'.")
        # population layout of the requests large enough to step on their own
        # kernels in the batch (AA_MIN_CELLS; smaller ones always take two
        # buffers): "ab", "aa" (one buffer updated in place, half the
        # population memory, 0.9x the rate), or "auto": "aa" only for a
        # request whose two-buffer footprint does not fit beside the running
        # ones while its one-buffer footprint does
        self.layout = layout
        self.hbm_cap = float(hbm_cap)
        self.max_members = int(max_members)
        self.chunk = int(chunk)
        self.window = int(window)
        self.tol = float(tol)
        self.device = device
        self.hist_capacity = int(hist_capacity)
        self.batch = Batch(max_members=max_members, device=device)
        self.stats: Dict[str, float] = {}
        # optional callback(case, solver) run before a new solver joins the
        # batch, e.g. to set a state of its own
        self.on_admit = on_admit
        # requests set up per round.  While a chunk runs, set-up continues as
        # long as this round's set-up time plus one more set-up (at its
        # running mean) stays within the previous chunk's GPU time (so it
        # hides behind the chunk), up to admit_per_round;
        # with nothing running, or before a chunk has been timed, at most
        # admit_idle, so a burst of arrivals does not hold the GPU idle
        # behind serial set-up
        self.admit_per_round = max(int(admit_per_round), 1)
        self.admit_idle = max(int(admit_idle), 1)
        # optional callback(server, round) after each round, e.g. to cancel requests
        self.on_round = on_round
        self.cancelled = set()

    def cancel(self, case_id: int) -> None:
        """Cancels a request: a waiting one is dropped, a running one leaves the
        batch at the end of the current round; either reports 'cancelled'."""
        self.cancelled.add(int(case_id))

    def run(self, cases: List[Case], clock=time.perf_counter, sleep=time.sleep) -> List[Result]:
        """Serves the cases (arrival times relative to the call) and returns
        one Result per case, in completion order.

        One round: launch the next chunk of steps for the members (the call
        returns at once), build the solvers of the requests admitted now on
        a side stream while that chunk runs, evaluate convergence (this
        waits for the chunk), retire finished members, then let the new
        solvers join."""
        import torch
        side = torch.cuda.Stream(self.batch.device)
        pending = sorted(cases, key=lambda c: (c.arrival, c.id))
        queue: List[Case] = []
        active: List[tuple] = []     # (case, solver, admitted, bytes), join order = batch order
        results: List[Result] = []
        used = 0
        aa_admitted = 0
        cell_steps = 0
        setup_s = 0.0
        wait_s = 0.0
        t0 = clock()
        rounds = 0
        chunk_s = None  # launch-to-result time of the last chunk
        setup_avg = None  # running mean of one request's set-up time
        while pending or queue or active:
            stepped = bool(active)
            t_launch = clock()
            if stepped:
                self.batch.step(self.chunk)
                cell_steps += self.chunk * sum(_cells(a[0]) for a in active)
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.pop(0))
            for lst in (pending, queue):
                for c in [c for c in lst if c.id in self.cancelled]:
                    lst.remove(c)
                    results.append(Result(c.id, "cancelled", 0, math.nan, math.nan, c.arrival, now, now,
                                          _cells(c), 0))
            # admission, first come first served, by device footprint
            joining = []
            budget = chunk_s if (stepped and chunk_s is not None) else None
            cap = self.admit_per_round if budget is not None else self.admit_idle
            while (queue and len(active) + len(joining) < self.max_members and len(joining) < cap
                   and (budget is None or not joining or clock() - t_launch + (setup_avg or 0.0) <= budget)):
                c = queue[0]
                layout = "ab"
                need = footprint(c, self.hist_capacity)
                if _cells(c) >= AA_MIN_CELLS and self.layout != "ab":
                    need_aa = footprint(c, self.hist_capacity, "aa")
                    if self.layout == "aa" or (used + need > self.hbm_cap and used + need_aa <= self.hbm_cap) \
                            or need > self.hbm_cap >= need_aa:
                        layout, need = "aa", need_aa
                if need > self.hbm_cap:
                    queue.pop(0)
                    t = clock() - t0
                    results.append(Result(c.id, "rejected", 0, math.nan, math.nan, c.arrival, t, t,
                                          _cells(c), need))
                    continue
                if used + need > self.hbm_cap:
                    break
                queue.pop(0)
                ts = clock()
                with torch.cuda.stream(side):
                    s = make_solver(c, self.device, self.hist_capacity, layout)
                    if self.on_admit is not None:
                        self.on_admit(c, s)
                        s._flush_host_state()
                aa_admitted += layout == "aa"
                dt = clock() - ts
                setup_s += dt
                setup_avg = dt if setup_avg is None else 0.8 * setup_avg + 0.2 * dt
                used += need
                joining.append((c, s, clock() - t0, need))
            if stepped:
                tw = clock()
                table = self.batch.converge(self.window, self.tol)  # waits for the chunk
                wait_s += clock() - tw
                if clock() - tw > 1e-4:
                    # the chunk outlasted this round's set-up, so the wait
                    # ended with it: launch-to-result is its GPU time
                    chunk_s = clock() - t_launch
                elif chunk_s is not None:
                    chunk_s *= 0.5  # set-up outlasted the chunk: the GPU idled, admit fewer
                rounds += 1
                t = clock() - t0
                keep = []
                for (c, s, t_adm, need), row in zip(active, table):
                    steps = int(row[_F["steps"]])
                    status = int(row[_F["status"]])
                    if c.id in self.cancelled:
                        verdict = "cancelled"
                    elif status & STATUS_DIVERGED:
                        verdict = "diverged"
                    elif row[_F["converged"]] > 0.5:
                        verdict = "converged"
                    elif steps >= c.max_steps:
                        verdict = "max_steps"
                    else:
                        keep.append((c, s, t_adm, need))
                        continue
                    self.batch.remove(s)
                    used -= need
                    results.append(Result(c.id, verdict, steps, float(row[_F["mean"]]), float(row[_F["ratio"]]),
                                          c.arrival, t_adm, t, _cells(c), need))
                    del s
                active = keep
            for j in joining:
                self.batch.add(j[1])
                active.append(j)
            if self.on_round is not None and stepped:
                self.on_round(self, rounds)
            if not active and not joining and pending and not queue:
                sleep(max(0.0, pending[0].arrival - (clock() - t0)))
        torch.cuda.synchronize(self.batch.device)
        wall = clock() - t0
        self.stats = {"wall_s": wall, "rounds": rounds, "cell_steps": float(cell_steps),
                      "mlups": cell_steps / wall / 1e6 if wall > 0 else 0.0,
                      "setup_s": setup_s, "gpu_wait_s": wait_s, "aa_admitted": aa_admitted}
        return results

    def close(self):
        self.batch.close()


def run_plain(cases: List[Case], chunk: int = 200, window: int = 2000, tol: float = 1e-3, device=None,
              hist_capacity: int = 4096, clock=time.perf_counter, stats: Optional[dict] = None) -> List[Result]:
    """Solves the cases one after another through the plain solver API, with
    the serving rule checked at the same step counts; arrival times are
    ignored (the queue is full from the start).  `stats`, if given, receives
    the time spent building solvers."""
    from .diagnostics import analyze_convergence
    results = []
    t0 = clock()
    setup_s = 0.0
    for c in cases:
        t_adm = clock() - t0
        s = make_solver(c, device, hist_capacity)
        setup_s += clock() - t0 - t_adm
        cd: List[float] = []
        verdict = "max_steps"
        ratio = math.inf
        while True:
            r = s.run(chunk, check_every=chunk + 1, verbose=False)
            cd = list(r["Cd_history"])  # run() returns the solver's whole history
            if s.status() & STATUS_DIVERGED:
                verdict = "diverged"
                break
            rep = analyze_convergence(cd, window=window, tol=tol)
            ratio = rep.ratio
            if rep.converged:
                verdict = "converged"
                break
            if len(cd) >= c.max_steps:
                break
        mean = float(np.mean(cd[-window:])) if len(cd) >= window else 0.0
        results.append(Result(c.id, verdict, len(cd), mean, float(ratio), 0.0, t_adm, clock() - t0,
                              _cells(c), footprint(c, hist_capacity)))
        del s
    if stats is not None:
        stats["setup_s"] = setup_s
        stats["wall_s"] = clock() - t0
    return results


def trace(n: int, seed: int = 0, rate: float = 1.0, frac_2d: float = 0.7, nx2=(256, 1024), nx3=(96, 320),
          size_frac=(0.04, 0.12), re=(50.0, 500.0), collisions=("bgk", "trt", "mrt"), les_above_re: float = 200.0,
          precision: str = "fp32", max_steps: int = 50000, tau_min: float = 0.51, u0_max: float = 0.1,
          step2: int = 64, step3: int = 32) -> List[Case]:
    """A seeded request trace: Poisson arrivals at `rate` per second; 2D
    (ny = nx/2) or 3D (ny = nz = nx/2) lattices, geometry sized a fraction
    of ny, Re log-uniform, collision drawn uniformly, Smagorinsky above
    `les_above_re`, u0 = max(0.05, the smallest value giving tau >= tau_min),
    capped at u0_max (Re is then lowered to keep tau >= tau_min).  Arrival
    times come from a stream of their own, so the cases of a trace do not
    depend on `rate`."""
    rng, arrivals = (np.random.default_rng(s) for s in np.random.SeedSequence(seed).spawn(2))
    t = 0.0
    out = []
    for k in range(n):
        t += float(arrivals.exponential(1.0 / rate)) if rate > 0 else 0.0
        dims = 2 if rng.random() < frac_2d else 3
        lo, hi = (nx2 if dims == 2 else nx3)
        step = step2 if dims == 2 else step3
        nx = int(rng.integers(lo // step, hi // step + 1)) * step
        ny = nx // 2
        nz = ny if dims == 3 else 1
        shape = (["cylinder", "rectangle"] if dims == 2 else ["sphere", "box"])[int(rng.integers(0, 2))]
        size = max(2.0, round(float(rng.uniform(*size_frac)) * ny / 2.0))
        Re = float(np.exp(rng.uniform(np.log(re[0]), np.log(re[1]))))
        D = 2.0 * size
        u0 = max(0.05, (tau_min - 0.5) * Re / (3.0 * D))
        if u0 > u0_max:
            u0 = u0_max
            Re = min(Re, 3.0 * u0 * D / (tau_min - 0.5))
        coll = collisions[int(rng.integers(0, len(collisions)))]
        out.append(Case(id=k, dims=dims, nx=nx, ny=ny, nz=nz, shape=shape, size=size, Re=Re, u0=u0,
                        collision=coll, les=Re > les_above_re, precision=precision, arrival=t,
                        max_steps=max_steps))
    return out


def summarize(results: List[Result], wall_s: float) -> dict:
    done = [r for r in results if r.status != "rejected"]
    lat = np.array([r.latency for r in done]) if done else np.zeros(1)
    return {
        "solves": len(done),
        "solves_per_s": len(done) / wall_s if wall_s > 0 else 0.0,
        "p50_latency_s": float(np.percentile(lat, 50)),
        "p99_latency_s": float(np.percentile(lat, 99)),
        "status": {k: sum(1 for r in results if r.status == k)
                   for k in ("converged", "max_steps", "diverged", "rejected", "cancelled")},
    }


def case_dict(c: Case) -> dict:
    return asdict(c)
