#!/usr/bin/env python
"""Headline benchmark: D3Q19 lattice updates per second (MLUPS) on B200.

Workload (default, ``--workload sphere512``): the 3D sphere wind tunnel of
the Aero reference, D3Q19 MRT collision + Smagorinsky LES (Cs 0.1) + Bouzidi
bounce-back on a 512x256x256 lattice (33.5 M cells), sphere radius 16 at
(96, 128, 128), u0 = 0.05, nu = 0.0016 (tau 0.5048), free-slip y walls,
periodic z, Zou-He inlet, convective outlet, sponge over the last 32 planes,
initial velocity with a seeded +-1 % uniform perturbation.  Populations are
stored in FP32 (``--precision``).  A "step" is one full solver step: the fused
stream/BC/collide kernel plus the momentum-exchange force reduction.

One JSON line on stdout (rank 0):
  value   : whole-job MLUPS from CUDA events around K steps run as the
            engine runs them (CUDA graphs), state resident in HBM (two 2.5 GB
            population buffers, larger than L2, so no flush is needed), max
            over ranks;
  e2e     : MLUPS through the public API, Solver3D.run(K), timed on the host,
            including the upload of the initial state from pinned host memory
            and the read-back of forces, stability plane and final fields;
  roofline: the fused step kernel's algorithmic bytes per launch
            (2 Q bytes-per-population + 1 flag byte per cell, plus the scalar
            lattice, and the 12-byte LES velocity side output where the LES
            rate is read from one) over its average CUDA-event duration,
            measured over a separate phase of 1000 steps (the sustained rate,
            whatever K is) with events around each kernel, against the
            measured HBM copy rate;
  clocks  : NVML samples (every ~2 ms) inside the K timed steps and the
            1000-step kernel phase;
  precision_variants: the same workload, K and W in the other storage
            formats (FP16 / BF16 deviations), with their kernel roofline;
  cpu_baseline: the FP64 oracle (C/OpenMP restatement of the reference step)
            on a bounded slab of the same workload, on this host's cores.

``--workload box256`` adds ``scalar_check``: the thermal channel in every
storage format against the FP64 engine at a stable relaxation time (Nusselt
numbers, mass and scalar totals, velocity).

``--impl reference`` times that CPU path alone (rank 0; other ranks exit).
Multi-GPU (torchrun): every rank advances its own replica (no exchange);
``scaling`` is "weak".
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "sphere512": dict(
        dims=3, nx=512, ny=256, nz=256, shape=("sphere", 16.0, 96 / 512, 0.5, 0.5),
        kwargs=dict(collision="mrt", les=True, les_cs=0.1, bouzidi=True, wall_bc="slip",
                    inlet_bc="velocity", outlet_bc="convective", streamwise_bc="open",
                    sponge_thickness=32, sponge_strength=0.1),
        u0=0.05, nu=0.0016, perturb=0.01,
        desc="D3Q19 MRT+Smagorinsky(0.1)+Bouzidi sphere r16, 512x256x256, slip walls, sponge 32"),
    "sphere256": dict(
        dims=3, nx=256, ny=128, nz=128, shape=("sphere", 8.0, 48 / 256, 0.5, 0.5),
        kwargs=dict(collision="mrt", les=True, les_cs=0.1, bouzidi=True, wall_bc="slip",
                    inlet_bc="velocity", outlet_bc="convective", streamwise_bc="open",
                    sponge_thickness=16, sponge_strength=0.1),
        u0=0.05, nu=0.0016, perturb=0.01,
        desc="half-size sphere512 (256x128x128, r8), for profiling captures"),
    "channel400": dict(
        dims=2, nx=400, ny=200, nz=1, shape=("cylinder", 20.0, 0.25, 0.5),
        kwargs=dict(collision="bgk", wall_bc="noslip", outlet_bc="zerogradient", inlet_bc="velocity"),
        u0=0.05, nu=0.02, perturb=0.0, perturb_uy=1e-4,
        desc="D2Q9 BGK cylinder channel 400x200, r20 at (100,100), Re 100 (tau 0.56), no-slip walls, "
             "zero-gradient outlet, uy seeded +-1e-4"),
    "box256": dict(
        dims=3, nx=256, ny=128, nz=128, shape=("box", 24.0, 24.0, 128.0, 76 / 256, 12 / 128, 0.5),
        kwargs=dict(collision="trt", trt_lambda=3 / 16, les=True, les_model="wale", les_cs=0.5,
                    wall_bc="noslip", streamwise_bc="periodic", body_force_x=1e-6, thermal=True,
                    T_hot=1.0, T_cold=0.0, alpha_T=0.01, buoyancy=True, g_gravity=1e-5, beta=1.0,
                    T_ref=0.5, scalar_lattice="reduced"),
        u0=0.05, nu=0.01, perturb=0.0, T_noise=1e-3,
        desc="D3Q19 TRT+WALE thermal channel 256x128x128, D3Q7 scalar, box obstacle, body force"),
}

PEAK_FALLBACK_GBS = 6650.0


def _rank_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """The largest x over all ranks (x itself without a process group)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_mlups(cells_per_rank: int, world: int, steps: int, seconds: float) -> float:
    """Cell updates of all replicas per second, in millions."""
    return cells_per_rank * world * steps / seconds / 1e6


def _peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK_GBS, "fallback"


def _geometry(w):
    from aero_b200 import Box, Cylinder, Sphere
    s = w["shape"]
    if s[0] == "cylinder":
        return Cylinder(radius=s[1], cx_frac=s[2], cy_frac=s[3])
    if s[0] == "sphere":
        g = Sphere(radius=s[1], cx_frac=s[2], cy_frac=s[3], cz_frac=s[4])
    else:
        g = Box(width=s[1], height=s[2], depth=s[3], cx_frac=s[4], cy_frac=s[5], cz_frac=s[6])
    return g


class ClockSampler:
    """Samples the SM clock, power draw and clock-event reasons of the bench
    GPU through NVML (read-only queries) every ~2 ms from a helper thread.
    Each sample carries its host time, so the summary can be restricted to
    the windows the caller timed (the K timed steps, the event-timed kernel
    phase); nvidia-smi polling is the fallback when NVML is unavailable."""

    REASON_BITS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
                   "hw_power_brake_slowdown": 0x80, "sw_power_cap": 0x4}

    def __init__(self, device, period_s: float = 0.002):
        self.device = device
        self.period = period_s
        self.samples = []  # (host time, sm MHz, max sm MHz, watts, reason bits)
        self._stop = threading.Event()
        self._h = None
        self._nvml = None
        self.windows = []

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        self._nvml = pynvml
        uuid = str(torch.cuda.get_device_properties(self.device).uuid)
        for cand in (uuid, "GPU-" + uuid):
            try:
                return pynvml.nvmlDeviceGetHandleByUUID(cand)
            except Exception:
                pass
        for k in range(pynvml.nvmlDeviceGetCount()):
            h = pynvml.nvmlDeviceGetHandleByIndex(k)
            u = pynvml.nvmlDeviceGetUUID(h)
            u = u.decode() if isinstance(u, bytes) else u
            if u.endswith(uuid):
                return h
        raise RuntimeError("GPU not found through NVML")

    def __enter__(self):
        try:
            self._h = self._handle()
            self._max = float(self._nvml.nvmlDeviceGetMaxClockInfo(self._h, self._nvml.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, daemon=True)
        except Exception:
            self._h = None
            self.t = threading.Thread(target=self._poll_smi, daemon=True)
        self.t.start()
        return self

    def _poll(self):
        nv, h = self._nvml, self._h
        while not self._stop.is_set():
            t = time.perf_counter()
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                w = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                bits = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.samples.append((t, mhz, self._max, w, bits))
            except Exception:
                pass
            self._stop.wait(self.period)

    def _poll_smi(self):
        fields = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_power_cap")
        try:
            idx = self.device.index if hasattr(self.device, "index") else int(self.device)
            proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={fields}", "--format=csv,noheader,nounits",
                                     "-lms", "100", "-i", str(idx)], stdout=subprocess.PIPE,
                                    stderr=subprocess.DEVNULL, text=True)
        except Exception:
            return
        bits_of = [0x8, 0x20, 0x40, 0x4]
        for line in proc.stdout:
            if self._stop.is_set():
                break
            parts = [p.strip() for p in line.split(",")]
            try:
                bits = sum(b for b, v in zip(bits_of, parts[3:7]) if v.lower() in ("active", "1"))
                self.samples.append((time.perf_counter(), float(parts[0]), float(parts[1]),
                                     float(parts[2]), bits))
            except (ValueError, IndexError):
                continue
        proc.terminate()

    def window(self, t0: float, t1: float) -> None:
        """Marks [t0, t1] (perf_counter seconds) as a region under load."""
        self.windows.append((t0, t1))

    def __exit__(self, *exc):
        self._stop.set()
        self.t.join(timeout=5)

    def summary(self):
        inside = [s for s in self.samples if any(a <= s[0] <= b for a, b in self.windows)] \
            if self.windows else list(self.samples)
        reasons = sorted(n for n, b in self.REASON_BITS.items() if any(s[4] & b for s in inside))
        mhz = [s[1] for s in inside]
        return {"sm_mhz": statistics.median(mhz) if mhz else None,
                "sm_max_mhz": inside[0][2] if inside else None,
                "reasons": reasons, "samples": len(inside),
                "power_w_max": max(s[3] for s in inside) if inside else None,
                "source": "nvml" if self._h is not None else "nvidia-smi",
                "windows_s": [round(b - a, 4) for a, b in self.windows]}


def cpu_oracle_sample(w, target_s=15.0, max_steps=None, nz_sample=32, threads=None):
    """Times the FP64 oracle on a slab (nz_sample planes) of the workload."""
    import numpy as np
    from oracle.oracle import OracleSolver
    threads = threads or len(os.sched_getaffinity(0))
    os.environ["OMP_NUM_THREADS"] = str(threads)
    g = _geometry(w)
    nz = min(nz_sample, w["nz"])
    shp = (w["ny"], w["nx"]) if w["dims"] == 2 else (nz, w["ny"], w["nx"])
    solid = g.mark_solid(*shp)
    phi = g.sdf_field(*shp)
    D = g.reference_length()
    omega = 1.0 / (3.0 * w["nu"] + 0.5)
    kw = dict(w["kwargs"])
    kw.pop("scalar_lattice", None)
    o = OracleSolver(solid=solid, omega=omega, u0=w["u0"], D=D, phi=phi, threads=threads, **kw)
    o.step()  # warm-up (page-in, OpenMP start)
    cells = solid.size
    if max_steps is None:
        max_steps = max(50, int(2e8 // cells))
    t0 = time.perf_counter()
    n = 0
    while n < max_steps:
        o.step()
        n += 1
        if time.perf_counter() - t0 >= target_s:
            break
    dt = time.perf_counter() - t0
    return {"value": cells * n / dt / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": f"{n} FP64 oracle steps of a {w['nx']}x{w['ny']}x{nz} slab of the workload "
                      f"({cells} cells, same physics options), {dt:.1f} s"
            if w["dims"] == 3 else f"{n} FP64 oracle steps of the whole {w['nx']}x{w['ny']} workload, "
                                   f"{dt:.1f} s"}


def run_reference(args, w):
    rank, world, _ = _rank_env()
    if rank != 0:
        return 0
    import numpy as np
    from oracle.oracle import OracleSolver
    threads = len(os.sched_getaffinity(0))
    os.environ["OMP_NUM_THREADS"] = str(threads)
    g = _geometry(w)
    # each step is a bounded sample: a slab sized so that W + K steps stay near a minute
    nz = 16 if args.steps <= 20 else 4
    shp = (w["ny"], w["nx"]) if w["dims"] == 2 else (nz, w["ny"], w["nx"])
    solid = g.mark_solid(*shp)
    phi = g.sdf_field(*shp)
    kw = dict(w["kwargs"])
    kw.pop("scalar_lattice", None)
    o = OracleSolver(solid=solid, omega=1.0 / (3.0 * w["nu"] + 0.5), u0=w["u0"],
                     D=g.reference_length(), phi=phi, threads=threads, **kw)
    for _ in range(args.warmup):
        o.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step()
    dt = time.perf_counter() - t0
    v = solid.size * args.steps / dt / 1e6
    sample = (f"each step: FP64 oracle step of a {w['nx']}x{w['ny']}x{nz} slab of the workload "
              f"({solid.size} cells), {args.steps} steps in {dt:.1f} s")
    line = {
        "impl": "reference", "metric": "D2Q9 MLUPS" if w["dims"] == 2 else "D3Q19 MLUPS", "value": v,
        "unit": "MLUPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "sample_cells": solid.size},
        "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# Batched workloads: a sweep of many cases in one batch, and a served trace
# ----------------------------------------------------------------------------
def sweep_cases(seed=96, precision="fp32"):
    """The 96-case sweep: 64 D2Q9 cases (nx 256..1024 step 64, ny = nx/2,
    cylinder or rectangle, radius / half-width 8..32, Re 40..200) and 32
    D3Q19 spheres (nx 96..256 step 32, ny = nz = nx/2, radius 6..16, Re
    50..300), TRT, u0 = max(0.05, the value giving tau >= 0.51), seeded."""
    import numpy as np
    from aero_b200.serve import Case
    rng = np.random.default_rng(seed)
    cases = []
    for k in range(96):
        if k < 64:
            dims, nx = 2, int(rng.integers(4, 17)) * 64
            shape = "cylinder" if rng.random() < 0.5 else "rectangle"
            size, Re = float(rng.integers(8, 33)), float(rng.uniform(40, 200))
        else:
            dims, nx = 3, int(rng.integers(3, 9)) * 32
            shape, size, Re = "sphere", float(rng.integers(6, 17)), float(rng.uniform(50, 300))
        ny = nx // 2
        size = min(size, ny / 4)
        u0 = min(max(0.05, 0.01 * Re / (3.0 * 2.0 * size)), 0.1)
        cases.append(Case(id=k, dims=dims, nx=nx, ny=ny, nz=ny if dims == 3 else 1, shape=shape, size=size,
                          Re=Re, u0=u0, collision="trt", precision=precision))
    return cases


def _bench_line(metric, value, unit, args, ms_per_step, dtype, config, **extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic", "config": config}
    line.update(extra)
    return line


def run_batch96(args):
    """All 96 sweep cases advance together in one batch for --steps steps
    (timed with CUDA events, state resident); then each case alone through
    the plain API for a bounded sample of steps, whose per-case rate gives
    the time the same sweep takes as sequential plain solves."""
    import torch
    from aero_b200 import Batch
    from aero_b200.serve import make_solver
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cases = sweep_cases(precision=args.precision)[::max(args.batch_every, 1)]
    t0 = time.perf_counter()
    solvers = [make_solver(c, dev) for c in cases]
    setup_s = time.perf_counter() - t0
    cells = [c.nx * c.ny * c.nz for c in cases]
    b = Batch(max_members=len(solvers), device=dev)
    for s in solvers:
        b.add(s)
    b.step(max(args.warmup, 3))
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        e0.record(stream)
        b.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    conv = b.converge(min(args.steps, 1000), 1e-3)
    diverged = int(sum(1 for r in conv if int(r[5]) & 1))
    for s in list(b.members):
        b.remove(s)
    b.close()
    # sequential plain solves: each case alone, its rate measured on a bounded sample
    sample = min(200, args.steps)
    seq_s = 0.0
    per_case = []
    for s, n in zip(solvers, cells):
        s.run(10, check_every=11, verbose=False)
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        s.run(sample, check_every=sample + 1, verbose=False)
        torch.cuda.synchronize(dev)
        dt = (time.perf_counter() - t1) / sample
        per_case.append(n / dt / 1e6)
        seq_s += dt * args.steps
    total = sum(cells)
    mlups = total * args.steps / (ms / 1e3) / 1e6
    batch_s = ms / 1e3
    line = _bench_line(
        "batched sweep MLUPS", mlups, "MLUPS", args, ms / args.steps,
        {"fp32": "f32", "fp64": "f64", "fp16s": "f16 storage / f32 compute",
         "bf16s": "bf16 storage / f32 compute"}[args.precision],
        {"workload": "batch96", "cases": len(cases), "every": args.batch_every, "cells_per_step": total,
         "precision": args.precision,
         "desc": "64 D2Q9 (nx 256..1024) + 32 D3Q19 spheres (nx 96..256), TRT, one batch"},
        gpu_launches=None,
        batch={"solves_per_s": len(cases) / batch_s, "seconds": batch_s, "setup_s": setup_s,
               "diverged_members": diverged},
        sequential_plain={"solves_per_s": len(cases) / seq_s, "seconds_estimated": seq_s,
                          "sample_steps_per_case": sample,
                          "median_case_mlups": float(sorted(per_case)[len(per_case) // 2])},
        speedup_vs_sequential=seq_s / batch_s,
        clocks=clk.summary())
    print(json.dumps(line), flush=True)
    return 0


def run_serve(args):
    """A served trace: seeded requests with Poisson arrivals at 80% of the
    capacity measured on the same trace with every request queued at t = 0;
    requests run until the drag converges (window, tolerance) or their step
    limit; then the same requests as sequential plain solves."""
    import numpy as np
    import torch
    from aero_b200 import serve
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    kw = dict(chunk=args.serve_chunk, window=args.serve_window, tol=args.serve_tol)
    nx2 = tuple(int(v) for v in args.serve_nx2.split(","))
    nx3 = tuple(int(v) for v in args.serve_nx3.split(","))
    mk = dict(n=args.serve_requests, seed=5, nx2=nx2, nx3=nx3, max_steps=args.steps,
              precision=args.precision, tau_min=args.serve_tau_min)
    # capacity: the whole trace queued at once
    cal = serve.trace(rate=0.0, **mk)
    srv = serve.Server(hbm_cap=args.serve_hbm_gb * 1e9, max_members=256, device=dev, **kw)
    res_cal = srv.run(cal)
    cap = len([r for r in res_cal if r.status != "rejected"]) / srv.stats["wall_s"]
    srv.close()
    # the served trace at 80% of capacity
    cases = serve.trace(rate=0.8 * cap, **mk)
    srv = serve.Server(hbm_cap=args.serve_hbm_gb * 1e9, max_members=256, device=dev, **kw)
    with ClockSampler(dev.index) as clk:
        res = srv.run(cases)
    stats = dict(srv.stats)
    srv.close()
    span = max(r.done for r in res)
    summ = serve.summarize(res, span)
    # sequential plain solves of the same requests (plain FP32 storage)
    plain_cases = serve.trace(rate=0.0, **dict(mk, precision="fp32"))
    t0 = time.perf_counter()
    pstats = {}
    plain = serve.run_plain(plain_cases, device=dev, stats=pstats, **kw)
    torch.cuda.synchronize(dev)
    plain_s = time.perf_counter() - t0
    pmap = {r.id: r for r in plain}

    def rel_dcd(kind):
        return [abs(r.cd_mean - pmap[r.id].cd_mean) / abs(pmap[r.id].cd_mean) for r in res
                if r.status == kind and pmap[r.id].status == kind
                and np.isfinite(pmap[r.id].cd_mean) and pmap[r.id].cd_mean != 0.0]
    dcd_conv, dcd_max = rel_dcd("converged"), rel_dcd("max_steps")
    same_verdict = sum(1 for r in res if pmap[r.id].status == r.status)
    line = _bench_line(
        "served solves/s", summ["solves_per_s"], "solves/s", args, None,
        {"fp32": "f32", "fp64": "f64", "fp16s": "f16 storage / f32 compute",
         "bf16s": "bf16 storage / f32 compute"}[args.precision],
        {"workload": "serve", "requests": len(cases), "arrivals": "Poisson at 0.8 x measured capacity",
         "nx2": list(nx2), "nx3": list(nx3),
         "capacity_solves_per_s": cap, "chunk": args.serve_chunk, "window": args.serve_window,
         "tol": args.serve_tol, "max_steps": args.steps, "hbm_cap_gb": args.serve_hbm_gb,
         "tau_min": args.serve_tau_min,
         "desc": f"70% D2Q9 (nx {nx2[0]}..{nx2[1]}) / 30% D3Q19 (nx {nx3[0]}..{nx3[1]}), "
                 "cylinder/rectangle/sphere/box, Re log-uniform 50..500, BGK/TRT/MRT, Smagorinsky above Re 200"},
        latency={"p50_s": summ["p50_latency_s"], "p99_s": summ["p99_latency_s"]},
        status=summ["status"], aggregate_mlups=stats["cell_steps"] / span / 1e6,
        served_time={"setup_s": stats["setup_s"], "gpu_wait_s": stats["gpu_wait_s"], "rounds": stats["rounds"]},
        sequential_plain={"solves_per_s": len(plain) / plain_s, "seconds": plain_s, "setup_s": pstats["setup_s"],
                          "status": {k: sum(1 for r in plain if r.status == k)
                                     for k in ("converged", "max_steps", "diverged")}},
        speedup_vs_sequential=summ["solves_per_s"] / (len(plain) / plain_s),
        cd_vs_plain={"same_verdict": same_verdict,
                     "converged_compared": len(dcd_conv),
                     "converged_max_rel_diff": max(dcd_conv) if dcd_conv else None,
                     "max_steps_compared": len(dcd_max),
                     "max_steps_max_rel_diff": max(dcd_max) if dcd_max else None},
        clocks=clk.summary())
    print(json.dumps(line), flush=True)
    return 0


def scalar_precision_check(w, args, dev, tau=0.8, steps=2000, formats=("fp32", "bf16s", "fp16s")):
    """The thermal channel (configuration 3) in each storage format against
    the FP64 engine, at a relaxation time where the reference's TRT is stable
    (its lambda semantics diverge at the configuration's tau 0.53): the
    configuration's geometry, body force, scalar and buoyancy, the scalar
    started at T_ref + seeded U(-1e-3, 1e-3), `steps` steps.  Reports per
    format the Nusselt numbers of both Dirichlet rows, the mass and scalar
    totals (FP64 sums on the device) and their relative differences to FP64,
    and the relative L2 difference of u."""
    import numpy as np
    import torch
    wk = dict(w, nu=(tau - 0.5) / 3.0)
    shp = (wk["nz"], wk["ny"], wk["nx"])
    gen = torch.Generator(device=dev)
    gen.manual_seed(4321)
    T0 = wk["kwargs"]["T_ref"] + 1e-3 * (2.0 * torch.rand(shp, generator=gen, device=dev, dtype=torch.float64) - 1.0)
    out = {"tau": tau, "steps": steps, "nu": wk["nu"],
           "desc": "configuration 3 at tau %.2f (stable under the reference's TRT lambda semantics), scalar "
                   "T_ref + U(-1e-3, 1e-3) seed 4321" % tau}
    ref = None
    for prec in ("fp64",) + tuple(formats):
        s = _build_solver(wk, prec, dev, steps, 0)
        s.set_equilibrium_state(T=T0)
        st0 = s.field_statistics()
        t0 = time.perf_counter()
        s._advance(steps)
        torch.cuda.synchronize(dev)
        dt = time.perf_counter() - t0
        st = s.field_statistics()
        u = s._engine.macroscopic_device()[1:].cpu().numpy()
        rec = {"Nu_bottom": st["Nu_bottom"], "Nu_top": st["Nu_top"], "mass": st["mass"],
               "scalar_total": st["scalar_total"], "mass_drift": (st["mass"] - st0["mass"]) / st0["mass"],
               "scalar_drift": (st["scalar_total"] - st0["scalar_total"]) / st0["scalar_total"],
               "status": s.status(), "seconds": dt}
        if ref is None:
            ref = dict(rec, u=u)
        else:
            rec["mass_err_vs_fp64"] = abs(st["mass"] - ref["mass"]) / ref["mass"]
            rec["scalar_err_vs_fp64"] = abs(st["scalar_total"] - ref["scalar_total"]) / ref["scalar_total"]
            rec["Nu_bottom_err_vs_fp64"] = abs(st["Nu_bottom"] - ref["Nu_bottom"]) / abs(ref["Nu_bottom"])
            rec["Nu_top_err_vs_fp64"] = abs(st["Nu_top"] - ref["Nu_top"]) / abs(ref["Nu_top"])
            rec["u_rel_l2_vs_fp64"] = float(np.linalg.norm(u - ref["u"]) / np.linalg.norm(ref["u"]))
        out[prec] = rec
        del s
        torch.cuda.empty_cache()
    out["fp64"].pop("u", None)
    return out


def sphere_precision_check(w, args, dev, tau=0.8, bouzidi=True, steps=6000, window=2000,
                           formats=("fp32", "fp16s", "bf16s")):
    """The sphere configuration in each storage format against the FP64
    engine where the flow is stable.  The configuration's tau 0.5048
    diverges, and so does every tau up to 0.6 with the reference's Bouzidi
    rule (half-way bounce-back is stable at 0.56): the configuration's
    geometry, MRT + Smagorinsky, Bouzidi or half-way bounce-back, slip walls,
    sponge and seeded +-1% inflow perturbation (seed 1234), `steps` steps.
    Reports per format the
    mean Cd and the mean lift coefficients over the last `window` steps and
    their differences to FP64, the centreline wake profile ux(x, ny/2, nz/2)
    behind the sphere (relative L2 to FP64), and the mass (FP64 sum on the
    device) relative to FP64."""
    import numpy as np
    import torch
    wk = dict(w, nu=(tau - 0.5) / 3.0, kwargs=dict(w["kwargs"], bouzidi=bouzidi))
    g = _geometry(wk)
    D = g.reference_length()
    x0 = int(wk["shape"][2] * wk["nx"] + wk["shape"][1]) + 2  # first plane behind the sphere
    out = {"tau": tau, "bouzidi": bouzidi, "steps": steps, "window": window, "nu": wk["nu"],
           "Re": wk["u0"] * D / wk["nu"],
           "desc": "configuration 2 at tau %.2f with %s, seeded +-1%% inflow perturbation"
                   % (tau, "Bouzidi" if bouzidi else "half-way bounce-back")}
    ref = None
    for prec in ("fp64",) + tuple(formats):
        s = _build_solver(wk, prec, dev, steps, 0)
        ux0, uy0, T0 = _initial_fields(wk, dev, 0, s)
        s.set_equilibrium_state(ux=ux0, uy=uy0, T=T0)
        t0 = time.perf_counter()
        c = s._coefficients(s._advance(steps))
        torch.cuda.synchronize(dev)
        dt = time.perf_counter() - t0
        m = s._engine.macroscopic_device()
        wake = m[1, wk["nz"] // 2, wk["ny"] // 2, x0:].cpu().numpy()
        mass = s.field_statistics()["mass"]
        rec = {"Cd_mean": float(np.mean(c["Cd"][-window:])), "Cly_mean": float(np.mean(c["Cly"][-window:])),
               "Clz_mean": float(np.mean(c["Clz"][-window:])), "mass": mass, "status": s.status(),
               "seconds": dt}
        if ref is None:
            ref = dict(rec, wake=wake, Cd=c["Cd"][-window:], Cly=c["Cly"][-window:])
        else:
            rec["Cd_rel_err_vs_fp64"] = abs(rec["Cd_mean"] - ref["Cd_mean"]) / abs(ref["Cd_mean"])
            rec["Cly_mean_abs_err_vs_fp64"] = abs(rec["Cly_mean"] - ref["Cly_mean"])
            rec["Clz_mean_abs_err_vs_fp64"] = abs(rec["Clz_mean"] - ref["Clz_mean"])
            rec["Cd_history_max_rel_err_vs_fp64"] = float(np.max(np.abs(c["Cd"][-window:] - ref["Cd"]))
                                                          / abs(ref["Cd_mean"]))
            rec["wake_rel_l2_vs_fp64"] = float(np.linalg.norm(wake - ref["wake"]) / np.linalg.norm(ref["wake"]))
            rec["mass_err_vs_fp64"] = abs(mass - ref["mass"]) / ref["mass"]
        out[prec] = rec
        del s, m
        torch.cuda.empty_cache()
    return out


ROOFLINE_STEPS = 1000  # event-timed steps of the kernel phase (about a second at sphere512)


def _build_solver(w, precision, dev, steps, warmup, layout="ab"):
    from aero_b200 import Solver, Solver3D
    g = _geometry(w)
    dims = w["dims"]
    nz, ny, nx = w["nz"], w["ny"], w["nx"]
    shp = (ny, nx) if dims == 2 else (nz, ny, nx)
    solid = g.mark_solid(*shp)
    phi = g.sdf_field(*shp) if w["kwargs"].get("bouzidi") else None
    cap = max(4096, steps + warmup + ROOFLINE_STEPS + 8)
    common = dict(solid=solid, omega=1.0 / (3.0 * w["nu"] + 0.5), u0=w["u0"], D=g.reference_length(),
                  phi=phi, precision=precision, device=dev, hist_capacity=cap, layout=layout, **w["kwargs"])
    return Solver(Ny=ny, Nx=nx, **common) if dims == 2 else Solver3D(Nz=nz, Ny=ny, Nx=nx, **common)


def _initial_fields(w, dev, rank, s):
    """The seeded initial fields of the workload (device FP64): ux = u0 (1 +
    p U(-1, 1)) with p the workload's perturbation; uy = U(-a, a) where the
    workload sets a; the scalar T = T_ref + U(-b, b) where it sets b."""
    import torch
    shp = (w["ny"], w["nx"]) if w["dims"] == 2 else (w["nz"], w["ny"], w["nx"])
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    ux = w["u0"] * (1.0 + w["perturb"] * (2.0 * torch.rand(shp, generator=gen, device=dev,
                                                           dtype=torch.float64) - 1.0))
    uy = (w["perturb_uy"] * (2.0 * torch.rand(shp, generator=gen, device=dev, dtype=torch.float64) - 1.0)
          if w.get("perturb_uy") else None)
    T = None
    if s.thermal and w.get("T_noise"):
        gen.manual_seed(4321 + rank)
        T = s.T_ref + w["T_noise"] * (2.0 * torch.rand(shp, generator=gen, device=dev, dtype=torch.float64) - 1.0)
    return ux, uy, T


def _bytes_per_cell(s, precision):
    """Algorithmic bytes of one cell update of the fused step: read and write
    Q populations (2 Q s) and the flag byte, the scalar populations where a
    scalar runs (2 Qg x 4 or 8), and the LES velocity side output the step
    reads back where the BGK/TRT LES rate is computed from it (3 values).
    Returns (bytes, the parts, bytes of the moments pass that are not
    algorithmic: its second read of the populations)."""
    sb = {"fp32": 4, "fp64": 8, "fp16s": 2, "bf16s": 2}[precision]
    rb = 8 if precision == "fp64" else 4
    Q = 9 if s.dims == 2 else 19
    parts = {"populations": 2 * Q * sb, "flags": 1}
    extra = 0
    if s.thermal:
        qg = (5 if s.dims == 2 else 7) if s.scalar_lattice == "reduced" else Q
        parts["scalar"] = 2 * qg * rb
    if s.les and s.collision != "mrt" and not s._engine.les_fused():
        parts["les_side_output"] = 3 * rb
        extra = Q * sb + 3 * rb
    return sum(parts.values()), parts, extra


def measure_lattice(w, precision, args, dev, rank=0, world=1, dist=None, e2e=True, label="main"):
    """One single-lattice measurement: set-up and autotune (untimed), W warm-up
    steps, K steps timed with CUDA events as the engine runs them (graphs),
    then ROOFLINE_STEPS steps with events around each kernel for the step
    kernel's sustained duration, clocks sampled over both; optionally the
    end-to-end run through the public API.  Returns a dict of results."""
    import numpy as np
    import torch
    s = _build_solver(w, precision, dev, args.steps, args.warmup, layout=args.layout)
    eng = s._engine
    ncells = w["nx"] * w["ny"] * w["nz"]
    ux0, uy0, T0 = _initial_fields(w, dev, rank, s)
    eng.set_equilibrium(ux=ux0, uy=uy0, T=T0)
    stream = torch.cuda.current_stream(dev)
    tune = None
    if args.kernel == "auto":
        tune = s.autotune(steps=10)
    elif args.kernel in ("pair", "quad"):
        eng.set_step_kernel(4 if args.kernel == "pair" else 5)
    eng.step(args.warmup)
    eng.read_forces()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        t0 = time.perf_counter()
        e0.record(stream)
        eng.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        clk.window(t0, time.perf_counter())
        if dist:
            dist.barrier()
        ms = e0.elapsed_time(e1)
        raw = eng.read_forces()
        # the step kernel's sustained duration: eager launches with events
        # around each kernel, over ROOFLINE_STEPS steps
        eng.enable_timing(True)
        eng.kernel_times()  # reset
        t1 = time.perf_counter()
        eng.step(ROOFLINE_STEPS)
        step_ms, force_ms, nt = eng.kernel_times()
        clk.window(t1, time.perf_counter())
        eng.enable_timing(False)
    eng.read_forces()
    s.step_count += args.warmup + args.steps + ROOFLINE_STEPS
    status, first_bad = eng.status(), eng.first_bad_step()
    ms = max_over_ranks(ms, dist, dev)
    peak, peak_kind = _peak_hbm()
    bpc, parts, extra = _bytes_per_cell(s, precision)
    k_ms = step_ms / max(nt, 1)
    achieved = bpc * ncells / (k_ms / 1e3) / 1e9
    plan = eng.step_plan()
    plan["kernel_id"] = eng.get_step_kernel()
    plan["les_fused"] = eng.les_fused()
    if tune is not None:
        plan["autotune_ms_per_step"] = {str(k): v for k, v in tune["ms_per_step"].items()}
    kname = "k_step_tiled" if plan["tiled"] else {4: "k_step_pair", 5: "k_step_quad",
                                                  6: "k_step_les"}.get(plan["kernel_id"], "k_step")
    if kname == "k_step" and s.layout == "aa":
        kname = "k_step_aa"
    # DRAM bytes per launch from the committed ncu summary of this kernel,
    # workload and precision (a smaller case scaled by cells where the summary
    # says so); None when no capture covers it
    traffic = None
    pat = re.compile(rf"^- {re.escape(args.workload)}: dram bytes per launch = (\d+)\s*$", re.M)
    others = ("k_step_tiled", "k_step_pair", "k_step_quad", "k_step_les", "k_step_aa", "k_step_batch")
    for md in sorted((ROOT / "profiles").glob(f"{kname}_*_{precision}.md")):
        if any(md.name.startswith(o + "_") for o in others if o != kname and o.startswith(kname)):
            continue  # a summary of another kernel whose name extends this one
        m = pat.search(md.read_text())
        if m:
            traffic = int(m.group(1))
            break
    res = {
        "solver": s, "ms": ms, "value": whole_job_mlups(ncells, world, args.steps, ms / 1e3), "raw": raw,
        "status": status, "first_bad": first_bad, "clocks": clk.summary(),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": traffic,
                     "kernel": f"{kname} (fused stream/BC/collide" + (
                         ", source rows staged in shared memory by bulk async copies)" if plan["tiled"]
                         else ", two cells per thread on packed FP32 arithmetic)" if plan["kernel_id"] == 4
                         else ", four cells per thread, 8-byte loads realigned by warp shuffles)"
                         if plan["kernel_id"] == 5
                         else ", BGK/TRT with the LES velocity stencil in shared memory)" if plan["kernel_id"] == 6
                         else ", per-cell global gather, blocks " + ("128x1", "256x1", "32x4")[plan["kernel_id"]]
                         + ")"),
                     "step_plan": plan, "alg_bytes_per_launch": bpc * ncells, "bytes_per_cell": bpc,
                     "bytes_per_cell_parts": parts, "non_algorithmic_bytes_per_cell": extra,
                     "kernel_ms": k_ms, "kernel_steps_timed": int(nt), "finalize_ms": force_ms / max(nt, 1)},
    }
    res["launches_per_step"] = 2 + (1 if (s.les and s.collision != "mrt" and not eng.les_fused()) else 0)
    # a persistent run takes the timed call's steps in one launch
    res["persistent"] = eng.persistent()
    res["state_bytes"] = 2 * s.Q * ncells * {"fp32": 4, "fp64": 8, "fp16s": 2, "bf16s": 2}[precision]
    if e2e:
        res["e2e"] = _measure_e2e(s, w, args, dev, (ux0, uy0, T0), world, dist)
    del ux0, uy0, T0
    return res


def _measure_e2e(s, w, args, dev, fields, world, dist):
    """MLUPS of Solver.run(K) end to end: the initial fields (ux, and uy / T
    where the workload seeds them) copied from pinned host memory and turned
    into the equilibrium state on the device (set_equilibrium_state), K
    steps, the force history and the result's fields read back, timed on the
    host."""
    import torch
    ncells = w["nx"] * w["ny"] * w["nz"]
    host = [None if a is None else a.cpu().pin_memory() for a in fields]
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    s.step_count = 0
    s._init_histories()
    s.set_equilibrium_state(ux=host[0], uy=host[1], T=host[2])
    t1 = time.perf_counter()
    # one stability check at the end would raise on a diverged state; the
    # throughput measurement does not depend on it, so none is requested
    r = s.run(args.steps, check_every=args.steps + 1, verbose=False)
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    dt = max_over_ranks(t2 - t0, dist, dev)
    h2d = sum(a.numel() * 8 for a in host if a is not None)
    d2h = (args.steps * 12 * 8 + (w["nz"] if w["dims"] == 3 else w["ny"]) * 3 * 8
           + (1 + w["dims"]) * ncells * 8 + (ncells * 8 if s.thermal else 0))
    return {"value": whole_job_mlups(ncells, world, args.steps, dt), "unit": "MLUPS",
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
            "call": f"{type(s).__name__}.set_equilibrium_state(fields from pinned host memory) + run(K)",
            "phases_s": {"initial_state": t1 - t0, "run_with_readback": t2 - t1,
                         "readback": getattr(s, "_last_readback_s", None)},
            "Cd_mean": r["Cd_mean"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="sphere512", choices=sorted(WORKLOADS) + ["batch96", "serve"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16s", "bf16s", "fp64"])
    ap.add_argument("--variants", default="fp16s,bf16s",
                    help="storage formats timed after the main run on the same workload, steps and warm-up "
                         "(comma-separated; 'none' to skip)")
    ap.add_argument("--layout", default="ab", choices=["ab", "aa", "auto"],
                    help="population layout: two buffers (ab), one buffer updated in place (aa), or auto "
                         "(ab when it fits the free device memory, else aa)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-scalar-check", action="store_true", help="box256: skip the storage-format check")
    ap.add_argument("--sphere-check", action="store_true",
                    help="sphere workloads: add the storage formats' Cd / lift / wake / mass against FP64 at a "
                         "stable relaxation time (about a minute at sphere512)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--collision", default=None, choices=["bgk", "trt", "mrt"],
                    help="override the workload's collision operator (profiling)")
    ap.add_argument("--kernel", default="auto", choices=["auto", "rowgather", "tiled", "pair", "quad"],
                    help="step kernel: chosen by the autotuner (default), the per-cell global gather, "
                         "rows staged in shared memory by bulk async copies, two cells per thread "
                         "on packed FP32 arithmetic, or four cells per thread (16-bit storage)")
    ap.add_argument("--batch-every", type=int, default=1,
                    help="batch96: keep every k-th case (a smaller batch for profiling captures)")
    ap.add_argument("--serve-requests", type=int, default=128)
    ap.add_argument("--serve-chunk", type=int, default=250)
    ap.add_argument("--serve-window", type=int, default=1000)
    ap.add_argument("--serve-tol", type=float, default=1e-3)
    ap.add_argument("--serve-hbm-gb", type=float, default=150.0)
    ap.add_argument("--serve-nx2", default="256,512",
                    help="nx range of the 2D requests (the configuration's trace: 256,1024)")
    ap.add_argument("--serve-nx3", default="96,160",
                    help="nx range of the 3D requests (the configuration's trace: 96,320)")
    ap.add_argument("--serve-tau-min", type=float, default=0.51,
                    help="smallest relaxation time of a request (u0 raised, then Re lowered, to reach it)")
    args = ap.parse_args()
    if args.workload == "batch96":
        return run_batch96(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.kernel == "tiled":
        os.environ["AERO_B200_TILES"] = "1"
    else:
        os.environ.pop("AERO_B200_TILES", None)
    w = dict(WORKLOADS[args.workload])
    if args.collision:
        w["kwargs"] = dict(w["kwargs"], collision=args.collision)
    if args.impl == "reference":
        return run_reference(args, w)
    args.warmup = max(args.warmup, 3)

    import numpy as np
    import torch
    rank, world, local = _rank_env()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)
    ncells = w["nx"] * w["ny"] * w["nz"]
    dims = w["dims"]

    m = measure_lattice(w, args.precision, args, dev, rank, world, dist, e2e=not args.no_e2e)
    s = m.pop("solver")
    layout = s.layout
    Cd_last = float(m["raw"][-1, 0] / s._drag_norm()) if len(m["raw"]) else 0.0
    links = int(len(s.surface_links))
    extra = {}
    if args.workload == "box256" and not args.no_scalar_check:
        extra["scalar_check"] = scalar_precision_check(w, args, dev)
    if args.sphere_check and args.workload in ("sphere512", "sphere256"):
        extra["sphere_check"] = [sphere_precision_check(w, args, dev, tau=0.8, bouzidi=True),
                                 sphere_precision_check(w, args, dev, tau=0.56, bouzidi=False)]
    del s
    torch.cuda.empty_cache()

    # the same workload, steps and warm-up in the other storage formats
    variants = {}
    if args.variants and args.variants != "none":
        for prec in [v for v in args.variants.split(",") if v and v != args.precision]:
            v = measure_lattice(w, prec, args, dev, rank, world, dist, e2e=False, label=prec)
            v.pop("solver")
            variants[prec] = {"value": v["value"], "unit": "MLUPS", "ms_per_step": v["ms"] / args.steps,
                              "speedup_vs_main": v["value"] / m["value"],
                              "kernel_ms": v["roofline"]["kernel_ms"],
                              "bytes_per_cell": v["roofline"]["bytes_per_cell"],
                              "achieved_gbs": v["roofline"]["achieved"], "frac": v["roofline"]["frac"],
                              "kernel": v["roofline"]["kernel"], "clocks": v["clocks"],
                              "status": v["status"], "first_nonfinite_step": v["first_bad"]}
            del v
            torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_oracle_sample(w)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": "D2Q9 MLUPS" if dims == 2 else "D3Q19 MLUPS", "value": m["value"], "unit": "MLUPS",
        "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp32": "f32", "fp64": "f64", "fp16s": "f16 storage / f32 compute",
                  "bf16s": "bf16 storage / f32 compute"}[args.precision],
        "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "cells": ncells,
                   "precision": args.precision, "layout": layout, "parallelism": f"replicas x{world}",
                   "l2": ("state (2 x Q x cells) far larger than L2; no flush needed" if m["state_bytes"] > 126e6
                          else "state (%.1f MB) fits in L2 and stays there between steps, as in the solver's own "
                               "runs; no flush" % (m["state_bytes"] / 1e6)),
                   "links": links},
        # per step: k_step, k_finalize (+ the LES moments pass where it runs);
        # per aero_step call: one launch recording the step whose profile is summed
        # the profile-step setter plus the step launches (one persistent launch per call)
        "gpu_launches": 2 if m["persistent"] else m["launches_per_step"] * args.steps + 1,
        "roofline": m["roofline"],
        "clocks": m["clocks"],
        "e2e": m.get("e2e"),
        "cpu_baseline": cpu,
        "precision_variants": variants,
        "status": m["status"],
        "first_nonfinite_step": m["first_bad"],
        "Cd_last": Cd_last,
    }
    line.update(extra)
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
