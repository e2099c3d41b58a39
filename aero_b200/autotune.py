"""Per-lattice choice of the step kernel by measurement.

The engine has several step kernels that compute the same update: the
per-cell-gather kernel with blocks of 128x1, 256x1 or 32x4 cells, the
row-tiled kernel that stages source rows in shared memory with bulk async
copies (where a lattice's rows fit it), the D3Q19 kernel that takes two
cells per thread on the packed FP32 instructions, and, for 16-bit storage,
the D3Q19 kernel that takes four cells per thread with one 8-byte load per
direction, and, for BGK / TRT with LES, the D3Q19 kernel that computes the
LES rate from a shared-memory velocity stencil instead of a moments pass.  Which is fastest depends on the
lattice's shape and storage format (short rows leave threads of wide blocks
idle; the tiled kernel pays per-tile overhead).  ``autotune`` times each one
on the lattice itself with CUDA events, keeps the fastest and puts the
lattice back in the state it had, so the run continues exactly as if no
steps had been taken.  It runs before the first step.  No counterpart in the
reference, which has a single CPU code path.
"""

from __future__ import annotations

from typing import Dict

import numpy as np

from ._lib import AeroError

KERNELS = {0: "per-cell gather, 128x1 blocks", 1: "per-cell gather, 256x1 blocks",
           2: "per-cell gather, 32x4 blocks", 3: "row-tiled, bulk async copies",
           4: "two cells per thread, packed FP32 arithmetic",
           5: "four cells per thread, 8-byte loads realigned by warp shuffles (16-bit storage)",
           6: "LES velocity stencil staged in shared memory, no moments pass (BGK/TRT + LES)"}


def autotune(solver, steps: int = 20, warmup: int = 2) -> Dict:
    """Times every step kernel on `solver` and selects the fastest.

    Returns {"kernel": id, "name": ..., "ms_per_step": {id: ms}}.  Requires
    step_count == 0: the state, the step counter, the force history and the
    synthetic-inflow fields all restart from where they were."""
    import torch
    if solver.step_count != 0:
        raise ValueError("autotune runs before the first step (step_count must be 0)")
    eng = solver._engine
    solver._flush_host_state()
    f, prev, g = eng.get_state_device()
    times: Dict[int, float] = {}
    inflow = getattr(solver, "_inflow", None)
    ring = solver._params.inflow_ring if inflow is not None else None
    n_total = warmup + steps
    for k in KERNELS:
        try:
            eng.set_step_kernel(k)
        except AeroError:
            continue  # e.g. rows that do not fit the tiled kernel
        eng.set_state(f, prev, g, 0)
        if inflow is not None:
            plane = int(np.prod(solver.solid.shape[:-1]))  # nz * ny (3D) or ny (2D)
            comps = 3 if solver._params.inflow_field == 2 else solver.dims - 1
            zeros = np.zeros((min(n_total, ring), comps, plane))
        done = 0
        ms = None
        stream = torch.cuda.current_stream(eng.device)
        while done < n_total:
            n = warmup if done == 0 else steps
            if inflow is not None:
                n = min(n, ring)
                eng.set_inflow(zeros[:n], done)
            if done == warmup:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                eng.step(n)
                e1.record(stream)
                torch.cuda.synchronize(eng.device)
                ms = e0.elapsed_time(e1) / n
            else:
                eng.step(n)
            eng.read_forces()
            done += n
        times[k] = ms
    best = min(times, key=times.get)
    eng.set_step_kernel(best)
    eng.set_state(f, prev, g, 0)
    return {"kernel": best, "name": KERNELS[best], "ms_per_step": times}
