"""Many solvers advanced together on one GPU.

A Batch steps all its member solvers (``Solver`` / ``Solver3D`` with
backend "b200", any mix of 2D and 3D, sizes, geometries, collision models
and storage formats) with one launch per lattice class and step kernel,
replayed as CUDA graphs (``aero_batch_*`` in the C ABI).  Members join and
leave between steps, so a serving loop can admit new cases while others
run (continuous batching).  While a member, a solver is advanced only by
the batch; its force history on the device is a rolling window, and the
batch can evaluate the reference's drag-convergence rule
(``analyze_convergence``, aero/diagnostics.py:87-120) for every member on
the device.

There is no counterpart in the reference, which advances one Solver at a
time from Python (aero/lbm/solver.py:517-570).
"""

from __future__ import annotations

import ctypes
from typing import List

import numpy as np

from . import _lib
from ._lib import check

CONVERGE_FIELDS = ("ratio", "mean_abs", "std", "converged", "steps", "status", "mean")


class Batch:
    """A set of solvers on one device that advance together."""

    def __init__(self, max_members: int = 256, device=None):
        import torch
        from .engine import _require_cuda
        self.torch = torch
        self.lib = _lib.load()
        self.device = _require_cuda(device)
        h = ctypes.c_void_p()
        check("aero_batch_create", self.lib.aero_batch_create(int(max_members), ctypes.byref(h)))
        self.h = h
        nbytes = ctypes.c_uint64()
        check("aero_batch_workspace_size", self.lib.aero_batch_workspace_size(h, ctypes.byref(nbytes)))
        with torch.cuda.device(self.device):
            self.workspace = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        check("aero_batch_bind_workspace", self.lib.aero_batch_bind_workspace(
            h, self.workspace.data_ptr(), int(nbytes.value)))
        self.members: List = []

    def _stream(self):
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def add(self, solver) -> None:
        """Adds a solver (its pending host-side state edits are uploaded first)."""
        if solver._engine.device != self.device:
            raise ValueError(f"solver is on {solver._engine.device}, the batch on {self.device}")
        solver._flush_host_state()
        check("aero_batch_add", self.lib.aero_batch_add(self.h, solver._engine.h, float(solver._drag_norm())))
        self.members.append(solver)

    def remove(self, solver) -> None:
        check("aero_batch_remove", self.lib.aero_batch_remove(self.h, solver._engine.h))
        self.members.remove(solver)

    def __len__(self) -> int:
        return len(self.members)

    def step(self, n: int) -> None:
        """Advances every member n steps (asynchronous on the current stream,
        except that members with synthetic inflow or an SEM inlet have their
        fields uploaded before each chunk of at most their ring's steps, which
        waits for the stream as Solver.run's upload does)."""
        for s in self.members:
            s._flush_host_state()  # raises if a member's state was edited on the host
        inflow = [s for s in self.members if getattr(s, "_inflow", None) is not None]
        chunk = min([s._params.inflow_ring for s in inflow], default=int(n)) or int(n)
        left = int(n)
        while left > 0:
            k = min(left, chunk)
            with self.torch.cuda.device(self.device):
                for s in inflow:
                    s._engine.set_inflow(s._inflow.fields(k), s.step_count)
                check("aero_batch_step", self.lib.aero_batch_step(self.h, k, self._stream()))
            for s in self.members:
                s.step_count += k
            left -= k

    def converge(self, window: int, tol: float) -> np.ndarray:
        """(members, 7) array, join order: ratio, mean|Cd|, std, converged,
        steps, status word, mean Cd (CONVERGE_FIELDS)."""
        out = np.zeros((max(len(self.members), 1), len(CONVERGE_FIELDS)), dtype=np.float64)
        with self.torch.cuda.device(self.device):
            check("aero_batch_converge", self.lib.aero_batch_converge(
                self.h, int(window), float(tol), out.ctypes.data, self._stream()))
        return out[: len(self.members)]

    def close(self) -> None:
        h = getattr(self, "h", None)
        if h is not None and h.value:
            self.lib.aero_batch_destroy(h)
            self.h = None
        self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
