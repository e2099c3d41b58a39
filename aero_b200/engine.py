"""One lattice on one GPU: the C-ABI handle plus its torch-owned workspace.

PyTorch provides the device memory (a single uint8 workspace tensor and the
FP64 staging tensors for state I/O) and the CUDA stream; all arithmetic on
the lattice runs in the sm_100a kernels of libaero_b200.so.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from ._lib import AeroParams, check

FORCE_VALUES = _lib.FORCE_VALUES

# Device-to-host copies of large results (run()'s rho / u fields, the state)
# go through two pinned bounce buffers of this many bytes: the copy engine
# fills one at PCIe / C2C rate while the host threads copy the other into the
# caller's array, instead of the driver's staged copy into pageable memory.
READBACK_CHUNK = 32 << 20
_bounce = []


def _bounce_buffers():
    """The process's two pinned bounce buffers, allocated on first use (a
    lattice whose results need them allocates them at set-up)."""
    import torch
    if not _bounce:
        _bounce.extend(torch.empty(READBACK_CHUNK, dtype=torch.uint8, pin_memory=True) for _ in range(2))
    return _bounce


def copy_to_host(src, out: Optional[np.ndarray] = None) -> np.ndarray:
    """Contiguous CUDA tensor -> host numpy array of the same dtype and shape
    (`out`, C-contiguous, or a new one).  Results above one bounce buffer are
    copied chunk by chunk on the tensor's current stream, the device-to-host
    copy of one chunk overlapping the host copy of the previous one."""
    import torch
    src = src.contiguous()
    if out is None:
        out = np.empty(tuple(src.shape), dtype=torch.empty((), dtype=src.dtype).numpy().dtype)
    dst = torch.from_numpy(out).reshape(-1).view(torch.uint8)
    flat = src.reshape(-1).view(torch.uint8)
    n = flat.numel()
    if n != dst.numel():
        raise ValueError("copy_to_host: size mismatch")
    if n <= READBACK_CHUNK:
        dst.copy_(flat)
        return out
    ring = _bounce_buffers()
    stream = torch.cuda.current_stream(src.device)
    done = [torch.cuda.Event(), torch.cuda.Event()]
    pending = None
    with torch.cuda.device(src.device):
        for k, off in enumerate(range(0, n, READBACK_CHUNK)):
            m = min(READBACK_CHUNK, n - off)
            # ring[k & 1] was last read by the host copy of chunk k - 2,
            # which finished in the previous iteration
            ring[k & 1][:m].copy_(flat[off:off + m], non_blocking=True)
            done[k & 1].record(stream)
            if pending is not None:
                pk, poff, pm = pending
                done[pk & 1].synchronize()
                dst[poff:poff + pm].copy_(ring[pk & 1][:pm])
            pending = (k, off, m)
        pk, poff, pm = pending
        done[pk & 1].synchronize()
        dst[poff:poff + pm].copy_(ring[pk & 1][:pm])
    return out


def _require_cuda(device):
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("aero_b200 needs a CUDA GPU (sm_100a); none is visible")
    dev = torch.device(device if device is not None else "cuda")
    if dev.type != "cuda":
        raise ValueError(f"aero_b200 runs on CUDA devices only, got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


class Engine:
    """Owns an AeroLattice handle and the device workspace bound to it."""

    # layout_auto: the share of the device's free memory the two-buffer
    # workspace may take before the lattice switches to the AA layout
    AUTO_LAYOUT_FREE_SHARE = 0.8

    def __init__(self, params: AeroParams, solid: np.ndarray, links: np.ndarray, q: np.ndarray,
                 phi: Optional[np.ndarray] = None, device=None, layout_auto: bool = False):
        import torch
        self.torch = torch
        self.lib = _lib.load()
        self.device = _require_cuda(device)
        self.params = params
        self.dims = params.dims
        self.shape = (params.nz, params.ny, params.nx) if params.dims == 3 else (params.ny, params.nx)
        self.ncells = params.nx * params.ny * params.nz
        q_ = ctypes.c_int32()
        qg = ctypes.c_int32()
        check("aero_lattice_q", self.lib.aero_lattice_q(ctypes.byref(params), ctypes.byref(q_), ctypes.byref(qg)))
        self.Q, self.Qg = q_.value, qg.value
        solid_u8 = np.ascontiguousarray(solid, dtype=np.uint8)
        links = np.ascontiguousarray(links, dtype=np.int32)
        q = np.ascontiguousarray(q, dtype=np.float32)
        phi_c = None if phi is None else np.ascontiguousarray(phi, dtype=np.float64)
        self._create(solid_u8, links, q, phi_c)
        if layout_auto and params.layout == 0:
            free, _ = torch.cuda.mem_get_info(self.device)
            if self.workspace_bytes > self.AUTO_LAYOUT_FREE_SHARE * free:
                # two population buffers do not fit: one buffer updated in place
                self.lib.aero_destroy(self.h)
                self.h = None
                params.layout = 1
                self._create(solid_u8, links, q, phi_c)
        h = self.h
        with torch.cuda.device(self.device):
            self.workspace = torch.empty(self.workspace_bytes, dtype=torch.uint8, device=self.device)
            check("aero_bind_workspace", self.lib.aero_bind_workspace(
                h, self.workspace.data_ptr(), self.workspace_bytes, self.stream()))
        self.hist_capacity = params.hist_capacity or 4096
        self.nprof = params.nz if params.dims == 3 else params.ny
        if (1 + self.dims) * self.ncells * 8 > READBACK_CHUNK:
            _bounce_buffers()  # set-up cost, not a per-run one

    def _create(self, solid_u8, links, q, phi_c):
        """aero_create + aero_set_geometry for self.params; sets self.h and
        self.workspace_bytes (nothing allocated on the device yet)."""
        h = ctypes.c_void_p()
        check("aero_create", self.lib.aero_create(ctypes.byref(self.params), ctypes.byref(h)))
        self.h = h
        check("aero_set_geometry", self.lib.aero_set_geometry(
            h, solid_u8.ctypes.data, links.ctypes.data if len(links) else None,
            q.ctypes.data if len(q) else None, len(links), None if phi_c is None else phi_c.ctypes.data))
        nbytes = ctypes.c_uint64()
        check("aero_workspace_size", self.lib.aero_workspace_size(h, ctypes.byref(nbytes)))
        self.workspace_bytes = int(nbytes.value)

    # ------------------------------------------------------------------
    def stream(self):
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                self.lib.aero_destroy(h)
            except Exception:
                pass
            self.h = None

    # ------------------------------------------------------------------
    def _dev(self, a, shape):
        t = self.torch
        if isinstance(a, t.Tensor):
            x = a.to(device=self.device, dtype=t.float64)
        else:
            x = t.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(self.device)
        return x.reshape(shape).contiguous()

    def set_state(self, f, f_outlet_prev=None, g=None, step_count: int = 0) -> None:
        """f: (Q, ...) absolute populations (numpy or torch); optional outlet state and scalar."""
        fd = self._dev(f, (self.Q,) + self.shape)
        pd = None if f_outlet_prev is None else self._dev(
            f_outlet_prev, (self.Q,) + self.shape[:-1])
        gd = None if g is None else self._dev(g, (self.Qg,) + self.shape)
        with self.torch.cuda.device(self.device):
            check("aero_set_state", self.lib.aero_set_state(
                self.h, fd.data_ptr(), None if pd is None else pd.data_ptr(),
                None if gd is None else gd.data_ptr(), int(step_count), self.stream()))
            # keep the staging tensors alive until the copies ran
            self.torch.cuda.current_stream(self.device).synchronize()

    def set_equilibrium(self, rho=None, ux=None, uy=None, uz=None, T=None, step_count: int = 0) -> None:
        """State = feq of the given fields (numpy or torch, host or device;
        None = the uniform value), built on the device (aero_set_equilibrium).
        Host fields are copied as FP64, one array per given field."""
        fields = [None if a is None else self._dev(a, self.shape) for a in (rho, ux, uy, uz, T)]
        with self.torch.cuda.device(self.device):
            check("aero_set_equilibrium", self.lib.aero_set_equilibrium(
                self.h, *[None if a is None else a.data_ptr() for a in fields], int(step_count), self.stream()))
            self.torch.cuda.current_stream(self.device).synchronize()

    def get_state_device(self, want_prev=True, want_g=True):
        t = self.torch
        f = t.empty((self.Q,) + self.shape, dtype=t.float64, device=self.device)
        p = t.empty((self.Q,) + self.shape[:-1], dtype=t.float64, device=self.device) if want_prev else None
        g = (t.empty((self.Qg,) + self.shape, dtype=t.float64, device=self.device)
             if (want_g and self.Qg) else None)
        with t.cuda.device(self.device):
            check("aero_get_state", self.lib.aero_get_state(
                self.h, f.data_ptr(), None if p is None else p.data_ptr(),
                None if g is None else g.data_ptr(), self.stream()))
        return f, p, g

    def get_state(self):
        f, p, g = self.get_state_device()
        return (copy_to_host(f), copy_to_host(p), None if g is None else copy_to_host(g))

    def get_slab_device(self, z0: int, nzs: int):
        t = self.torch
        out = t.empty((self.Q, nzs) + self.shape[-2:], dtype=t.float64, device=self.device)
        with t.cuda.device(self.device):
            check("aero_get_state_slab", self.lib.aero_get_state_slab(
                self.h, int(z0), int(nzs), out.data_ptr(), self.stream()))
        return out

    def macroscopic_device(self):
        """(1 + dims, *shape) float64 device tensor: rho, ux, uy (, uz) of the state."""
        t = self.torch
        out = t.empty((1 + self.dims,) + self.shape, dtype=t.float64, device=self.device)
        with t.cuda.device(self.device):
            check("aero_get_macroscopic", self.lib.aero_get_macroscopic(self.h, out.data_ptr(), self.stream()))
        return out

    def field_stats(self, z0: int = 0, nzs: Optional[int] = None) -> np.ndarray:
        """FP64 statistics of the state over planes z0 .. z0+nzs-1 (all by
        default), reduced on the device (aero_field_stats)."""
        nzs = (self.params.nz - int(z0)) if nzs is None else int(nzs)
        out = np.empty(_lib.FIELD_STATS, dtype=np.float64)
        with self.torch.cuda.device(self.device):
            check("aero_field_stats", self.lib.aero_field_stats(self.h, int(z0), nzs, out.ctypes.data,
                                                                self.stream()))
        return out

    def set_inflow(self, fields: np.ndarray, first_step: int) -> None:
        """Uploads the transverse inlet velocities of steps first_step.. (n, dims-1, nz*ny)."""
        a = np.ascontiguousarray(fields, dtype=np.float64)
        with self.torch.cuda.device(self.device):
            check("aero_set_inflow", self.lib.aero_set_inflow(
                self.h, a.ctypes.data, int(first_step), int(a.shape[0]), self.stream()))

    def step(self, n: int) -> None:
        with self.torch.cuda.device(self.device):
            check("aero_step", self.lib.aero_step(self.h, int(n), self.stream()))

    def read_forces(self, max_steps: Optional[int] = None) -> np.ndarray:
        cap = self.hist_capacity if max_steps is None else int(max_steps)
        out = np.empty((cap, FORCE_VALUES), dtype=np.float64)
        n = ctypes.c_int64()
        with self.torch.cuda.device(self.device):
            check("aero_read_forces", self.lib.aero_read_forces(
                self.h, out.ctypes.data, cap, ctypes.byref(n), self.stream()))
        return out[: n.value]

    def read_profile(self) -> np.ndarray:
        out = np.empty((self.nprof, 3), dtype=np.float64)
        with self.torch.cuda.device(self.device):
            check("aero_read_profile", self.lib.aero_read_profile(self.h, out.ctypes.data, self.stream()))
        return out

    def status(self) -> int:
        v = ctypes.c_uint32()
        with self.torch.cuda.device(self.device):
            check("aero_status", self.lib.aero_status(self.h, ctypes.byref(v), self.stream()))
        return int(v.value)

    def first_bad_step(self) -> int:
        v = ctypes.c_int64()
        with self.torch.cuda.device(self.device):
            check("aero_first_bad_step", self.lib.aero_first_bad_step(self.h, ctypes.byref(v), self.stream()))
        return int(v.value)

    def set_step_kernel(self, kernel: int) -> None:
        check("aero_set_step_kernel", self.lib.aero_set_step_kernel(self.h, int(kernel)))

    def set_persistent(self, enable: bool) -> None:
        """Persistent runs of small lattices (one cooperative launch per call;
        on by default where the lattice qualifies, aero_set_persistent)."""
        check("aero_set_persistent", self.lib.aero_set_persistent(self.h, 1 if enable else 0))

    def kernel_variant(self) -> int:
        """0: the generic kernels; else the kernel set compiled for the
        lattice's feature word and wall type (aero_kernel_variant)."""
        k = ctypes.c_int32()
        check("aero_kernel_variant", self.lib.aero_kernel_variant(self.h, ctypes.byref(k)))
        return int(k.value)

    def persistent(self) -> bool:
        """Whether calls of two or more steps run persistently."""
        k = ctypes.c_int32()
        check("aero_get_persistent", self.lib.aero_get_persistent(self.h, ctypes.byref(k)))
        return bool(k.value)

    def get_step_kernel(self) -> int:
        k = ctypes.c_int32()
        check("aero_get_step_kernel", self.lib.aero_get_step_kernel(self.h, ctypes.byref(k)))
        return int(k.value)

    def les_fused(self) -> bool:
        """Whether the step kernel computes the LES rate from a shared-memory
        velocity stencil of its own (step kernel 6) rather than reading the
        velocity side output of a separate moments pass."""
        return self.get_step_kernel() == 6

    def step_plan(self) -> dict:
        """Step kernel in use: {"tiled": bool, "tile_rows": r, "blocks": b}."""
        t, r, b = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check("aero_step_plan", self.lib.aero_step_plan(self.h, ctypes.byref(t), ctypes.byref(r), ctypes.byref(b)))
        return {"tiled": bool(t.value), "tile_rows": int(r.value), "blocks": int(b.value)}

    # ------------------------------------------------------------------ timing
    def enable_timing(self, on: bool = True) -> None:
        check("aero_enable_timing", self.lib.aero_enable_timing(self.h, 1 if on else 0))

    def kernel_times(self):
        """(summed ms of the fused step kernel, of the force kernels, steps timed)."""
        a, b, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        with self.torch.cuda.device(self.device):
            check("aero_kernel_times", self.lib.aero_kernel_times(
                self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(n), self.stream()))
        return a.value, b.value, n.value
