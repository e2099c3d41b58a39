"""ctypes binding of the aero_b200 C ABI (include/aero_b200.h).

The shared library libaero_b200.so is built in-tree by aero_b200._build.  If
it is missing and cannot be built, importing this module raises ImportError:
there is no CPU fallback for the engine.
"""

from __future__ import annotations

import ctypes
import pathlib

from . import _build

ABI_VERSION = 3
FORCE_VALUES = 12
FIELD_STATS = 10

STORE = {"fp32": 0, "fp64": 1, "fp16s": 2, "bf16s": 3}
COLLISION = {"bgk": 0, "trt": 1, "mrt": 2}
INLET = {"none": 0, "velocity": 1, "pressure": 2}
OUTLET = {"none": 0, "convective": 1, "zerogradient": 2, "pressure": 3}
WALL = {"none": 0, "slip": 1, "noslip": 2, "moving": 3}
LES_MODEL = {"smagorinsky": 0, "wale": 1}

ERRORS = {0: "AERO_OK", -1: "AERO_ERR_INVALID", -2: "AERO_ERR_CUDA", -3: "AERO_ERR_STATE",
          -4: "AERO_ERR_UNSUPPORTED", -5: "AERO_ERR_CAPACITY"}
ERRORS_BY_NAME = {v: k for k, v in ERRORS.items()}

# exported entry points with their argument types
_I32, _I64, _U64, _D, _VP = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double, ctypes.c_void_p


class AeroParams(ctypes.Structure):
    _fields_ = [(n, _I32) for n in (
        "abi_version", "dims", "nx", "ny", "nz", "storage", "collision", "inlet_bc", "outlet_bc",
        "wall_bc", "streamwise_open", "les", "les_model", "van_driest", "bouzidi", "thermal",
        "buoyancy", "scalar_reduced", "sponge_thickness", "hist_capacity")] + [
        (n, _D) for n in (
            "omega", "u0", "rho0", "rho_in", "rho_out", "inlet_perturbation", "trt_lambda",
            "sponge_strength", "les_cs", "van_driest_A", "wall_velocity_top",
            "wall_velocity_bottom")] + [
        ("body_force", _D * 3)] + [
        (n, _D) for n in ("alpha_T", "T_hot", "T_cold", "g_gravity", "beta", "T_ref")] + [
        ("center", _D * 3)] + [
        (n, _I32) for n in ("recycling", "inflow_field", "inflow_ring", "layout")]


SIGNATURES = {
    "aero_abi_version": ([], ctypes.c_int),
    "aero_params_size": ([], ctypes.c_int),
    "aero_last_error": ([], ctypes.c_char_p),
    "aero_lattice_q": ([ctypes.POINTER(AeroParams), ctypes.POINTER(_I32), ctypes.POINTER(_I32)], ctypes.c_int),
    "aero_create": ([ctypes.POINTER(AeroParams), ctypes.POINTER(_VP)], ctypes.c_int),
    "aero_set_geometry": ([_VP, _VP, _VP, _VP, _I64, _VP], ctypes.c_int),
    "aero_workspace_size": ([_VP, ctypes.POINTER(_U64)], ctypes.c_int),
    "aero_bind_workspace": ([_VP, _VP, _U64, _VP], ctypes.c_int),
    "aero_set_state": ([_VP, _VP, _VP, _VP, _I64, _VP], ctypes.c_int),
    "aero_get_state": ([_VP, _VP, _VP, _VP, _VP], ctypes.c_int),
    "aero_get_state_slab": ([_VP, _I32, _I32, _VP, _VP], ctypes.c_int),
    "aero_get_macroscopic": ([_VP, _VP, _VP], ctypes.c_int),
    "aero_field_stats": ([_VP, _I32, _I32, _VP, _VP], ctypes.c_int),
    "aero_set_equilibrium": ([_VP, _VP, _VP, _VP, _VP, _VP, _I64, _VP], ctypes.c_int),
    "aero_step": ([_VP, _I64, _VP], ctypes.c_int),
    "aero_read_forces": ([_VP, _VP, _I64, ctypes.POINTER(_I64), _VP], ctypes.c_int),
    "aero_read_profile": ([_VP, _VP, _VP], ctypes.c_int),
    "aero_status": ([_VP, ctypes.POINTER(ctypes.c_uint32), _VP], ctypes.c_int),
    "aero_step_count": ([_VP, ctypes.POINTER(_I64)], ctypes.c_int),
    "aero_step_plan": ([_VP, ctypes.POINTER(_I32), ctypes.POINTER(_I32), ctypes.POINTER(_I32)], ctypes.c_int),
    "aero_set_inflow": ([_VP, _VP, _I64, _I64, _VP], ctypes.c_int),
    "aero_set_step_kernel": ([_VP, _I32], ctypes.c_int),
    "aero_get_step_kernel": ([_VP, ctypes.POINTER(_I32)], ctypes.c_int),
    "aero_set_persistent": ([_VP, _I32], ctypes.c_int),
    "aero_get_persistent": ([_VP, ctypes.POINTER(_I32)], ctypes.c_int),
    "aero_kernel_variant": ([_VP, ctypes.POINTER(_I32)], ctypes.c_int),
    "aero_first_bad_step": ([_VP, ctypes.POINTER(_I64), _VP], ctypes.c_int),
    "aero_destroy": ([_VP], ctypes.c_int),
    "aero_mrt_operator": ([_I32, _D, _VP, _VP], ctypes.c_int),
    "aero_enable_timing": ([_VP, _I32], ctypes.c_int),
    "aero_collide_host": ([ctypes.POINTER(AeroParams), _VP, _VP, _VP, _I64], ctypes.c_int),
    "aero_link_forces_static": ([_I32, _I32, _I32, _I32, _VP, _VP, _VP, _I64, _VP, _VP, _VP, _VP],
                                ctypes.c_int),
    "aero_kernel_times": ([_VP, ctypes.POINTER(_D), ctypes.POINTER(_D), ctypes.POINTER(_I64), _VP],
                          ctypes.c_int),
    "aero_batch_create": ([_I32, ctypes.POINTER(_VP)], ctypes.c_int),
    "aero_batch_workspace_size": ([_VP, ctypes.POINTER(_U64)], ctypes.c_int),
    "aero_batch_bind_workspace": ([_VP, _VP, _U64], ctypes.c_int),
    "aero_batch_add": ([_VP, _VP, _D], ctypes.c_int),
    "aero_batch_remove": ([_VP, _VP], ctypes.c_int),
    "aero_batch_size": ([_VP, ctypes.POINTER(_I32)], ctypes.c_int),
    "aero_batch_step": ([_VP, _I64, _VP], ctypes.c_int),
    "aero_batch_converge": ([_VP, _I32, _D, _VP, _VP], ctypes.c_int),
    "aero_batch_destroy": ([_VP], ctypes.c_int),
    "aero_surface_links_scratch_size": ([_I32, _I32, _I32, _I32, ctypes.POINTER(_U64)], ctypes.c_int),
    "aero_surface_links_device": ([_I32, _I32, _I32, _I32, _VP, _VP, _VP, _U64, _VP, _VP, _I64,
                                   ctypes.POINTER(_I64), _VP], ctypes.c_int),
}


class AeroError(RuntimeError):
    """A C-ABI call returned an error code."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed with {ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load(build_if_missing: bool = True) -> ctypes.CDLL:
    """Loads libaero_b200.so (building it with nvcc when absent)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not path.exists():
        if not build_if_missing:
            raise ImportError(f"aero_b200: {path.name} not found; build it with python -m aero_b200._build")
        try:
            _build.build()
        except Exception as exc:  # no nvcc, compile error, ...
            if not path.exists():
                raise ImportError(f"aero_b200: cannot build {path.name}: {exc}") from exc
    lib = ctypes.CDLL(str(path))
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if lib.aero_abi_version() != ABI_VERSION:
        raise ImportError(f"aero_b200: ABI version {lib.aero_abi_version()} != {ABI_VERSION}")
    if lib.aero_params_size() != ctypes.sizeof(AeroParams):
        raise ImportError("aero_b200: AeroParams layout mismatch between Python and C")
    _lib = lib
    return lib


def check(fn: str, code: int) -> None:
    if code != 0:
        msg = load().aero_last_error()
        raise AeroError(fn, code, msg.decode() if msg else "")


def library_path() -> pathlib.Path:
    return _build.LIB
