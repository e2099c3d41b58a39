"""aero_b200 -- B200-native (sm_100a) lattice Boltzmann engine for the Aero
wind-tunnel solver's per-step hot path.

    from aero_b200 import Solver, Solver3D, Cylinder, Sphere

``Solver`` / ``Solver3D`` take the reference constructor options and run every
step in hand-written CUDA kernels (libaero_b200.so, C ABI in
include/aero_b200.h).  The CUDA library is built in-tree by
``aero_b200._build.build()``; without it (or without a CUDA GPU) the solvers
raise instead of falling back to a CPU path.
"""

from .geometry import Box, Cylinder, Rectangle, Sphere
from .links import build_surface_links, build_surface_links_3d, build_surface_links_device

__all__ = ["Solver", "Solver3D", "Batch", "Cylinder", "Rectangle", "Sphere", "Box", "build_surface_links",
           "build_surface_links_3d", "build_surface_links_device", "build"]


def build(force: bool = False):
    """Compiles libaero_b200.so for sm_100a (in-tree) and returns its path."""
    from . import _build
    return _build.build(force=force)


def __getattr__(name):
    if name == "Solver":
        from .solver import Solver
        return Solver
    if name == "Solver3D":
        from .solver3d import Solver3D
        return Solver3D
    if name == "Batch":
        from .batch import Batch
        return Batch
    raise AttributeError(name)
