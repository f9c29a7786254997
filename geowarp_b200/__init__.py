"""geowarp_b200: B200-native implicit cpGIMP material point engine.

A drop-in for GeoWarp's solver classes (quasi_static_solver_2d,
quasi_static_coupled_solver_2d, quasi_static_coupled_solver_3d) whose load
step runs on hand-written sm_100a CUDA kernels (libgeowarp_b200.so, C ABI in
include/geowarp_b200.h).  There is no CPU fallback.
"""
from .launch import launch

__all__ = ["launch", "quasi_static_solver_2d", "quasi_static_coupled_solver_2d", "quasi_static_coupled_solver_3d"]


def __getattr__(name):
    if name in ("quasi_static_solver_2d", "quasi_static_coupled_solver_2d", "quasi_static_coupled_solver_3d"):
        from . import solvers
        return getattr(solvers, name)
    raise AttributeError(name)
