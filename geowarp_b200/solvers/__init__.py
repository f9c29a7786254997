"""Drop-in solver classes with the reference's names and constructor dicts."""
from .quasi_static_solver_2d import quasi_static_solver_2d
from .quasi_static_coupled_solver_2d import quasi_static_coupled_solver_2d
from .quasi_static_coupled_solver_3d import quasi_static_coupled_solver_3d

__all__ = ["quasi_static_solver_2d", "quasi_static_coupled_solver_2d", "quasi_static_coupled_solver_3d"]
