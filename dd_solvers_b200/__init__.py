"""B200-native Schwarz-preconditioned CG with the ``dd_solvers`` Python API.

``from dd_solvers_b200 import CG, AdditiveSchwarz, HybridSchwarz, Inv, CUDSS`` is
the drop-in for ``from dd_solvers import ...`` (src/dd_solvers/dd_solvers/__init__.py:1-3).
``DiffusionSolve`` / ``Q1Diffusion`` add a differentiable solve (no counterpart
in the reference).
"""
from .solvers import *  # noqa: F401,F403
from .solvers import __all__ as _solver_names
from .autograd import DiffusionSolve, Q1Diffusion  # noqa: F401

__all__ = list(_solver_names) + ["DiffusionSolve", "Q1Diffusion"]
