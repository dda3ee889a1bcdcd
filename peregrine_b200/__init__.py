"""PEREGRINE's right-hand side and Runge-Kutta stage, B200-native.

The reference's case API (``Config``, ``get_backend``, ``get_solver``,
``mesher.CubeMesher``) over a CUDA library for sm_100a (``libpgb200.so``,
include/pgb200.h).
"""

from peregrine_b200 import mesher
from peregrine_b200.config import Config, ConfigError
from peregrine_b200.solver import Backend, Solver, get_backend, get_solver

__all__ = ["Config", "ConfigError", "Backend", "Solver", "get_backend", "get_solver", "mesher"]
