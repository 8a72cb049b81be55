"""wakis_b200: B200-native FIT leap-frog stepper and wake integration behind
the Wakis ``GridFIT3D`` / ``SolverFIT3D`` / ``WakeSolver`` / ``Field`` API.

Importing the package does not need a GPU; constructing a solver does, and
loads the in-tree native library ``libwakis_b200.so``.
"""

from . import geometry, materials, sources
from .field import Field
from .gridFIT3D import GridFIT3D
from .logger import Logger
from .solverFIT3D import SolverFIT3D
from .wakeSolver import WakeSolver

__version__ = "0.1.0"

__all__ = ["Field", "GridFIT3D", "SolverFIT3D", "WakeSolver", "Logger", "geometry",
           "materials", "sources"]
