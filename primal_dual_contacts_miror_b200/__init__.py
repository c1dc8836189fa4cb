"""B200-native (sm_100a) primal-dual interior-point contact solver.

Drop-in for the reference's ForceSolver::fillForces (src/Solver/ForceSolverBase.h:78-82)
behind the C ABI in include/pdc.h; see solver.py for the Python mirror of the
reference interface and lib.py for the ctypes binding.
"""
from . import abi  # noqa: F401

__version__ = "0.1.0"
