"""diablo_b200: B200 (sm_100a) implementation of DIABLO's RK3/Crank-Nicolson
channel and triply periodic steppers behind the reference's subroutine
boundary (C-ABI in include/diablo_b200.h)."""
from .params import Params  # noqa: F401
from . import grid, ics, configs  # noqa: F401

__version__ = "0.1.0"


def __getattr__(name):
    # the solver classes need the CUDA library; import them lazily
    if name in ("Channel", "Periodic", "DiabloError"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
