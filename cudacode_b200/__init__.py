"""B200 Monte Carlo engine for classical Heisenberg spins on the pyrochlore
lattice: colour-pass Metropolis and over-relaxation sweeps, FP64 observables
and replica exchange as hand-written sm_100a CUDA behind the C-ABI of
``include/pyro.h``."""
from .engine import (Engine, PyroError, System, geometric_ladder, load_library,  # noqa: F401
                     neighbour_table)

__all__ = ["Engine", "PyroError", "System", "geometric_ladder", "load_library",
           "neighbour_table"]
