"""B200-native Gay-Berne Monte Carlo sweep (drop-in for MCnptColloid.c's MC path).

The compute path is liblcmc.so (hand-written CUDA for sm_100a behind the C ABI
in include/lcmc.h); this package is its Python host mirror.
"""
from ._lib import LcmcError, Params, Stats, lib  # noqa: F401
from .mc import GBSystem, default_params, lattice, load_initial_conditions, run, run_simulation  # noqa: F401

__all__ = ["GBSystem", "LcmcError", "Params", "Stats", "default_params", "lattice", "lib",
           "load_initial_conditions", "run", "run_simulation"]
