"""gpuga_b200: a B200-native fitness engine for GPUGA (genetic-algorithm fitting
of empirical interatomic potentials: minimal Tersoff, rigid-ion, NN 2-body).

The compute lives in libgpuga_b200.so (CUDA for sm_100a + host C++, C ABI in
include/gpuga.h); this package holds thin ctypes bindings that mirror the
reference's Fitness / GA interfaces and the seeded synthetic workloads.
"""
from ._lib import (PATH_BATCHED, PATH_PLAIN32, PATH_PLAIN64, GpugaError, load)  # noqa: F401
from .fitness import GA, Fitness, Server, options  # noqa: F401

__all__ = ["Fitness", "GA", "Server", "options", "load", "GpugaError", "PATH_BATCHED", "PATH_PLAIN64",
           "PATH_PLAIN32"]
