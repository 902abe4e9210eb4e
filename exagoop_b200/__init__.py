"""B200-native explicit MPM time step: a drop-in for the per-step
particle/grid path of the ExaGOOP MPM solver.

The compute path is libexg.so (hand-written sm_100a CUDA behind the C ABI in
include/exg.h); this package holds its ctypes binding and the seeded scene
generators used by the tests and the benchmark.
"""
from .native import (Context, ExgError, Inputs, Particles, Specs, default_specs, lib)  # noqa: F401

__all__ = ["Context", "ExgError", "Inputs", "Particles", "Specs", "default_specs", "lib"]
