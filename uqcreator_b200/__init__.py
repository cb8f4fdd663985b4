"""B200-native implementation of UQCreator's per-time-step IPM hot path.

The product is the CUDA extension libuqc_b200.so (C ABI: include/uqc.h);
this package holds its build recipe, the ctypes binding and a Python mirror of
the reference's Closure / MomentSolver / Settings operator surface.
"""
from . import workloads
from ._lib import UqcError, lib, LIB_PATH, FP64, MIXED, LAYOUT_REF, LAYOUT_STATE_MAJOR
from .solver import Settings, Solver, Closure, MomentSolver

__all__ = ["Settings", "Solver", "Closure", "MomentSolver", "UqcError", "lib", "LIB_PATH", "FP64", "MIXED",
           "LAYOUT_REF", "LAYOUT_STATE_MAJOR", "workloads"]
