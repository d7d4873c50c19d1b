"""latticeu1_b200: B200-native (sm_100a) U(1) lattice-gauge Monte Carlo hot path.

The compute path is the CUDA library libu1b200.so behind the C ABI in
include/u1_b200.h; this package is its Python host layer.
"""
from ._lib import U1Error, launch_count, lib  # noqa: F401  (raises if the library is missing)
from .lattice import Batch, Context, Lattice, Rng  # noqa: F401

__all__ = ["Batch", "Context", "Lattice", "Rng", "U1Error", "launch_count", "lib"]
