"""crushrs_b200 — a B200-native (sm_100a) engine for the explicit time step of
crushrs-style crash models: one-point honeycomb hexahedra with rank-12
hourglass control, deterministic node-gather force assembly, central-difference
integration with selective mass scaling, stable-dt reduction and node-to-face
penalty contact over a device-built uniform grid.

The product is the C ABI in include/crush.h, implemented by the CUDA/C++
library libcrush_b200.so built in-tree (crushrs_b200/build.py). This package
holds the ctypes mirror of that ABI and thin Python wrappers over it.
"""
from . import abi  # noqa: F401

__all__ = ["abi"]
