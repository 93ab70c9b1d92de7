"""B200-native spectral-element time step behind Salvus's plugin vocabulary.

The compute path is libsalvus_b200.so (hand-written sm_100a CUDA kernels
behind a C ABI, include/salvus_b200.h); this package is the Python host
mirror of the reference's Problem / Order2Newmark interface over that ABI.
"""
from .core import (ACOUSTIC, ELASTIC3D, FP32, FP64, HEX, QUAD, RUN_GRAPH, RUN_PLAIN, Mesh,
                   Problem, SalvusError, launch_count, lib)

__all__ = ["ACOUSTIC", "ELASTIC3D", "FP32", "FP64", "HEX", "QUAD", "RUN_GRAPH", "RUN_PLAIN",
           "Mesh", "Problem", "SalvusError", "launch_count", "lib"]
