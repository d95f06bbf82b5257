"""sod2d_refmap_b200 — B200-native (sm_100a) explicit spectral-element RHS of SOD2D.

The compute path is libsod2d_b200.so (CUDA, C ABI in include/sod2d_b200.h); this package
holds its ctypes binding, the host-side mirror of the reference solver interface, mesh and
initial-state generators, and the autograd wrapper of the adjoint.
"""
from . import mesh  # noqa: F401

__all__ = ["mesh", "solver", "build"]
