"""ghost_b200: GHOST's 3D HD pseudospectral hot path on B200 (sm_100a).

The compute path is libghost_b200.so (hand-written CUDA kernels behind the
C ABI of include/ghost_b200.h); this package is the host-side mirror of
GHOST's fftp / pseudospec3D interface over that ABI.
"""
from ._lib import GhostError, load  # noqa: F401
from .pseudospec import GHOST_COMPLEX_TO_REAL, GHOST_REAL_TO_COMPLEX, Ensemble, FFTPlan, Ghost, io_filename  # noqa: F401

__all__ = ["Ghost", "Ensemble", "FFTPlan", "GhostError", "load", "GHOST_REAL_TO_COMPLEX", "GHOST_COMPLEX_TO_REAL",
           "io_filename"]
