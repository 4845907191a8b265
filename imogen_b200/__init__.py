"""imogen_b200: B200-native relaxing-TVD fluid + magnet update (Imogen's hot path).

The compute path is the in-tree CUDA library ``libimogen_b200.so`` (C ABI in
include/imogen_b200.h); this package is its host-side binding and the reference-shaped call
surface.  There is no CPU fallback: without the CUDA library every call raises.
"""
from . import _lib
from ._lib import ImogenError, lib
from .run import ImogenBatch, ImogenRun, TimeManager, bytes_required, flux, magnetFlux, make_config, relaxingFluid

__all__ = ["ImogenBatch", "ImogenRun", "TimeManager", "ImogenError", "flux", "relaxingFluid", "magnetFlux",
           "make_config", "bytes_required", "lib"]
