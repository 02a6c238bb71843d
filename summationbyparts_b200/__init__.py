"""sbp_b200: B200-native SBP-SAT Euler time stepping (the hot path of mulimoen/SummationByParts).

The compute runs in libsbp_b200.so (hand-written CUDA for sm_100a behind the C ABI in
include/sbp_b200.h); this package is the host-side mirror of the reference's Rust API.
"""
from . import _capi
from ._capi import SbpError, version
from .operators import SBP4, SBP8, Pair, Upwind4, Upwind4h2, Upwind9, Upwind9h2
from .system import BlockSpec, BlockSystem, Vortice, VortexParameters

__all__ = ["SbpError", "version", "SBP4", "SBP8", "Pair", "Upwind4", "Upwind4h2", "Upwind9", "Upwind9h2",
           "BlockSpec", "BlockSystem", "Vortice", "VortexParameters", "_capi"]
