"""seiscl_b200 -- a B200-native staggered-grid FDTD engine with the
single-device forward-modelling and adjoint-gradient path of SeisCL.

The compute path is libseiscl_b200.so (hand-written sm_100a CUDA behind a
C ABI, include/seiscl_b200.h).  This package holds its Python binding and the
SeisCL-compatible front end.
"""
from .engine import Config, Plan, SeisCLEngineError, load_library, source_type_mask  # noqa: F401

__all__ = ["Config", "Plan", "SeisCLEngineError", "load_library", "source_type_mask"]
