"""B200-native rebuild of RESET's set-intersection hot path.

The computation lives in libreset.so (hand-written sm_100a CUDA behind the C
ABI of include/reset.h).  This package holds its Python host side: the ctypes
binding (_lib), the tensor-level API (api), and the build script (build).
"""
from .build import build as build_library  # noqa: F401

__all__ = ["build_library"]
