"""B200 implementation of Canard's per-step hot path.

The compute path is the in-tree CUDA library ``libcanard_b200.so`` (sm_100a)
behind the C ABI of ``include/canard_gpu.h``; this package is its Python host
side. There is no CPU fallback: if the library is missing, importing
``canard_b200.api`` raises.
"""
from . import cases  # noqa: F401

__all__ = ["cases", "api"]
