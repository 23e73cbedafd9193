"""ofeli_b200 -- OFELI's P1 assembly + preconditioned Krylov path on B200.

The compute path is libofeli_gpu.so (hand-written sm_100a CUDA behind the C
ABI of include/ofeli_gpu.h); ``ofeli_b200.ofeli`` mirrors OFELI's C++ API
names on top of it and ``ofeli_b200.capi`` is the raw binding.
"""
from . import capi  # noqa: F401

__all__ = ["capi", "ofeli", "fields"]
