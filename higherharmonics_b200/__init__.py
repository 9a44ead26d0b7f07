"""B200 engine for HigherHarmonics' per-k-point Bloch integration.

The compute path is the sm_100a library ``libhhg_gpu.so`` behind the C ABI in
``include/hhg_gpu.h``; ``api`` binds it with ctypes and ``workloads`` holds
the synthetic benchmark configurations.
"""
from . import api  # noqa: F401

__all__ = ["api"]
