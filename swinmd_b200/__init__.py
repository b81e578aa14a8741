"""SwinMD per-step force and integration path on NVIDIA B200 (sm_100a).

The compute path is the CUDA library ``libswinmd_b200.so`` behind the C ABI
of ``include/swinmd_b200.h``; this package holds its ctypes binding, the
host-side mirror of SwinMD's Ensemble / Force / Integrator interface, and the
synthetic benchmark systems.
"""
from . import systems  # noqa: F401

__all__ = ["systems", "engine", "build"]
