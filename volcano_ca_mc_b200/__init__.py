"""B200-native lava cellular automaton and Potts crystallisation (volcano-ca-mc hot paths).

The compute lives in ``lib/libvca.so`` (hand-written sm_100a CUDA behind the C ABI of
``include/vca.h``); ``bin/engine`` is the C++17 command-line engine with the reference's
surface.  ``capi`` is the ctypes binding for Python callers.
"""
from .capi import (CaParams, LavaCA, McParams, PottsMC, VcaError, SWEEP_ACTIVE, SWEEP_DENSE,  # noqa: F401
                   LIB_PATH, ENGINE_PATH)

__all__ = ["CaParams", "LavaCA", "McParams", "PottsMC", "VcaError", "SWEEP_ACTIVE", "SWEEP_DENSE",
           "LIB_PATH", "ENGINE_PATH"]
