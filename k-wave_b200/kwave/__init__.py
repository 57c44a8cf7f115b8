"""kwave: host side of the B200 k-space pseudospectral acoustic solver.

The time loop runs in ``libkwave_b200.so`` (hand-written sm_100a CUDA
kernels behind the C ABI in ``include/kwave_b200.h``); this package holds the
ctypes binding and the reference's MATLAB-side pre- and post-processing.

Names are resolved on first use: importing the pre-processing modules
(``kwave.simulation``, ``kwave.workloads``, ``kwave.utils``) does not load
the CUDA library, so a CPU-only caller can build inputs without mapping it.
Every solve still goes through the library, and fails loudly when it is
missing.
"""
import importlib

_LAZY = {
    "KwaveError": "_lib",
    "Session": "_lib",
    "solve": "_lib",
    "version": "_lib",
    "kspace_first_order": "simulation",
    "kspaceFirstOrder2D": "simulation",
    "kspaceFirstOrder3D": "simulation",
    "kspaceFirstOrderAS": "simulation",
    "prepare": "simulation",
    "KWaveTransducer": "transducer",
    "KWaveGrid": "utils",
}

__all__ = sorted(_LAZY)


def __getattr__(name):
    mod = _LAZY.get(name)
    if mod is None:
        raise AttributeError(f"module 'kwave' has no attribute {name!r}")
    value = getattr(importlib.import_module("." + mod, __name__), name)
    globals()[name] = value
    return value
