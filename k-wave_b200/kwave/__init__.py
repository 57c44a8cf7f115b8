"""kwave: host side of the B200 k-space pseudospectral acoustic solver.

The time loop runs in ``libkwave_b200.so`` (hand-written sm_100a CUDA
kernels behind the C ABI in ``include/kwave_b200.h``); this package holds the
ctypes binding and the reference's MATLAB-side pre- and post-processing.
"""
from ._lib import KwaveError, Session, solve, version  # noqa: F401
from .simulation import kspace_first_order, kspaceFirstOrder2D, kspaceFirstOrder3D, kspaceFirstOrderAS, prepare  # noqa: F401
from .transducer import KWaveTransducer  # noqa: F401
from .utils import KWaveGrid  # noqa: F401
