"""gpk_b200 — B200 (sm_100a) implementation of the GPK per-step hot path.

The public surface mirrors the reference's C++ interface (include/gpk_core.hpp
of albert-hzbn/GPK): :class:`GPKGrid` with ``step``/``run`` and the public
fields, and one descriptor factory per ``ThermoModel`` subclass in
:mod:`gpk_b200.thermo`.  All stepping runs in libgpk_b200.so on the GPU.
This package is the plain ctypes binding of the C ABI and uses NumPy only;
the PyTorch-facing layer (device tensors, the autograd Function of the
adjoint, the spectral and Al-Cu drop-ins) is the ``gpk`` package under
python/.
"""
from . import thermo
from .grid import GPKGrid, voronoi
from ._lib import GPKError, lib
from .batch import GPKBatch

__all__ = ["GPKGrid", "voronoi", "thermo", "GPKError", "lib", "GPKBatch"]
