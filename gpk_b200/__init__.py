"""gpk_b200 — B200 (sm_100a) implementation of the GPK per-step hot path.

The public surface mirrors the reference's C++ interface (include/gpk_core.hpp
of albert-hzbn/GPK): :class:`GPKGrid` with ``step``/``run`` and the public
fields, and one descriptor factory per ``ThermoModel`` subclass in
:mod:`gpk_b200.thermo`.  All stepping runs in libgpk_b200.so on the GPU.
"""
from . import thermo
from .grid import GPKGrid, voronoi
from ._lib import GPKError, lib
from .spectral import SpectralElasticity, spectral_elasticity
from .batch import GPKBatch
from . import alcu

__all__ = ["GPKGrid", "voronoi", "thermo", "GPKError", "lib", "SpectralElasticity", "spectral_elasticity",
           "GPKBatch", "alcu"]
