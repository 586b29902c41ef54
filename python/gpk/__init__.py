"""gpk — the Python package of the GPK hot path on B200.

It takes the place of the reference's python/gpk (albert-hzbn/GPK,
python/gpk/__init__.py exports GPKGrid, ThermoModel and SolidificationThermo)
and is the one place where PyTorch enters: device tensors for the spectral
elasticity and Al-Cu drop-ins, and the torch.autograd.Function of the
adjoint calibration loss.  The grid itself is the C++ GPKGrid's
(include/gpk_core.hpp) over libgpk_b200.so, bound without torch in the
gpk_b200 package.

    GPKGrid, ThermoModel, SolidificationThermo   the reference's names
    thermo                                       one factory per ThermoModel subclass
    SpectralElasticity, spectral_elasticity      FP64 cuFFT micro-elasticity
    AdjointProblem, GPKLoss, gpk_loss            gradients at a fixed label map
    alcu                                         the Al-Cu transport and remap drop-ins
"""
import os as _os
import sys as _sys

_ROOT = _os.path.dirname(_os.path.dirname(_os.path.dirname(_os.path.abspath(__file__))))
if _ROOT not in _sys.path:
    _sys.path.insert(0, _ROOT)

from gpk_b200 import GPKBatch, GPKError, GPKGrid, thermo, voronoi  # noqa: E402
from gpk_b200.thermo import ThermoDesc  # noqa: E402

from . import alcu  # noqa: E402
from .adjoint import AdjointProblem, calibration_case  # noqa: E402
from .autograd import GPKLoss, gpk_loss  # noqa: E402
from .spectral import SpectralElasticity, spectral_elasticity, variant_eigenstrains  # noqa: E402


def ThermoModel(**fields) -> ThermoDesc:
    """The plain ThermoModel (its default virtuals) with member overrides."""
    d = ThermoDesc("base")
    for k, v in fields.items():
        setattr(d, k, v)
    return d


SolidificationThermo = thermo.solidification

__all__ = ["GPKGrid", "ThermoModel", "SolidificationThermo", "thermo", "voronoi", "GPKError", "GPKBatch",
           "SpectralElasticity", "spectral_elasticity", "variant_eigenstrains", "AdjointProblem",
           "calibration_case", "GPKLoss", "gpk_loss", "alcu"]
