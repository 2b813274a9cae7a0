"""Local-PSF (RANA) renderer on the GPU: data contracts and the operator."""

from .fields import FullFieldPSF
from .depth import DepthFullFieldRenderer, DepthPSFBank
from .operator import RanaOperator, _axis_weights
from ._fft import LocalFFTPlan
from ._backends import get_backend
from .cubic import CubicFullFieldRenderer

__all__ = ["FullFieldPSF", "DepthPSFBank", "RanaOperator", "LocalFFTPlan", "get_backend", "CubicFullFieldRenderer",
           "DepthFullFieldRenderer"]
