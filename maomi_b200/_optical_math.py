"""Optical parameter records and the scalar helpers the stage geometry needs.

Mirrors the parts of maomi/_optical_math.py used on the optical path:
``VolParams``/``PsfParams`` (:11-17, :87-113), ``gaussian_beam_size``
(:116-118) and the Zernike index / radial-polynomial conventions (:137-173),
the latter as host-side coefficient tables consumed by the CUDA pupil kernel.
"""

from dataclasses import dataclass, field
from math import factorial
import typing

import numpy as np


@dataclass
class VolParams:
    vol_sz: np.ndarray = field(default_factory=lambda: np.array([100, 100, 30], dtype=np.float32))
    vres: float = 2.0
    vol_depth: float = 100.0
    vasc_sz: typing.Optional[np.ndarray] = None
    verbose: int = 1


@dataclass
class PsfParams:
    NA: float = 0.6
    objNA: float = 0.8
    n: float = 1.35
    lambda_exc: float = 0.92
    obj_fl: float = 4.5
    ss: int = 4
    sampling: int = 1
    zernikeDst: typing.Optional[np.ndarray] = None
    zernikeWt: typing.Optional[typing.Any] = None
    custom_phase: typing.Optional[np.ndarray] = None
    scatter_sz: typing.Optional[np.ndarray] = None
    scatter_wt: typing.Optional[np.ndarray] = None
    type: str = "gaussian"
    psf_sz: np.ndarray = field(default_factory=lambda: np.array([20.0, 20.0, 50.0], dtype=np.float32))
    prop_sz: float = 10.0
    n_diff: float = 0.02
    fastmask: bool = True
    propcrop: bool = True
    taillength: typing.Optional[float] = 50.0
    bprof: str = "gaussian"
    length: typing.Optional[float] = None
    cylscale: typing.Optional[np.ndarray] = None
    scaling: typing.Optional[str] = None


def gaussian_beam_size(psf_params, dist, apod=2.0):
    """Lateral window (um) that holds the objective cone at ``dist`` um:
    ceil(1.5 * tan(asin(objNA/n)) * dist) * apod, as a float32 (x, y, 0) triple."""
    half = np.ceil(np.tan(np.arcsin(psf_params.objNA / psf_params.n)) * dist * 1.5) * apod
    return np.array([half, half, 0], dtype=np.float32)


def zernike_degree(i):
    """Radial degree of mode ``i`` in the reference's single-index ordering."""
    return int(np.ceil(np.sqrt(0.25 + 2 * i) - 1.5))


def zernike_azimuth(i):
    """Azimuthal frequency of mode ``i`` in the reference's single-index ordering."""
    deg = zernike_degree(i)
    rest = i - (deg + 1) * deg / 2
    if deg % 2 == 0:
        return int(2 * np.floor(rest / 2))
    return int(2 * np.ceil(rest / 2) - 1)


def zernike_terms(i):
    """(norm, m, use_cos, [(coef, power), ...]) for mode ``i``.

    Z_i(r, t) = norm * sum(coef * r**power) * {1, cos(m t), sin(m t)}, with the
    standard radial polynomial sum_s (-1)^s (n-s)! / (s! ((n+m)/2-s)! ((n-m)/2-s)!)."""
    deg, m = zernike_degree(i), zernike_azimuth(i)
    terms = []
    for s in range(int((deg - m) / 2) + 1):
        c = ((-1) ** s) * factorial(deg - s) / (
            factorial(s) * factorial(int((deg + m) / 2 - s)) * factorial(int((deg - m) / 2 - s)))
        terms.append((c, deg - 2 * s))
    norm = np.sqrt(deg + 1) if m == 0 else np.sqrt(2 * (deg + 1))
    return float(norm), m, (i % 2 == 0), terms
