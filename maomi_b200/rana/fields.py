"""Full-field effective-intensity PSF contract (maomi/rana/fields.py:17-110).

Axes field_X, field_Y, kernel_X, kernel_Y[, kernel_Z]; kernel origin shape//2;
coordinates and pitches in specimen micrometres; the same validation and the
same ``maomi.full_field_psf.v1`` file format as the reference, so banks move
between the two implementations unchanged.
"""

import json
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

SCHEMA = "maomi.full_field_psf.v1"


@dataclass(frozen=True)
class FullFieldPSF:
    kernels: np.ndarray
    x_um: np.ndarray
    y_um: np.ndarray
    voxel_size_um: tuple
    wavelength_nm: float
    operator: str
    provenance: dict = field(default_factory=dict)

    def __post_init__(self):
        if np.iscomplexobj(self.kernels):
            raise ValueError("Supply effective real intensity, not a complex optical field")
        k = np.array(self.kernels, dtype=np.float64, copy=True)
        axes = [np.array(c, dtype=float, copy=True) for c in (self.x_um, self.y_um)]
        for c in axes:
            if c.ndim != 1 or len(c) < 2 or not np.isfinite(c).all() or (np.diff(c) <= 0).any():
                raise ValueError("Full-field PSFs require at least two increasing finite nodes on EACH XY axis")
        if (k.ndim not in (4, 5) or k.shape[:2] != tuple(len(c) for c in axes) or min(k.shape[2:]) < 1
                or not np.isfinite(k).all() or (k < 0).any()):
            raise ValueError("Supply nonnegative finite kernels with axes field_X,field_Y,kernel_X,kernel_Y[,kernel_Z]")
        gains = k.sum(axis=tuple(range(2, k.ndim)))
        if not np.isfinite(gains).all() or (gains <= 0).any():
            raise ValueError("Every local PSF must have positive finite energy")
        pitch = tuple(float(v) for v in self.voxel_size_um)
        if len(pitch) != k.ndim - 2 or not np.isfinite(pitch).all() or min(pitch) <= 0:
            raise ValueError("Specify one positive voxel pitch per kernel dimension")
        if not np.isfinite(self.wavelength_nm) or self.wavelength_nm <= 0:
            raise ValueError("wavelength_nm must be positive and finite")
        if self.operator not in ("detection", "excitation"):
            raise ValueError("Declare operator='detection' or operator='excitation' explicitly")
        meta = json.loads(json.dumps(self.provenance, allow_nan=False))
        for a in (k, *axes):
            a.setflags(write=False)
        object.__setattr__(self, "kernels", k)
        object.__setattr__(self, "x_um", axes[0])
        object.__setattr__(self, "y_um", axes[1])
        object.__setattr__(self, "voxel_size_um", pitch)
        object.__setattr__(self, "provenance", meta)

    def save(self, path):
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(path, schema=SCHEMA, kernels=self.kernels, x_um=self.x_um, y_um=self.y_um,
                            voxel_size_um=self.voxel_size_um, wavelength_nm=self.wavelength_nm,
                            operator=self.operator, provenance=json.dumps(self.provenance, allow_nan=False))

    @classmethod
    def load(cls, path):
        with np.load(path, allow_pickle=False) as d:
            if str(d["schema"]) != SCHEMA:
                raise ValueError("Unsupported full-field PSF schema")
            return cls(d["kernels"], d["x_um"], d["y_um"], tuple(d["voxel_size_um"]), float(d["wavelength_nm"]),
                       str(d["operator"]), json.loads(str(d["provenance"])))
