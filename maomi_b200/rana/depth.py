"""Depth-dependent PSF bank (maomi/rana/depth.py:9-69): one complete XYZ
FullFieldPSF per focal depth, linear depth weights, ``maomi.depth_psf_bank.v1``."""

import json
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .fields import FullFieldPSF

SCHEMA = "maomi.depth_psf_bank.v1"


@dataclass(frozen=True)
class DepthPSFBank:
    depths_um: np.ndarray
    fields: tuple

    def __post_init__(self):
        z = np.array(self.depths_um, dtype=float, copy=True)
        fields = tuple(self.fields)
        if z.ndim != 1 or len(z) < 2 or (np.diff(z) <= 0).any() or not np.isfinite(z).all() or (z < 0).any():
            raise ValueError("A depth bank requires >= 2 increasing nonnegative finite depths")
        if len(fields) != len(z) or any(not isinstance(f, FullFieldPSF) or f.kernels.ndim != 5 for f in fields):
            raise ValueError("One complete XYZ-kernel FullFieldPSF per depth is required")
        first = fields[0]
        for f in fields[1:]:
            if (f.kernels.shape != first.kernels.shape or f.voxel_size_um != first.voxel_size_um
                    or f.operator != first.operator or f.wavelength_nm != first.wavelength_nm
                    or not np.array_equal(f.x_um, first.x_um) or not np.array_equal(f.y_um, first.y_um)):
                raise ValueError("Depth fields must share shape, XY nodes, pitch, operator and wavelength")
        z.setflags(write=False)
        object.__setattr__(self, "depths_um", z)
        object.__setattr__(self, "fields", fields)

    @property
    def voxel_size_um(self):
        return self.fields[0].voxel_size_um

    @property
    def operator(self):
        return self.fields[0].operator

    @property
    def wavelength_nm(self):
        return self.fields[0].wavelength_nm

    def save(self, path):
        p = Path(path)
        p.parent.mkdir(parents=True, exist_ok=True)
        f = self.fields[0]
        np.savez_compressed(p, schema=SCHEMA, depths_um=self.depths_um,
                            kernels=np.stack([x.kernels for x in self.fields]), x_um=f.x_um, y_um=f.y_um,
                            voxel_size_um=f.voxel_size_um, wavelength_nm=f.wavelength_nm, operator=f.operator,
                            provenance=json.dumps([x.provenance for x in self.fields], allow_nan=False))

    @classmethod
    def load(cls, path):
        with np.load(path, allow_pickle=False) as d:
            if str(d["schema"]) != SCHEMA:
                raise ValueError("Unsupported depth-bank schema")
            meta = json.loads(str(d["provenance"]))
            if len(meta) != len(d["depths_um"]) or len(d["kernels"]) != len(d["depths_um"]):
                raise ValueError("Malformed depth bank: inconsistent depth, kernel or provenance counts")
            return cls(d["depths_um"], tuple(
                FullFieldPSF(k, d["x_um"], d["y_um"], tuple(d["voxel_size_um"]), float(d["wavelength_nm"]),
                             str(d["operator"]), m) for k, m in zip(d["kernels"], meta)))
