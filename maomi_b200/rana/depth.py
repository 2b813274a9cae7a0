"""Depth banks of local-PSF fields: ``DepthPSFBank`` (maomi/rana/depth.py:9-69).

A bank pairs focal depths (micrometres, >= 0, strictly increasing, at least
two) with one complete XYZ ``FullFieldPSF`` per depth.  All fields must be
interchangeable apart from their kernel values: same kernel shape, lateral
nodes, pitch, operator and wavelength.  A renderer weights the fields
linearly in depth (``depth_weights``).  Files use ``maomi.depth_psf_bank.v1``.
"""

import json
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .fields import FullFieldPSF

SCHEMA = "maomi.depth_psf_bank.v1"


def _same_layout(a, b):
    return (a.kernels.shape == b.kernels.shape and a.voxel_size_um == b.voxel_size_um and a.operator == b.operator
            and a.wavelength_nm == b.wavelength_nm and np.array_equal(a.x_um, b.x_um)
            and np.array_equal(a.y_um, b.y_um))


def depth_weights(depths_um, z_um):
    """Linear interpolation weights (len(depths), len(z)) between the two
    depth nodes bracketing each plane centre: the hat functions of the depth
    nodes, so every column sums to one and has at most two nonzero entries.
    The planes must lie within [depths[0], depths[-1]]."""
    d = np.asarray(depths_um, float)
    z = np.atleast_1d(np.asarray(z_um, float))
    hats = np.eye(len(d))
    return np.stack([np.interp(z, d, hats[k]) for k in range(len(d))])


@dataclass(frozen=True)
class DepthPSFBank:
    depths_um: np.ndarray
    fields: tuple

    def __post_init__(self):
        z = np.array(self.depths_um, dtype=float, copy=True)
        fields = tuple(self.fields)
        if z.ndim != 1 or z.size < 2 or not np.all(np.isfinite(z)) or np.any(z < 0) or not np.all(z[1:] > z[:-1]):
            raise ValueError("depths_um: a bank needs at least two strictly increasing, finite, nonnegative depths")
        if len(fields) != z.size:
            raise ValueError(f"{z.size} depths but {len(fields)} fields: give one field per depth")
        if not all(isinstance(f, FullFieldPSF) and f.kernels.ndim == 5 for f in fields):
            raise ValueError("every depth needs a FullFieldPSF with XYZ kernels")
        if not all(_same_layout(fields[0], f) for f in fields[1:]):
            raise ValueError("the fields of a bank must agree in kernel shape, lateral nodes, pitch, operator "
                             "and wavelength")
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

    @classmethod
    def from_provider(cls, provider, x_um, y_um, depths_um, *, voxel_size_um, wavelength_nm, operator="excitation",
                      provenance=None):
        """Bank sampled from ``provider(x_um, y_um, depth_um) -> kernel``; each
        field's provenance records its focal depth.  maomi/rana/depth.py:44-48."""
        def at_depth(depth):
            return FullFieldPSF.from_provider(lambda x, y: provider(x, y, depth), x_um, y_um,
                                              voxel_size_um=voxel_size_um, wavelength_nm=wavelength_nm,
                                              operator=operator,
                                              provenance=dict(provenance or {}, focal_depth_um=depth))
        return cls(depths_um, tuple(at_depth(float(d)) for d in np.asarray(depths_um, float)))

    def save(self, path):
        p = Path(path)
        p.parent.mkdir(parents=True, exist_ok=True)
        head = self.fields[0]
        np.savez_compressed(p, schema=SCHEMA, depths_um=self.depths_um,
                            kernels=np.stack([f.kernels for f in self.fields]), x_um=head.x_um, y_um=head.y_um,
                            voxel_size_um=head.voxel_size_um, wavelength_nm=head.wavelength_nm,
                            operator=head.operator,
                            provenance=json.dumps([f.provenance for f in self.fields], allow_nan=False))

    @classmethod
    def load(cls, path):
        with np.load(path, allow_pickle=False) as d:
            found = str(d["schema"]) if "schema" in d.files else "<none>"
            if found != SCHEMA:
                raise ValueError(f"not a {SCHEMA} file (schema {found})")
            meta = json.loads(str(d["provenance"]))
            count = len(d["depths_um"])
            if len(meta) != count or len(d["kernels"]) != count:
                raise ValueError(f"malformed depth bank: {count} depths, {len(d['kernels'])} kernel sets, "
                                 f"{len(meta)} provenance records")
            common = (d["x_um"], d["y_um"], tuple(d["voxel_size_um"]), float(d["wavelength_nm"]), str(d["operator"]))
            return cls(d["depths_um"], tuple(FullFieldPSF(k, *common, m) for k, m in zip(d["kernels"], meta)))


class DepthFullFieldRenderer:
    """Cubic XY fields with linear focal-depth weights (maomi/rana/depth.py:72-104).

    One ``CubicFullFieldRenderer`` per depth field; detection weights the
    source planes before the convolution, excitation weights the image planes
    after the correlation.  The depth sum runs on the device; fields whose
    depth weights are all zero are skipped."""

    def __init__(self, bank, shape, *, voxel_size_um, origin_um=(0., 0.), z_origin_um=0., device="cuda"):
        from .cubic import CubicFullFieldRenderer
        if not isinstance(bank, DepthPSFBank) or len(shape) != 3:
            raise TypeError("Depth rendering requires DepthPSFBank and an XYZ volume")
        if not np.isfinite(z_origin_um):
            raise ValueError("z_origin_um must be finite")
        end = z_origin_um + shape[2] * voxel_size_um[2]
        if z_origin_um < bank.depths_um[0] or end > bank.depths_um[-1]:
            raise ValueError("Depth bank must cover the entire Z extent including edges")
        self.bank, self.shape = bank, tuple(shape)
        z = z_origin_um + (np.arange(shape[2]) + .5) * voxel_size_um[2]
        self.weights = depth_weights(bank.depths_um, z)
        self.renderers = [CubicFullFieldRenderer(f, shape, voxel_size_um=voxel_size_um, origin_um=origin_um,
                                                 device=device) for f in bank.fields]
        self.device = self.renderers[0].device
        self.validation = {"depth_nodes_um": bank.depths_um.tolist(), "checked_xyz_positions": int(np.prod(shape)),
                           "shared_psf_fallback": False, "depth_interpolation": "positive linear",
                           "fields": [r.validation for r in self.renderers]}

    def __call__(self, density):
        import torch
        from .. import _lib
        src = (density.to(device=self.device, dtype=torch.float64) if isinstance(density, torch.Tensor)
               else _lib.upload(np.asarray(density, dtype=float), self.device))
        result = torch.zeros(self.shape, dtype=torch.float64, device=self.device)
        for w, renderer in zip(self.weights, self.renderers):
            if not np.any(w):
                continue
            wd = torch.as_tensor(w, dtype=torch.float64, device=self.device)[None, None, :]
            if self.bank.operator == "detection":
                result += _checked(renderer, src * wd)
            else:
                result += _checked(renderer, src) * wd
        return result.cpu().numpy()


def _checked(renderer, src):
    """One field's image with the single-field renderer's input and output checks."""
    import torch
    if (tuple(src.shape) != renderer.shape or not bool(torch.isfinite(src).all()) or bool((src < 0).any())):
        raise ValueError("Density must be finite, nonnegative and match the prepared shape")
    return renderer.render_device(src)
