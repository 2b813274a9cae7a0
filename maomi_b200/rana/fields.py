"""Local-PSF fields as data: ``FullFieldPSF`` (maomi/rana/fields.py:17-110).

A field holds one effective-intensity kernel per lateral node of a
rectilinear grid: ``kernels`` has axes (node_x, node_y, kernel_x, kernel_y
[, kernel_z]), each kernel's origin at ``shape // 2``, node positions and
voxel pitches in specimen micrometres.  The renderers rely on this contract,
so it is enforced when a field is built:

* kernels are real, finite, nonnegative float64 and every local kernel has a
  positive total gain (no normalisation is ever applied);
* the node axes strictly increase, with at least two nodes each;
* one positive pitch per kernel axis, a positive wavelength;
* ``operator`` says how the kernels act: "detection" (weights on the source
  side, convolution) or "excitation" (weights on the scan side, correlation).

Files use the ``maomi.full_field_psf.v1`` npz layout, so a bank written by
either implementation loads in the other.
"""

import json
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

SCHEMA = "maomi.full_field_psf.v1"
OPERATORS = ("detection", "excitation")


def node_axis(values, what="node axis"):
    """Float64 copy of a node coordinate axis; >= 2 strictly increasing finite values."""
    a = np.array(values, dtype=float, copy=True)
    if a.ndim != 1 or a.size < 2 or not np.all(np.isfinite(a)) or not np.all(a[1:] > a[:-1]):
        raise ValueError(f"{what}: a full-field PSF needs at least two strictly increasing finite positions "
                         "per lateral axis")
    return a


def intensity_kernels(kernels, nodes):
    """Float64 copy of the kernel array, checked against the node counts."""
    if np.iscomplexobj(kernels):
        raise ValueError("kernels must be real effective intensities (got a complex field)")
    k = np.array(kernels, dtype=np.float64, copy=True)
    if k.ndim not in (4, 5) or k.shape[:2] != tuple(nodes) or min(k.shape[2:], default=0) < 1:
        raise ValueError(f"kernels need axes (node_x, node_y, kernel_x, kernel_y[, kernel_z]) with {nodes} nodes; "
                         f"got shape {k.shape}")
    if not np.all(np.isfinite(k)) or np.any(k < 0):
        raise ValueError("kernels must be finite and nonnegative")
    gain = k.reshape(k.shape[0], k.shape[1], -1).sum(-1)
    if not np.all(np.isfinite(gain)) or np.any(gain <= 0):
        raise ValueError("each local kernel needs a positive finite total gain")
    return k


def _pitch(voxel_size_um, dims):
    try:
        p = tuple(float(v) for v in voxel_size_um)
    except TypeError:
        raise ValueError("voxel_size_um must list one pitch per kernel axis") from None
    if len(p) != dims or not all(np.isfinite(v) and v > 0 for v in p):
        raise ValueError(f"voxel_size_um must hold {dims} positive finite pitches")
    return p


def _frozen(*arrays):
    for a in arrays:
        a.setflags(write=False)


@dataclass(frozen=True)
class FullFieldPSF:
    """Effective local kernels on a lateral node grid (see the module docstring)."""

    kernels: np.ndarray
    x_um: np.ndarray
    y_um: np.ndarray
    voxel_size_um: tuple
    wavelength_nm: float
    operator: str
    provenance: dict = field(default_factory=dict)

    def __post_init__(self):
        x, y = node_axis(self.x_um, "x_um"), node_axis(self.y_um, "y_um")
        k = intensity_kernels(self.kernels, (x.size, y.size))
        pitch = _pitch(self.voxel_size_um, k.ndim - 2)
        wl = float(self.wavelength_nm)
        if not (np.isfinite(wl) and wl > 0):
            raise ValueError("wavelength_nm must be a positive finite number")
        if self.operator not in OPERATORS:
            raise ValueError(f"operator must be one of {OPERATORS}, stated explicitly")
        # provenance must survive a JSON round trip (it is stored as text)
        meta = json.loads(json.dumps(self.provenance, allow_nan=False))
        _frozen(k, x, y)
        for name, value in (("kernels", k), ("x_um", x), ("y_um", y), ("voxel_size_um", pitch),
                            ("provenance", meta)):
            object.__setattr__(self, name, value)

    # ----------------------------------------------------------- builders
    @classmethod
    def from_psf_field(cls, psf_field, *, operator, gains=None):
        """Field from a 2-D PSF field object (``intensity`` (node_x, node_y, kx,
        ky), ``x_um``, ``y_um``, ``pixel_size_um``, ``wavelength_nm``,
        ``provenance``), whose per-node PSFs are unit-sum shapes: ``gains``
        (node_x, node_y) restores their energies, unit gains when omitted.
        Counterpart of maomi/rana/fields.py:67-81."""
        needed = ("intensity", "x_um", "y_um", "pixel_size_um", "wavelength_nm")
        if not all(hasattr(psf_field, a) for a in needed) or np.ndim(psf_field.intensity) != 4:
            raise TypeError("from_psf_field needs a PSF field (per-node 2-D intensities), not a shared PSF")
        nodes = np.shape(psf_field.intensity)[:2]
        g = np.ones(nodes) if gains is None else np.asarray(gains, dtype=float)
        if g.shape != nodes or not np.all(np.isfinite(g)) or np.any(g <= 0):
            raise ValueError(f"gains must be {nodes} positive finite values, one per node")
        meta = {"source": getattr(psf_field, "provenance", {}),
                "gain_source": "unit gains" if gains is None else "explicit node gains"}
        return cls(np.asarray(psf_field.intensity) * g[:, :, None, None], psf_field.x_um, psf_field.y_um,
                   psf_field.pixel_size_um, psf_field.wavelength_nm, operator, meta)

    @classmethod
    def from_provider(cls, provider, x_um, y_um, *, voxel_size_um, wavelength_nm, operator, provenance=None):
        """Field sampled from ``provider(x_um, y_um) -> kernel`` at every node,
        taken as returned (no renormalisation).  maomi/rana/fields.py:83-94."""
        x, y = node_axis(x_um, "x_um"), node_axis(y_um, "y_um")
        grid = np.array([[np.asarray(provider(float(a), float(b))) for b in y] for a in x])
        return cls(grid, x, y, voxel_size_um, wavelength_nm, operator, dict(provenance or {}))

    # ---------------------------------------------------------------- files
    def save(self, path):
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(path, schema=SCHEMA, kernels=self.kernels, x_um=self.x_um, y_um=self.y_um,
                            voxel_size_um=self.voxel_size_um, wavelength_nm=self.wavelength_nm,
                            operator=self.operator, provenance=json.dumps(self.provenance, allow_nan=False))

    @classmethod
    def load(cls, path):
        with np.load(path, allow_pickle=False) as d:
            found = str(d["schema"]) if "schema" in d.files else "<none>"
            if found != SCHEMA:
                raise ValueError(f"not a {SCHEMA} file (schema {found})")
            return cls(d["kernels"], d["x_um"], d["y_um"], tuple(d["voxel_size_um"]), float(d["wavelength_nm"]),
                       str(d["operator"]), json.loads(str(d["provenance"])))
