"""``RanaOperator`` on the GPU (maomi/rana/operator.py:20-167).

The same node weights (C1 smoothstep hats between XY nodes, linear depth
weights), the same detection / excitation / native conventions and the same
``static`` and ``scan_slab`` entry points; every projection runs through
``mm_local_render`` in FP64, with the depth weight of a bank field applied
inside the render launch."""

from collections import OrderedDict

import numpy as np

from .depth import DepthPSFBank
from .fields import FullFieldPSF
from ._backends import get_backend
from ._fft import LocalFFTPlan


def _axis_weights(nodes, positions):
    """C1 smoothstep t^2(3-2t) between the two nodes bracketing each position."""
    ids = np.clip(np.searchsorted(nodes, positions, side="right") - 1, 0, len(nodes) - 2)
    t = np.clip((positions - nodes[ids]) / (nodes[ids + 1] - nodes[ids]), 0, 1)
    t = t * t * (3 - 2 * t)
    w = np.zeros((len(nodes), len(positions)))
    cols = np.arange(len(positions))
    w[ids, cols] = 1 - t
    w[ids + 1, cols] = t
    return w


def _resolve(field):
    if isinstance(field, (FullFieldPSF, DepthPSFBank)):
        return field
    build = getattr(field, "build_field", None)
    if not callable(build):
        raise TypeError("Supply FullFieldPSF, DepthPSFBank or a PSFProvider with build_field()")
    out = build()
    if not isinstance(out, (FullFieldPSF, DepthPSFBank)):
        raise TypeError("PSFProvider.build_field() must return FullFieldPSF or DepthPSFBank")
    return out


class RanaOperator:
    def __init__(self, field, *, native=False, origin_um=(0., 0.), z_origin_um=0., device="cuda"):
        field = _resolve(field)
        self.bank = field if isinstance(field, DepthPSFBank) else None
        self.fields = field.fields if self.bank is not None else (field,)
        if any(not isinstance(f, FullFieldPSF) or f.kernels.ndim != 5 for f in self.fields):
            raise TypeError("The acquisition add-on requires complete XYZ-kernel fields")
        self.field = self.fields[0]
        self.kernel_shape = self.field.kernels.shape[2:]
        self.voxel_size_um = self.field.voxel_size_um
        self.origin_um, self.z_origin_um = np.asarray(origin_um, float), float(z_origin_um)
        self.native, self.device = native, str(device)
        if (self.origin_um.shape != (2,) or not np.isfinite(self.origin_um).all()
                or not np.isfinite(self.z_origin_um)):
            raise ValueError("Supply finite XY and Z origins")
        self._backend = get_backend(self.device)
        self._cache = {}
        self._plans = OrderedDict()
        self._scan_kernels = {}
        self.settings = {"enabled": True, "operator": "native_scan" if native else self.field.operator,
                         "interpolation": "positive local cubic tensor weights",
                         "field_nodes": list(self.field.kernels.shape[:2]), "kernel_shape": list(self.kernel_shape),
                         "depth_nodes_um": None if self.bank is None else self.bank.depths_um.tolist(),
                         "shared_psf_fallback": False, "device": self.device,
                         "provenance": [f.provenance for f in self.fields]}

    @property
    def _detection(self):
        return not self.native and self.field.operator == "detection"

    @property
    def _correlate(self):
        return not self.native and self.field.operator == "excitation"

    def _weights(self, shape):
        shape = tuple(shape[:2])
        if shape not in self._cache:
            pitch = np.array(self.voxel_size_um[:2])
            lower = np.array([self.field.x_um[0], self.field.y_um[0]])
            upper = np.array([self.field.x_um[-1], self.field.y_um[-1]])
            if ((self.origin_um < lower - 1e-10).any()
                    or (self.origin_um + np.array(shape) * pitch > upper + 1e-10).any()):
                raise ValueError("RANA field must cover the entire acquisition FOV")
            coords = [o + (np.arange(n) + .5) * p for o, n, p in zip(self.origin_um, shape, pitch)]
            self._cache[shape] = tuple(_axis_weights(nodes, q)
                                       for nodes, q in zip((self.field.x_um, self.field.y_um), coords))
        return self._cache[shape]

    def _depth_weights(self, z):
        if self.bank is None:
            return np.ones((1, np.size(z)))
        z = np.atleast_1d(z)
        if (z < self.bank.depths_um[0] - 1e-10).any() or (z > self.bank.depths_um[-1] + 1e-10).any():
            raise ValueError("RANA depth bank does not cover the requested acquisition depths")
        return np.stack([np.interp(z, self.bank.depths_um, row) for row in np.eye(len(self.fields))])

    def clear_cache(self):
        self._plans.clear()
        self._scan_kernels.clear()
        self._cache.clear()

    @property
    def cache_info(self):
        names = ("kernel_fft_builds", "cache_hits")
        return dict(plans=len(self._plans), fft_bytes=sum(p.cache_bytes for p in self._plans.values()),
                    **{k: sum(p.stats[k] for p in self._plans.values()) for k in names})

    def _plan(self, shape, kernels, plane):
        key = (tuple(shape), id(kernels), plane)
        if key not in self._plans:
            limit = max(2, 2 * len(self.fields))
            while len(self._plans) >= limit:
                self._plans.popitem(last=False)[1].clear()
            self._plans[key] = LocalFFTPlan(shape, kernels, self._weights(shape), plane=plane,
                                            detection=self._detection, correlate=self._correlate,
                                            device=self.device, cache_mb=256 / limit)
        self._plans.move_to_end(key)
        return self._plans[key]

    def _finish(self, result):
        return np.maximum(self._backend.to_numpy(result), 0.)

    @staticmethod
    def physical_tail(values):
        """Remove negative intensity ringing without changing integrated gain."""
        a = np.asarray(values)
        if np.iscomplexobj(a) or not np.isfinite(a).all() or a.sum(dtype=float) <= 0:
            raise ValueError("Tail intensity must have positive finite integrated gain")
        if np.any(a < 0):
            positive = np.maximum(a, 0)
            return positive * (a.sum(dtype=float) / positive.sum(dtype=float))
        return a

    @staticmethod
    def _density(volume):
        if np.iscomplexobj(volume):
            raise ValueError("Fluorescence must be real")
        a = np.asarray(volume, dtype=float)
        if a.ndim != 3 or not np.isfinite(a).all() or (a < 0).any():
            raise ValueError("Supply finite nonnegative XYZ fluorescence")
        return a

    def static(self, volume):
        """Whole-volume render: detection weights sources per depth before the
        local convolution, excitation weights the local correlation after."""
        a = self._density(volume)
        z = self.z_origin_um + (np.arange(a.shape[2]) + .5) * self.voxel_size_um[2]
        weights = self._depth_weights(z)
        src = self._backend.array(a)
        result = self._backend.zeros(a.shape)
        for f, w in zip(self.fields, weights):
            if not np.any(w):
                continue
            self._plan(a.shape, f.kernels, False)(src, zweight=w, out=result)
        return self._finish(result)

    def scan_slab(self, slab, *, z_start=0, scan_avg=1):
        a = self._density(slab)
        if a.shape[2] != self.kernel_shape[2]:
            raise ValueError("Focal slab depth must match the RANA kernel")
        if not isinstance(scan_avg, (int, np.integer)) or scan_avg < 1:
            raise ValueError("scan_avg must be a positive integer")
        center = self.kernel_shape[2] // 2
        z = self.z_origin_um + (z_start + np.arange(a.shape[2]) + .5) * self.voxel_size_um[2]
        detection = self._detection
        weights = self._depth_weights(z if detection else [z[center]])
        starts = np.arange(0, a.shape[2], scan_avg)
        dev = self._backend.array(a)
        result = self._backend.zeros(a.shape[:2])
        for index, (f, w) in enumerate(zip(self.fields, weights)):
            if not np.any(w):
                continue
            source = dev * self._backend.array(w) if detection else dev
            key = (index, scan_avg, detection)
            if key not in self._scan_kernels:
                kernels = f.kernels
                if detection:
                    ids = 2 * center - np.arange(a.shape[2])
                    kernels = np.take(kernels, np.minimum(ids, a.shape[2] - 1), axis=-1).copy()
                    kernels[..., ids >= a.shape[2]] = 0
                if scan_avg > 1:
                    kernels = np.add.reduceat(kernels, starts, axis=-1)
                self._scan_kernels[key] = kernels
            if scan_avg > 1:
                source = self._backend.group_sum(source, starts, scan_avg)
            piece = self._plan(tuple(source.shape), self._scan_kernels[key], True)(source)
            result += piece * (1 if detection else float(w[0]))
        return self._finish(result)
