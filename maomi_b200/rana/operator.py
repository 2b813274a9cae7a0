"""Spatially varying local-PSF operator on the GPU: ``RanaOperator``.

Drop-in for maomi/rana/operator.py:20-167 (constructor, ``static``,
``scan_slab``, ``clear_cache``, ``cache_info``, ``physical_tail``, and the
attributes the movie and adapter code read: ``bank``, ``fields``, ``field``,
``kernel_shape``, ``voxel_size_um``, ``origin_um``, ``z_origin_um``,
``native``, ``device``, ``settings``).

How it renders:

* lateral weights: every output pixel centre gets the C1 smoothstep hat
  weights t^2 (3 - 2 t) of the two nodes bracketing it on each axis
  (maomi/rana/operator.py:10-17), so at most 2 x 2 node pairs act per pixel;
* depth weights: the fields of a ``DepthPSFBank`` are mixed linearly in the
  depth of each plane centre (operator.py:91-97);
* ``static``: ONE ``mm_local_render`` launch for the whole bank, the depth
  weights applied per output plane (excitation / native) or per source plane
  (detection) inside the kernel, then the result clipped at zero;
* ``scan_slab``: per field a plane-mode render of the slab, the kernels
  mirrored in depth for detection and binned by ``scan_avg``
  (operator.py:136-167).

Arithmetic is FP64 throughout, as in the reference.
"""

import numpy as np

from ._backends import get_backend
from ._fft import DeviceRender
from .depth import DepthPSFBank, depth_weights
from .fields import FullFieldPSF

_COVER_TOL = 1e-10


def _axis_weights(nodes, positions):
    """(len(nodes), len(positions)) smoothstep hat weights: a position between
    nodes a and a+1 at fraction t gives node a 1 - s(t) and node a+1 s(t),
    s(t) = t^2 (3 - 2 t); positions beyond the end nodes clamp to them."""
    nodes = np.asarray(nodes, float)
    pos = np.asarray(positions, float)
    a = np.searchsorted(nodes, pos, side="right") - 1
    a = np.minimum(np.maximum(a, 0), len(nodes) - 2)
    t = (pos - nodes[a]) / (nodes[a + 1] - nodes[a])
    t = np.minimum(np.maximum(t, 0.0), 1.0)
    s = t * t * (3 - 2 * t)
    w = np.zeros((len(nodes), len(pos)))
    col = np.arange(len(pos))
    w[a, col] = 1 - s
    w[a + 1, col] = s
    return w


def resolve_field(source):
    """A FullFieldPSF / DepthPSFBank, or what a provider's build_field() returns."""
    if isinstance(source, (FullFieldPSF, DepthPSFBank)):
        return source
    build = getattr(source, "build_field", None)
    if not callable(build):
        raise TypeError("expected a FullFieldPSF, a DepthPSFBank or a provider with build_field()")
    built = build()
    if not isinstance(built, (FullFieldPSF, DepthPSFBank)):
        raise TypeError("a provider's build_field() must return a FullFieldPSF or a DepthPSFBank")
    return built


def _mirror_depth(kernels, center):
    """Kernel planes reflected about ``center`` (plane p takes plane
    2*center - p); planes whose mirror falls outside the kernel are zero."""
    out = np.zeros_like(kernels)
    kz = kernels.shape[-1]
    for p in range(kz):
        src = 2 * center - p
        if 0 <= src < kz:
            out[..., p] = kernels[..., src]
    return out


def _bin_planes(a, width):
    """Sums over consecutive groups of ``width`` planes of the last axis."""
    return np.stack([a[..., s:s + width].sum(-1) for s in range(0, a.shape[-1], width)], -1)


class RanaOperator:
    def __init__(self, field, *, native=False, origin_um=(0., 0.), z_origin_um=0., device="cuda"):
        source = resolve_field(field)
        if isinstance(source, DepthPSFBank):
            self.bank, self.fields = source, tuple(source.fields)
        else:
            self.bank, self.fields = None, (source,)
        if not all(isinstance(f, FullFieldPSF) and f.kernels.ndim == 5 for f in self.fields):
            raise TypeError("the local operator renders XYZ kernels only (FullFieldPSF with 5-D kernels)")
        self.field = self.fields[0]
        self.kernel_shape = self.field.kernels.shape[2:]
        self.voxel_size_um = self.field.voxel_size_um
        self.origin_um = np.asarray(origin_um, dtype=float)
        self.z_origin_um = float(z_origin_um)
        if self.origin_um.shape != (2,) or not np.all(np.isfinite(self.origin_um)) or not np.isfinite(self.z_origin_um):
            raise ValueError("origin_um needs two finite values and z_origin_um one")
        self.native, self.device = bool(native), str(device)
        self._backend = get_backend(self.device)
        self._lateral = {}      # (X, Y) -> host weight tables (wx, wy)
        self._static = {}       # volume shape -> DeviceRender of the whole bank
        self._planes = {}       # (shape, field, scan_avg, detection) -> DeviceRender of one field
        self._reuses = 0
        mode = "native_scan" if self.native else self.field.operator
        self.settings = {
            "enabled": True, "operator": mode,
            "interpolation": "positive local cubic tensor weights",
            "field_nodes": list(self.field.kernels.shape[:2]), "kernel_shape": list(self.kernel_shape),
            "depth_nodes_um": None if self.bank is None else self.bank.depths_um.tolist(),
            "shared_psf_fallback": False, "device": self.device,
            "renderer": "maomi_b200 mm_local_render (FP64 direct sum over the active node pairs)",
            "provenance": [f.provenance for f in self.fields],
        }

    # --------------------------------------------------------------- weights
    @property
    def _detection(self):
        return self.field.operator == "detection" and not self.native

    @property
    def _correlate(self):
        return self.field.operator == "excitation" and not self.native

    def _weights(self, shape):
        """Lateral hat weights of the pixel centres of an (X, Y, ...) volume."""
        key = tuple(int(v) for v in shape[:2])
        if key not in self._lateral:
            pitch = np.asarray(self.voxel_size_um[:2], float)
            nodes = (self.field.x_um, self.field.y_um)
            lo = np.array([n[0] for n in nodes])
            hi = np.array([n[-1] for n in nodes])
            end = self.origin_um + np.asarray(key) * pitch
            if np.any(self.origin_um < lo - _COVER_TOL) or np.any(end > hi + _COVER_TOL):
                raise ValueError("the PSF field's nodes must cover the whole acquisition field of view")
            centres = [o + (np.arange(n) + 0.5) * p for o, n, p in zip(self.origin_um, key, pitch)]
            self._lateral[key] = tuple(_axis_weights(nd, c) for nd, c in zip(nodes, centres))
        return self._lateral[key]

    def _depth_weights(self, z_um):
        """(fields, planes) depth weights of plane centres at ``z_um``."""
        z = np.atleast_1d(np.asarray(z_um, float))
        if self.bank is None:
            return np.ones((1, z.size))
        d = self.bank.depths_um
        if np.any(z < d[0] - _COVER_TOL) or np.any(z > d[-1] + _COVER_TOL):
            raise ValueError("the depth bank does not span the requested plane depths")
        return depth_weights(d, z)

    def _plane_centres(self, first, count):
        return self.z_origin_um + (first + np.arange(count) + 0.5) * self.voxel_size_um[2]

    # ----------------------------------------------------------------- cache
    def clear_cache(self):
        """Drop the device-resident kernels, weights and workspaces."""
        self._static.clear()
        self._planes.clear()
        self._lateral.clear()

    @property
    def cache_info(self):
        renders = list(self._static.values()) + list(self._planes.values())
        return dict(plans=len(renders), fft_bytes=0, kernel_fft_builds=0, cache_hits=self._reuses)

    def _cached(self, table, key, build):
        if key in table:
            self._reuses += 1
        else:
            table[key] = build()
        return table[key]

    # ------------------------------------------------------------------ maths
    @staticmethod
    def physical_tail(values):
        """Clip negative ringing of a tail intensity to zero and rescale the rest
        so the integrated gain is unchanged; the input must be real, finite and
        of positive total."""
        a = np.asarray(values)
        total = a.sum(dtype=float) if not np.iscomplexobj(a) else np.nan
        if np.iscomplexobj(a) or not np.all(np.isfinite(a)) or not total > 0:
            raise ValueError("a tail intensity must be real and finite with a positive integrated gain")
        if not np.any(a < 0):
            return a
        kept = np.maximum(a, 0)
        return kept * (total / kept.sum(dtype=float))

    @staticmethod
    def _density(volume):
        if np.iscomplexobj(volume):
            raise ValueError("fluorescence must be a real density")
        a = np.asarray(volume, dtype=float)
        if a.ndim != 3 or not np.all(np.isfinite(a)) or np.any(a < 0):
            raise ValueError("fluorescence must be a finite, nonnegative (X, Y, Z) volume")
        return a

    def _finish(self, result):
        return np.maximum(self._backend.to_numpy(result), 0.0)

    # ------------------------------------------------------------ rendering
    def static(self, volume):
        """Render a whole volume: every plane through the depth-weighted fields."""
        a = self._density(volume)
        wz = self._depth_weights(self._plane_centres(0, a.shape[2]))

        def build():
            wx, wy = self._weights(a.shape)
            kern = np.stack([f.kernels for f in self.fields])
            return DeviceRender(a.shape, kern, wx, wy, plane=False, detection=self._detection,
                                correlate=self._correlate, device=self.device)

        render = self._cached(self._static, a.shape, build)
        b = self._backend
        out = b.zeros(a.shape)
        render(b.array(a), zweight=wz if self.bank is not None else None, out=out)
        return self._finish(out)

    def scan_slab(self, slab, *, z_start=0, scan_avg=1):
        """Image of one focal slab (depth = kernel depth) starting at plane
        ``z_start``: the 2-D operator summed over the slab's planes, averaged
        in groups of ``scan_avg`` planes."""
        a = self._density(slab)
        kz = self.kernel_shape[2]
        if a.shape[2] != kz:
            raise ValueError(f"the slab must have the kernel's depth ({kz} planes), got {a.shape[2]}")
        if isinstance(scan_avg, bool) or not isinstance(scan_avg, (int, np.integer)) or scan_avg < 1:
            raise ValueError("scan_avg must be a positive integer")
        width = int(scan_avg)
        centre = kz // 2
        z = self._plane_centres(z_start, kz)
        detect = self._detection
        # detection weights each source plane by its own depth; excitation and
        # native scans weight the whole slab by the depth of its centre plane
        wz = self._depth_weights(z if detect else z[centre:centre + 1])
        b = self._backend
        src = b.array(a)
        out = b.zeros(a.shape[:2])
        wx, wy = self._weights(a.shape)
        for index, (f, w) in enumerate(zip(self.fields, wz)):
            if not np.any(w):
                continue
            source = src * b.array(w) if detect else src
            if width > 1:
                source = b.group_sum(source, range(0, kz, width), width)
            nz = int(source.shape[2])

            def build(f=f):
                k = _mirror_depth(f.kernels, centre) if detect else f.kernels
                if width > 1:
                    k = _bin_planes(k, width)
                return DeviceRender((a.shape[0], a.shape[1], nz), k[None], wx, wy, plane=True,
                                    detection=detect, correlate=self._correlate, device=self.device)

            render = self._cached(self._planes, (a.shape, index, width, detect), build)
            piece = render(source)
            out += piece if detect else piece * float(w[0])
        return self._finish(out)
