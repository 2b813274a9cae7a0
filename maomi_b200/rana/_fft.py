"""``LocalFFTPlan`` drop-in (maomi/rana/_fft.py:8-99) over ``mm_local_render``.

The reference overlap-adds zero-padded FFT convolutions of the source tiles
around every node pair.  Zero padding to the linear-convolution length makes
that equal to the direct sum over each pair's compact support, which
``mm_local_render`` evaluates in FP64.  The plan construction of the
reference (node supports, tile bounds) becomes the lateral tile tables of
``mm_local_tiles``.  No kernel spectra exist, so the spectrum cache stays
empty: ``stats['kernel_fft_builds']`` is 0 and ``cache_bytes`` 0;
``stats['cache_hits']`` counts calls that reused the device-resident plan.
"""

import numpy as np

from .. import _lib
from ._backends import get_backend

TILE_INTS = 8


def lateral_tiles(weights):
    """mm_local_tiles of a (nodes, n) host weight table: int32 (tiles, 8)."""
    w = np.ascontiguousarray(weights, dtype=np.float64)
    nodes, n = w.shape
    table = np.zeros((n, TILE_INTS), np.int32)
    count = _lib.load().mm_local_tiles(_lib.c_void_p(w.ctypes.data), nodes, n, 0,
                                       _lib.c_void_p(table.ctypes.data), n)
    if count < 0:
        _lib.check(count, "mm_local_tiles")
    return table[:count].copy()


class DeviceRender:
    """Device-resident inputs of one ``mm_local_render`` configuration: the
    kernels of one field or of a whole depth bank (nfields, nodes_x, nodes_y,
    kx, ky, kz), lateral weights, tile tables and the transpose workspace."""

    def __init__(self, shape, kernels, wx, wy, *, plane, detection, correlate, device):
        self.shape = tuple(int(v) for v in shape)
        self.plane, self.detection, self.correlate = bool(plane), bool(detection), bool(correlate)
        self.backend = get_backend(device)
        k = np.asarray(kernels, dtype=np.float64)
        if k.ndim != 6:
            raise ValueError("kernels must have axes field, node_x, node_y, kernel_x, kernel_y, kernel_z")
        sx, sy, sz = self.shape
        if np.shape(wx) != (k.shape[1], sx) or np.shape(wy) != (k.shape[2], sy):
            raise ValueError(f"weights must be ({k.shape[1]}, {sx}) and ({k.shape[2]}, {sy})")
        if self.plane and k.shape[5] != sz:
            raise ValueError("plane mode needs one kernel plane per source plane")
        self.nfields = k.shape[0]
        self.kernel_shape = k.shape[3:]
        b = self.backend
        self.kernels = b.array(k)
        self.wx, self.wy = b.array(wx), b.array(wy)
        self.tiles = None
        if not self.detection:
            self.tiles = [b.torch.as_tensor(lateral_tiles(w), device=b.device) for w in (wx, wy)]
        self.desc = self._desc()
        nbytes = _lib.load().mm_local_render_workspace_size(self.desc)
        self.workspace = b.torch.empty(max(nbytes, 8), dtype=b.torch.uint8, device=b.device)

    def _desc(self):
        d = _lib.LocalDesc()
        d.sx, d.sy, d.sz = self.shape
        d.kx, d.ky, d.kz = self.kernel_shape
        d.nodes_x, d.nodes_y = self.kernels.shape[1:3]
        d.kernels, d.wx, d.wy = self.kernels.data_ptr(), self.wx.data_ptr(), self.wy.data_ptr()
        d.detection, d.correlate, d.plane = int(self.detection), int(self.correlate), int(self.plane)
        d.nfields = self.nfields
        if self.tiles is not None:
            d.tiles_x, d.ntiles_x = self.tiles[0].data_ptr(), self.tiles[0].shape[0]
            d.tiles_y, d.ntiles_y = self.tiles[1].data_ptr(), self.tiles[1].shape[0]
        return d

    def __call__(self, source, *, zweight=None, out=None):
        """Accumulate the render of ``source`` (device float64 (sx, sy, sz))
        into ``out`` (zeros when omitted); ``zweight`` (nfields, sz)."""
        b = self.backend
        src = b.array(source)
        if tuple(src.shape) != self.shape:
            raise ValueError(f"source must have shape {self.shape}, got {tuple(src.shape)}")
        if out is None:
            out = b.zeros(self.shape[:2] if self.plane else self.shape)
        zw = None
        if zweight is not None:
            zw = b.array(np.asarray(zweight, np.float64).reshape(self.nfields, self.shape[2]))
        _lib.check(_lib.load().mm_local_render(self.desc, _lib.ptr(src), _lib.ptr(zw), _lib.ptr(out),
                                                _lib.ptr(self.workspace), self.workspace.numel(),
                                                _lib.stream_of(src.device)), "local render")
        return out


class LocalFFTPlan:
    """Same constructor and call as the reference's plan; one field."""

    def __init__(self, shape, kernels, weights, *, plane, detection, correlate, device, batch_size=8, cache_mb=256):
        self.shape = tuple(shape)
        self.plane, self.detection, self.correlate = bool(plane), bool(detection), bool(correlate)
        self.device, self.batch_size = device, batch_size
        self.kernels = kernels
        k = np.asarray(kernels, dtype=np.float64)
        if k.ndim == 4:
            k = k[..., None]
        if k.ndim != 5:
            raise ValueError("kernels must have axes node_x, node_y, kernel_x, kernel_y[, kernel_z]")
        wx, wy = weights
        self._render = DeviceRender(self.shape, k[None], wx, wy, plane=plane, detection=detection,
                                    correlate=correlate, device=device)
        self.backend = self._render.backend
        self.cache_limit = int(cache_mb * 1024 ** 2)
        self.cache_bytes = 0
        self.stats = dict(kernel_fft_builds=0, cache_hits=0)
        self._calls = 0

    def __call__(self, source):
        self.stats["cache_hits"] += int(self._calls > 0)
        self._calls += 1
        return self._render(source)

    def clear(self):
        self.cache_bytes = 0
