"""``LocalFFTPlan`` drop-in (maomi/rana/_fft.py:8-99) on the GPU.

Same constructor and call: ``LocalFFTPlan(shape, kernels, weights, plane=...,
detection=..., correlate=..., device=...)(source)``.  The reference overlap-adds
zero-padded FFT convolutions of the tiles around every node pair; the result
is the direct sum over the compact supports, which ``mm_local_render``
evaluates in FP64 in one launch (no spectra, so the spectrum cache is empty
and ``stats['kernel_fft_builds']`` stays 0)."""

import numpy as np

from .. import _lib
from ._backends import get_backend


def render(desc_args, source, out, zweight=None):
    """Launch mm_local_render; ``out`` (device float64) is accumulated into."""
    kern, wx, wy, detection, correlate, plane = desc_args
    d = _lib.LocalDesc()
    sx, sy, sz = source.shape
    d.sx, d.sy, d.sz = sx, sy, sz
    d.kx, d.ky, d.kz = kern.shape[2:5]
    d.nodes_x, d.nodes_y = kern.shape[:2]
    d.kernels, d.wx, d.wy = kern.data_ptr(), wx.data_ptr(), wy.data_ptr()
    d.detection, d.correlate, d.plane = int(detection), int(correlate), int(plane)
    zw = None if zweight is None else zweight.contiguous()
    _lib.check(_lib.load().mm_local_render(d, _lib.ptr(source.contiguous()), _lib.ptr(zw), _lib.ptr(out), None, 0,
                                            _lib.stream_of(source.device)), "local render")
    return out


class LocalFFTPlan:
    def __init__(self, shape, kernels, weights, *, plane, detection, correlate, device, batch_size=8, cache_mb=256):
        self.shape = tuple(shape)
        self.plane, self.detection, self.correlate = bool(plane), bool(detection), bool(correlate)
        self.device, self.batch_size = device, batch_size
        self.backend = get_backend(device)
        k = np.asarray(kernels, dtype=np.float64)
        if k.ndim == 4:
            k = k[..., None]
        if k.ndim != 5:
            raise ValueError("kernels must have axes field_X, field_Y, kernel_X, kernel_Y[, kernel_Z]")
        if self.plane and k.shape[4] != self.shape[2]:
            raise ValueError("plane mode needs one kernel plane per source plane")
        wx, wy = weights
        if np.shape(wx) != (k.shape[0], self.shape[0]) or np.shape(wy) != (k.shape[1], self.shape[1]):
            raise ValueError("weights must be (nodes_x, X) and (nodes_y, Y)")
        self.kernels = kernels
        self._args = (self.backend.array(k), self.backend.array(wx), self.backend.array(wy),
                      self.detection, self.correlate, self.plane)
        self.cache_limit = int(cache_mb * 1024 ** 2)
        self.cache_bytes = 0
        self.stats = dict(kernel_fft_builds=0, cache_hits=0)

    def __call__(self, source, *, zweight=None, out=None):
        src = self.backend.array(source)
        if tuple(src.shape) != self.shape:
            raise ValueError(f"source must have shape {self.shape}")
        if out is None:
            out = self.backend.zeros(self.shape[:2] if self.plane else self.shape)
        self.stats["cache_hits"] += 1
        return render(self._args, src, out, None if zweight is None else self.backend.array(zweight))

    def clear(self):
        self.cache_bytes = 0
