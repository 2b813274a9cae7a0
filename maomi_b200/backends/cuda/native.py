"""Screen gather and power resample (drop-in for maomi/backends/cuda/native.py).

``gather`` replaces the NVRTC ``gather_screens`` kernel (native.py:19-24) and
``ResamplePlan`` the ``resample_power`` kernel (native.py:51-105); both run the
library's sm_100a kernels on torch's current stream.
"""

import numpy as np

from ... import _lib
from ...numerics import resample_matrix, sparse_rows

__all__ = ["gather", "resample_matrix", "ResamplePlan"]


def gather(src, edge, offsets, n):
    """(B, Z, n, n) windows of the (Z, H, W) screens at ``offsets``, times ``edge``."""
    import torch
    b = len(offsets)
    z, h, w = src.shape
    if src.dtype != torch.complex64 or not src.is_cuda:
        raise ValueError("gather expects a CUDA complex64 (Z,H,W) tensor")
    off = torch.as_tensor(offsets, dtype=torch.int32, device=src.device).contiguous()
    if b and (int(off.min()) < 0 or int(off[:, 0].max()) + n > h or int(off[:, 1].max()) + n > w):
        raise ValueError("Outside FOV")
    edge = torch.as_tensor(edge, dtype=torch.float32, device=src.device).contiguous()
    out = torch.empty((b, z, n, n), device=src.device, dtype=src.dtype)
    _lib.call("mm_gather_screens", _lib.ptr(src.contiguous()), _lib.ptr(edge), _lib.ptr(off), _lib.ptr(out),
              b, z, h, w, n, _lib.stream_of(src.device))
    return out


class ResamplePlan:
    """|E|^(2*order) resampled by imresize(1/ss) o imtranslate(ss/2-0.5)."""

    def __init__(self, h, w, ss, device="cuda"):
        import torch
        mx, my = resample_matrix(h, ss), resample_matrix(w, ss)
        self.mx = torch.tensor(mx, dtype=torch.float32, device=device)
        self.my = torch.tensor(my, dtype=torch.float32, device=device)
        (ix, wx), (iy, wy) = sparse_rows(mx), sparse_rows(my)
        self.ix, self.wx = torch.as_tensor(ix, device=device), torch.as_tensor(wx, device=device)
        self.iy, self.wy = torch.as_tensor(iy, device=device), torch.as_tensor(wy, device=device)

    def __call__(self, field, scale, native=True, order=2, axial=None):
        """field (B,Z,H,W) complex64 -> (B,X,Y,Z) float32."""
        import torch
        field = field.contiguous()
        b, z, h, w = field.shape
        x, y = self.mx.shape[0], self.my.shape[0]
        if order not in (1, 2, 3):
            raise ValueError("Photon order must be 1, 2 or 3")
        axial = (torch.ones(z, device=field.device) if axial is None
                 else torch.as_tensor(axial, dtype=torch.float32, device=field.device))
        if tuple(axial.shape) != (z,):
            raise ValueError("One axial weight per plane required")
        out = torch.empty((b, x, y, z), device=field.device)
        _lib.call("mm_resample_power", _lib.ptr(field), _lib.ptr(self.ix), _lib.ptr(self.wx), _lib.ptr(self.iy),
                  _lib.ptr(self.wy), _lib.ptr(axial.contiguous()), _lib.ptr(out), b, z, h, w, x, y,
                  self.ix.shape[1], self.iy.shape[1], order, float(np.float32(scale)), _lib.stream_of(field.device))
        return out
