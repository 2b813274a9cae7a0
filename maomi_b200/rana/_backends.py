"""Device arrays for the local-PSF operator (maomi/rana/_backends.py:13-106).

``get_backend("cuda[:i]")`` returns float64 torch arrays on that device; the
renderer's arithmetic runs in ``mm_local_render``.  There is no CPU backend in
this package (the reference's NumPy backend stays with the reference)."""

import numpy as np


class CudaBackend:
    def __init__(self, device):
        import torch
        from .. import _lib
        _lib.require_cuda(device)
        self.device = str(device)
        self.torch = torch

    def array(self, value):
        t = self.torch
        if isinstance(value, t.Tensor):
            return value.to(device=self.device, dtype=t.float64).contiguous()
        return t.as_tensor(np.array(value, dtype=np.float64, copy=True, order="C"), device=self.device)

    def zeros(self, shape):
        return self.torch.zeros(tuple(shape), device=self.device, dtype=self.torch.float64)

    def stack(self, values, axis=0):
        return self.torch.stack(values, dim=axis)

    def sum(self, value, axis):
        return value.sum(dim=axis)

    def group_sum(self, value, starts, width):
        return self.torch.stack([value[..., s:s + width].sum(-1) for s in starts], dim=-1).contiguous()

    def nbytes(self, value):
        return value.numel() * value.element_size()

    def to_numpy(self, value):
        return value.cpu().numpy()


def get_backend(device):
    device = str(device)
    if device.startswith("cuda"):
        return CudaBackend(device)
    if device == "cpu":
        raise ValueError("maomi_b200 renders on CUDA only; use the reference package for CPU")
    raise ValueError("device must be cpu or cuda[:index]")
