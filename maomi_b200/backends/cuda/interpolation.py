"""Float64 MATLAB-v4 evaluation (drop-in for maomi/backends/cuda/interpolation.py).

``evaluate_v4`` keeps the reference's signature and NumPy float64 result; the
library's kernel evaluates every value column in one pass with the points and
coefficients staged through shared memory, and the queries are uploaded once
instead of per chunk.
"""

import numpy as np

from ... import _lib

__all__ = ["evaluate_v4"]


def evaluate_v4(points, coefficients, queries, *, chunk=16384, device="cuda"):
    import torch
    if not isinstance(chunk, (int, np.integer)) or chunk < 1:
        raise ValueError("chunk must be a positive integer")
    _lib.require_cuda(device)
    p = torch.as_tensor(np.ascontiguousarray(points, np.float64), device=device)
    c = torch.as_tensor(np.ascontiguousarray(np.asarray(coefficients, np.float64).reshape(len(p), -1)), device=device)
    q = torch.as_tensor(np.ascontiguousarray(np.asarray(queries, np.float64).reshape(-1, 2)), device=device)
    out = torch.empty((q.shape[0], c.shape[1]), dtype=torch.float64, device=device)
    if q.shape[0]:
        _lib.call("mm_green_apply", _lib.ptr(p), _lib.ptr(c), _lib.ptr(q), _lib.ptr(out), p.shape[0], q.shape[0],
                  c.shape[1], _lib.stream_of(device))
    return out.cpu().numpy()
