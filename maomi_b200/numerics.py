"""Resampling tables and the FP64 v4 interpolation on the GPU.

Host-side tables (index/weight plans) follow maomi/numerics.py:8-39 and
maomi/backends/cuda/native.py:27-48; the arithmetic on arrays runs in the CUDA
library.  ``v4_interpolate`` mirrors maomi/numerics.py:93-153 with the dense
FP64 Green system built on the GPU, solved on the GPU, and evaluated by the
library's FP64 kernel.
"""

import numpy as np

from . import _lib


def keys_cubic(x):
    """Keys cubic convolution kernel with a = -0.5 (MATLAB imresize 'bicubic')."""
    a = np.abs(x)
    inner = (1.5 * a - 2.5) * a * a + 1
    outer = ((-0.5 * a + 2.5) * a - 4) * a + 2
    return np.where(a <= 1, inner, np.where(a < 2, outer, 0.0))


def resize_table(n, scale):
    """Index and weight table of a 1-D imresize by ``scale`` (half-pixel
    centres, symmetric extension, antialiasing when shrinking)."""
    m = int(np.ceil(n * scale))
    shrink = min(scale, 1)
    centres = (np.arange(m) + 0.5) / scale - 0.5
    width = 4 / shrink
    taps = int(np.ceil(width)) + 2
    idx = np.floor(centres - width / 2).astype(int)[:, None] + np.arange(taps)[None, :]
    w = keys_cubic((centres[:, None] - idx) * shrink) * shrink
    w /= w.sum(1, keepdims=True)
    idx %= 2 * n
    idx = np.where(idx < n, idx, 2 * n - 1 - idx)
    return idx, w


def is_identity_table(idx, w):
    """True when a resize table reproduces its input exactly (scale 1)."""
    m, _ = idx.shape
    nz = w != 0
    return (m == idx.max() + 1 and np.all(nz.sum(1) == 1) and np.all(w[nz] == 1.0)
            and np.array_equal(idx[nz], np.arange(m)))


def resample_matrix(n, ss):
    """Dense (ceil(n/ss), n) operator: imresize(1/ss) after imtranslate(ss/2-0.5)
    with linear interpolation and zero fill (the composition
    maomi/backends/cuda/native.py:27-48 builds)."""
    idx, w = resize_table(n, 1 / ss)
    shift = ss / 2 - 0.5
    m = idx.shape[0]
    out = np.zeros((m, n))
    for i in range(m):
        for j, wt in zip(idx[i], w[i]):
            a = int(np.floor(j - shift))
            f = j - shift - a
            if 0 <= a < n:
                out[i, a] += wt * (1 - f)
            if 0 <= a + 1 < n:
                out[i, a + 1] += wt * f
    return out


def sparse_rows(matrix):
    """(indices, weights) of the nonzeros of each row, padded to the widest row."""
    k = max(1, max(np.count_nonzero(row) for row in matrix))
    inds = np.zeros((len(matrix), k), np.int32)
    wts = np.zeros((len(matrix), k), np.float32)
    for i, row in enumerate(matrix):
        j = np.nonzero(row)[0]
        inds[i, :len(j)] = j
        wts[i, :len(j)] = row[j]
    return inds, wts


# ----------------------------------------------------------------------- v4 --

def _grid_shape(q):
    """(X, Y) if queries are the pixel centres (i+0.5, j+0.5), else None."""
    if q.ndim != 3 or q.shape[-1] != 2:
        return None
    X, Y = q.shape[:2]
    if X * Y == 0:
        return None
    gx = np.arange(X)[:, None] + 0.5
    gy = np.arange(Y)[None, :] + 0.5
    if np.array_equal(q[..., 0], np.broadcast_to(gx, (X, Y))) and np.array_equal(q[..., 1], np.broadcast_to(gy, (X, Y))):
        return X, Y
    return None


def v4_coefficients_device(points, values, device="cuda"):
    """Solve the dense v4 Green system on the GPU (FP64). Returns device tensors (p, coef)."""
    import torch

    def dev64(a):
        if isinstance(a, torch.Tensor):
            return a.to(device=device, dtype=torch.float64).contiguous()
        return torch.as_tensor(np.ascontiguousarray(a, np.float64), device=device)

    p, v = dev64(points), dev64(values)
    n = p.shape[0]
    G = torch.empty((n, n), dtype=torch.float64, device=device)
    _lib.call("mm_green_matrix", _lib.ptr(p), _lib.ptr(G), n, _lib.stream_of(device))
    coef = torch.linalg.solve(G, v.reshape(n, -1))
    return p, coef


def v4_evaluate_grid_device(p, coef, X, Y, device="cuda"):
    import torch
    out = torch.empty((X, Y, coef.shape[1]), dtype=torch.float64, device=device)
    _lib.call("mm_green_apply_grid", _lib.ptr(p), _lib.ptr(coef.contiguous()), _lib.ptr(out), p.shape[0], X, Y,
              coef.shape[1], _lib.stream_of(device))
    return out


def v4_interpolate(points, values, queries, chunk=16384, *, backend="auto", device="cuda"):
    """MATLAB v4 interpolation in float64 (maomi/numerics.py:93-153), on the GPU.

    ``backend`` accepts "auto" and "cuda"; the reference's CPU evaluator is
    not part of this package."""
    import torch
    if backend not in ("auto", "cpu", "cuda"):
        raise ValueError("backend must be auto, cpu or cuda")
    if backend == "cpu":
        raise ValueError("maomi_b200 evaluates v4 on CUDA only; use the reference package for CPU")
    if not isinstance(chunk, (int, np.integer)) or chunk < 1:
        raise ValueError("chunk must be a positive integer")
    p, v, q = np.asarray(points, float), np.asarray(values, float), np.asarray(queries, float)
    if p.ndim != 2 or p.shape[1] != 2 or not len(p):
        raise ValueError("points must be a nonempty (N, 2) array")
    if v.ndim not in (1, 2) or len(v) != len(p) or (v.ndim == 2 and v.shape[1] == 0):
        raise ValueError("values must have shape (N,) or (N, C) with C > 0")
    if q.ndim < 1 or q.shape[-1] != 2:
        raise ValueError("queries must have shape (..., 2)")
    shape = q.shape[:-1] + v.shape[1:]
    if len(p) == 1:
        return np.broadcast_to(v[0], shape).copy()
    flat = q.reshape(-1, 2)
    if not len(flat):
        return np.empty(shape, dtype=np.float64)
    _lib.require_cuda(device)
    dp, coef = v4_coefficients_device(p, v, device)
    grid = _grid_shape(q)
    if grid is not None:
        out = v4_evaluate_grid_device(dp, coef, *grid, device=device)
    else:
        out = evaluate_v4_device(dp, coef, torch.as_tensor(np.ascontiguousarray(flat), device=device))
    return out.cpu().numpy().reshape(shape)


def evaluate_v4_device(p, coef, queries):
    import torch
    coef = coef.reshape(p.shape[0], -1).contiguous()
    out = torch.empty((queries.shape[0], coef.shape[1]), dtype=torch.float64, device=p.device)
    _lib.call("mm_green_apply", _lib.ptr(p), _lib.ptr(coef), _lib.ptr(queries.contiguous()), _lib.ptr(out),
              p.shape[0], queries.shape[0], coef.shape[1], _lib.stream_of(p.device))
    return out
