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
    src = idx.astype(float) - shift
    a = np.floor(src).astype(np.int64)
    f = src - a
    out = np.zeros((m, n))
    rows = np.broadcast_to(np.arange(m)[:, None], idx.shape)
    for col, wt in ((a, w * (1 - f)), (a + 1, w * f)):
        ok = (col >= 0) & (col < n)
        np.add.at(out, (rows[ok], col[ok]), wt[ok])
    return out


def sparse_rows(matrix):
    """(indices, weights) of the nonzeros of each row, padded to the widest row."""
    nz = matrix != 0
    k = max(1, int(nz.sum(1).max()) if len(matrix) else 1)
    inds = np.zeros((len(matrix), k), np.int32)
    wts = np.zeros((len(matrix), k), np.float32)
    r, c = np.nonzero(nz)
    slot = np.arange(len(r)) - np.searchsorted(r, r)
    inds[r, slot] = c
    wts[r, slot] = matrix[r, c]
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


def _dev64(a, device):
    import torch
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=torch.float64).contiguous()
    return _lib.upload(np.asarray(a, np.float64), device)


def lattice_index(points):
    """(nx, ny, idx) when ``points`` fill an nx x ny lattice whose x and y
    coordinates are symmetric about their centres (idx[i*ny + j] = the point
    at the i-th x and j-th y), else None."""
    p = np.asarray(points, float).reshape(-1, 2)
    xs, ys = np.unique(p[:, 0]), np.unique(p[:, 1])
    nx, ny = len(xs), len(ys)
    if nx < 2 or ny < 2 or nx * ny != len(p):
        return None
    tol = 1e-12 * max(1.0, float(np.abs(p).max()))
    if np.abs(xs + xs[::-1] - (xs[0] + xs[-1])).max() > tol or np.abs(ys + ys[::-1] - (ys[0] + ys[-1])).max() > tol:
        return None
    lin = np.searchsorted(xs, p[:, 0]) * ny + np.searchsorted(ys, p[:, 1])
    if len(np.unique(lin)) != len(p):
        return None
    idx = np.empty(nx * ny, np.int32)
    idx[lin] = np.arange(len(p), dtype=np.int32)
    return nx, ny, idx


_BLOCK_STREAMS = {}


def _block_streams(device):
    """Four high-priority streams per device for the parity-block factorisations."""
    import torch
    key = str(torch.device(device))
    if key not in _BLOCK_STREAMS:
        _BLOCK_STREAMS[key] = [torch.cuda.Stream(device=device, priority=-1) for _ in range(4)]
    return _BLOCK_STREAMS[key]


class V4Factor:
    """LU factors of the v4 Green system: dense, or for a symmetric lattice the
    four independent blocks of its even/odd reflection parities."""

    def __init__(self, p, lu, piv, lattice=None, idx=None, m=0):
        self.p, self.lu, self.piv, self.lattice, self.idx, self.m = p, lu, piv, lattice, idx, m

    def tensors(self):
        return [t for t in (self.p, self.lu, self.piv, self.idx) if t is not None]


def v4_factor_device(points, device="cuda", *, structured=True):
    """Factor the dense v4 Green system of ``points`` (FP64, on the current
    stream, no host synchronisation).  Points on a full lattice symmetric under
    both axis reflections (the fixed site lattice) use the reflection-parity
    block form: four independent systems of about n/4 unknowns."""
    import torch
    p = _dev64(points, device)
    n = p.shape[0]
    lat = lattice_index(points.cpu().numpy() if isinstance(points, torch.Tensor) else points) if structured else None
    if lat is not None:
        nx, ny, idx = lat
        m = ((nx + 1) // 2) * ((ny + 1) // 2)
        idx_d = _lib.upload(idx, device)
        B = torch.empty((4, m, m), dtype=torch.float64, device=device)
        _lib.call("mm_green_blocks", _lib.ptr(p), _lib.ptr(idx_d), nx, ny, m, _lib.ptr(B), _lib.stream_of(device))
        # one (non-batched) LU per parity block: the batched path of the solver
        # library launches hundreds of small kernels for blocks of this size
        lu = torch.empty_like(B)
        piv = torch.empty((4, m), dtype=torch.int32, device=device)
        # the four blocks are independent: one stream each, joined at the end
        here = torch.cuda.current_stream(device)
        streams = _block_streams(device)
        for b, st in enumerate(streams):
            st.wait_stream(here)
            with torch.cuda.stream(st):
                f, piv[b], _ = torch.linalg.lu_factor_ex(B[b])
                lu[b] = f.mT  # column-major storage, as the factorisation leaves it
        for st in streams:
            here.wait_stream(st)
        for t in (B, lu, piv):
            for st in streams:
                t.record_stream(st)
        return V4Factor(p, lu, piv, (nx, ny), idx_d, m)
    G = torch.empty((n, n), dtype=torch.float64, device=device)
    _lib.call("mm_green_matrix", _lib.ptr(p), _lib.ptr(G), n, _lib.stream_of(device))
    lu, piv, _ = torch.linalg.lu_factor_ex(G)
    return V4Factor(p, lu, piv)


def v4_solve_device(factor, values):
    """v4 coefficients for ``values`` (N,) or (N, C) from ``v4_factor_device``."""
    import torch
    p = factor.p
    n = p.shape[0]
    v = _dev64(values, p.device).reshape(n, -1).contiguous()
    if factor.lattice is None:
        return p, torch.linalg.lu_solve(factor.lu, factor.piv, v)
    nx, ny = factor.lattice
    C, m, dev = v.shape[1], factor.m, p.device
    stream = _lib.stream_of(dev)
    W = torch.empty((4, m, C), dtype=torch.float64, device=dev)
    _lib.call("mm_v4_parity", _lib.ptr(factor.idx), nx, ny, m, C, 0, _lib.ptr(v), _lib.ptr(W), stream)
    if C <= 4:
        _lib.call("mm_lu_solve_batched", _lib.ptr(factor.lu), _lib.ptr(factor.piv), 4, m, C, _lib.ptr(W), stream)
        D = W
    else:
        D = torch.linalg.lu_solve(factor.lu.mT, factor.piv, W).contiguous()
    coef = torch.empty((n, C), dtype=torch.float64, device=dev)
    _lib.call("mm_v4_parity", _lib.ptr(factor.idx), nx, ny, m, C, 1, _lib.ptr(D), _lib.ptr(coef), stream)
    return p, coef


def v4_coefficients_device(points, values, device="cuda"):
    """Solve the dense v4 Green system on the GPU (FP64). Returns device tensors (p, coef)."""
    return v4_solve_device(v4_factor_device(points, device), values)


def v4_evaluate_grid_device(p, coef, X, Y, device="cuda", *, points_host=None):
    """v4 values on the X x Y pixel-centre grid (FP64).  With ``points_host``
    (the same points on the host) at integer coordinates, the Green function
    is tabulated once per query-point offset (bitwise the same sums)."""
    import torch
    out = torch.empty((X, Y, coef.shape[1]), dtype=torch.float64, device=device)
    c = coef.contiguous()
    if points_host is not None:
        ph = np.asarray(points_host, float).reshape(-1, 2)
        if np.array_equal(ph, np.round(ph)) and np.abs(ph).max() < 2 ** 20:
            lo, hi = ph.min(0).astype(int), ph.max(0).astype(int)
            tw, th = X - lo[0] + hi[0], Y - lo[1] + hi[1]
            table = torch.empty(tw * th, dtype=torch.float64, device=device)
            _lib.call("mm_green_apply_grid_table", _lib.ptr(p), _lib.ptr(c), _lib.ptr(out), p.shape[0], X, Y,
                      c.shape[1], int(lo[0]), int(hi[0]), int(lo[1]), int(hi[1]), _lib.ptr(table), table.numel() * 8,
                      _lib.stream_of(device))
            return out
    _lib.call("mm_green_apply_grid", _lib.ptr(p), _lib.ptr(c), _lib.ptr(out), p.shape[0], X, Y,
              c.shape[1], _lib.stream_of(device))
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
