"""CPU restatement of MaoMi's local-PSF (RANA) renderer (TEST INFRASTRUCTURE ONLY).

Restates maomi/rana/_fft.py:8-95 (LocalFFTPlan: per node-pair tiles, zero
padded FFT convolution or correlation, overlap-add) and the parts of
maomi/rana/operator.py:10-17, 61-67, 122-167 that drive it (smoothstep node
weights, linear depth weights, ``static`` and ``scan_slab``), in float64 with
``scipy.fft`` exactly as the reference's NumPy backend does.
"""

import numpy as np
from scipy import fft


def axis_weights(nodes, positions):
    """operator.py:10-17."""
    ids = np.clip(np.searchsorted(nodes, positions, side="right") - 1, 0, len(nodes) - 2)
    t = np.clip((positions - nodes[ids]) / (nodes[ids + 1] - nodes[ids]), 0, 1)
    t = t * t * (3 - 2 * t)
    w = np.zeros((len(nodes), len(positions)))
    w[ids, np.arange(len(positions))] = 1 - t
    w[ids + 1, np.arange(len(positions))] = t
    return w


def local_fft(shape, kernels, weights, source, *, plane, detection, correlate):
    """_fft.py:9-95 with one tile per batch (the CPU backend's batch size)."""
    kshape = kernels.shape[2:]
    centers = np.array([(k - 1 - k // 2) if correlate else k // 2 for k in kshape])
    dims = (1, 2) if plane else (1, 2, 3)
    wx, wy = weights
    out = np.zeros(shape[:2] if plane else shape)
    src = np.asarray(source, float)
    for i in range(len(wx)):
        for j in range(len(wy)):
            xi, yi = np.flatnonzero(wx[i]), np.flatnonzero(wy[j])
            if not len(xi) or not len(yi):
                continue
            lo, hi = np.array([xi[0], yi[0]]), np.array([xi[-1] + 1, yi[-1] + 1])
            w = wx[i, lo[0]:hi[0], None] * wy[j, None, lo[1]:hi[1]]
            if detection:
                start, end = lo, hi
                tstart = np.maximum(0, lo - centers[:2])
                tend = np.minimum(shape[:2], hi + np.array(kshape[:2]) - 1 - centers[:2])
                rstart = tstart - lo + centers[:2]
            else:
                start = np.maximum(0, lo - np.array(kshape[:2]))
                end = np.minimum(shape[:2], hi + np.array(kshape[:2]))
                tstart, tend = lo, hi
                rstart = lo - start + centers[:2]
            sl = tuple(slice(int(a), int(b)) for a, b in zip(start, end))
            tg = tuple(slice(int(a), int(b)) for a, b in zip(tstart, tend))
            resp = tuple(slice(int(a), int(a + b - c)) for a, b, c in zip(rstart, tend, tstart))
            if not plane:
                resp += (slice(int(centers[2]), int(centers[2] + shape[2])),)
            sshape = tuple(end - start) + (shape[2],)
            lengths = tuple(fft.next_fast_len(sshape[d] + kshape[d] - 1) for d in ((0, 1) if plane else (0, 1, 2)))
            tile = src[sl] * w[..., None] if detection else src[sl]
            k = kernels[i, j]
            if correlate:
                k = np.flip(k, axis=(0, 1) if plane else (0, 1, 2))
            spec = fft.rfftn(tile[None], lengths, axes=dims) * fft.rfftn(k[None], lengths, axes=dims)
            if plane:
                spec = spec.sum(axis=3)
            full = fft.irfftn(spec, lengths, axes=dims)[0]
            piece = full[resp]
            out[tg] += piece if detection else piece * (w if plane else w[..., None])
    return out


def node_weights(field_x, field_y, shape, pitch, origin=(0.0, 0.0)):
    """operator.py:48-59 (coverage check omitted)."""
    coords = [o + (np.arange(n) + .5) * p for o, n, p in zip(origin, shape[:2], pitch)]
    return axis_weights(np.asarray(field_x, float), coords[0]), axis_weights(np.asarray(field_y, float), coords[1])


def depth_weights(depths, z):
    """operator.py:61-67."""
    if depths is None:
        return np.ones((1, np.size(z)))
    return np.stack([np.interp(np.atleast_1d(z), depths, row) for row in np.eye(len(depths))])


def static(kernel_list, x_um, y_um, pitch, volume, *, operator, native=False, depths=None, z_origin=0.0,
           origin=(0.0, 0.0)):
    """operator.py:122-134."""
    a = np.asarray(volume, float)
    detection = not native and operator == "detection"
    correlate = not native and operator == "excitation"
    z = z_origin + (np.arange(a.shape[2]) + .5) * pitch[2]
    wz = depth_weights(depths, z)
    wts = node_weights(x_um, y_um, a.shape, pitch, origin)
    result = np.zeros_like(a)
    for k, w in zip(kernel_list, wz):
        if not np.any(w):
            continue
        src = a * w if detection else a
        result += local_fft(a.shape, k, wts, src, plane=False, detection=detection,
                            correlate=correlate) * (1 if detection else w)
    return np.maximum(result, 0.)


def scan_slab(kernel_list, x_um, y_um, pitch, slab, *, operator, native=False, depths=None, z_origin=0.0,
              z_start=0, scan_avg=1, origin=(0.0, 0.0)):
    """operator.py:136-167."""
    a = np.asarray(slab, float)
    detection = not native and operator == "detection"
    correlate = not native and operator == "excitation"
    kz = kernel_list[0].shape[-1]
    center = kz // 2
    z = z_origin + (z_start + np.arange(a.shape[2]) + .5) * pitch[2]
    wz = depth_weights(depths, z if detection else [z[center]])
    starts = np.arange(0, a.shape[2], scan_avg)
    result = np.zeros(a.shape[:2])
    for k, w in zip(kernel_list, wz):
        if not np.any(w):
            continue
        source = a * w if detection else a
        kern = k
        if detection:
            ids = 2 * center - np.arange(a.shape[2])
            kern = np.take(kern, np.minimum(ids, a.shape[2] - 1), axis=-1).copy()
            kern[..., ids >= a.shape[2]] = 0
        if scan_avg > 1:
            kern = np.add.reduceat(kern, starts, axis=-1)
            source = np.add.reduceat(source, starts, axis=2)
        wts = node_weights(x_um, y_um, source.shape, pitch, origin)
        result += local_fft(source.shape, kern, wts, source, plane=True, detection=detection,
                            correlate=correlate) * (1 if detection else w[0])
    return np.maximum(result, 0.)
