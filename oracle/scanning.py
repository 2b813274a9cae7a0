"""CPU restatement of MaoMi's static and per-frame scan operators (TEST INFRASTRUCTURE ONLY).

Restates, in float64 NumPy/SciPy:

* ``zstack`` -- maomi/scanning.py:8-53 (``matlab_convn``: zero extension, 3-D
  linear convolution, MATLAB ``floor(k/2)`` crop; ``legacy_circular``: periodic
  XY, zero-extended Z, correlation in Z, crop from ``k - 1 - k//2``);
* ``single_scan`` -- maomi/movie.py:48-66 with ``psf_fft`` (:37-42),
  ``_group_z`` (:32-35) and ``_smooth_length`` (:22-29);
* ``blurred_background`` -- maomi/movie.py:69-102 with ``conv2_same`` (:14-19).

Linear convolutions are written as explicit full convolutions (SciPy's
``fftconvolve`` in FP64) and crops; where the reference evaluates a circular
FFT convolution whose size it chooses (the frequency-domain background), the
size is reproduced and the wrap is restated explicitly.
"""

import numpy as np
from scipy import fft as sfft
from scipy.signal import fftconvolve


def smooth_length(n):
    """movie.py:22-29: the smallest m >= n with no prime factor above 7."""
    while True:
        m = n
        for prime in (2, 3, 5, 7):
            while m % prime == 0:
                m //= prime
        if m == 1:
            return n
        n += 1


def group_z(a, count):
    """movie.py:32-35: sums of ``count`` consecutive planes (the last group may be short)."""
    if not isinstance(count, (int, np.integer)) or count < 1:
        raise ValueError("scan_avg must be a positive integer")
    return np.add.reduceat(a, np.arange(0, a.shape[2], count), axis=2) if count > 1 else a


def zstack(volume, psf, *, mode="matlab_convn", mask=None, collection_mask=None):
    """scanning.py:8-53 in float64."""
    v = np.asarray(volume, np.float64)
    p = np.asarray(psf, np.float64)
    if v.ndim != 3 or p.ndim != 3:
        raise ValueError("Expected X,Y,Z arrays")
    for m in (mask, collection_mask):
        if m is not None:
            m = np.asarray(m, np.float64)
            if m.shape != v.shape[:2]:
                raise ValueError("Mask must match volume XY")
            v = v * m[..., None]
    if mode == "matlab_convn":
        full = fftconvolve(v, p, mode="full")
        return full[tuple(slice(b // 2, b // 2 + a) for a, b in zip(v.shape, p.shape))]
    if mode == "legacy_circular":
        h, w, z = v.shape
        a, b, k = p.shape
        if a > h or b > w:
            raise ValueError("Legacy operator requires PSF XY <= image XY")
        kernel = np.zeros((h, w, k))
        kernel[:a, :b] = p[:, :, ::-1]
        kernel = np.roll(kernel, (-a // 2, -b // 2), (0, 1))
        n = (h, w, z + k - 1)
        full = sfft.irfftn(sfft.rfftn(v, s=n) * sfft.rfftn(kernel, s=n), s=n)
        start = k - 1 - k // 2
        return full[:, :, start:start + z]
    raise ValueError(f"Unknown operator: {mode}")


def single_scan(volume, psf, *, scan_avg=1):
    """movie.py:48-66 (no precomputed spectrum): the sum over grouped planes of
    the 2-D linear convolutions, cropped at floor(k/2)."""
    v = np.asarray(volume, np.float64)
    p = np.asarray(psf, np.float64)
    if v.ndim != 3 or p.ndim != 3 or v.shape[2] != p.shape[2]:
        raise ValueError("Volume slab and PSF must have the same axial length")
    gv, gp = group_z(v, scan_avg), group_z(p, scan_avg)
    X, Y = v.shape[:2]
    a, b = p.shape[:2]
    acc = np.zeros((X + a - 1, Y + b - 1))
    for j in range(gv.shape[2]):
        acc += fftconvolve(gv[:, :, j], gp[:, :, j], mode="full")
    return acc[a // 2:a // 2 + X, b // 2:b // 2 + Y]


def conv2_same(image, kernel):
    """movie.py:14-19: full 2-D convolution cropped at floor(k/2)."""
    image = np.asarray(image, np.float64)
    kernel = np.asarray(kernel, np.float64)
    full = fftconvolve(image, kernel, mode="full")
    i, j = np.asarray(kernel.shape) // 2
    return full[i:i + image.shape[0], j:j + image.shape[1]]


def background_image(volume, indices, *, power_ratio=1.0, mask=None, zscale=None, extra_volumes=()):
    """movie.py:86-95: the scaled plane mean that the background kernel blurs."""
    volume = np.asarray(volume, np.float64)
    indices = np.asarray(indices, int).ravel()
    if indices.size == 0:
        raise ValueError("Background requires at least one axial slice")
    if np.any(indices < 0) or np.any(indices >= volume.shape[2]):
        raise ValueError("Invalid background indices")
    scale = (np.asarray(zscale, np.float64).ravel()[:len(indices)]
             if zscale is not None and np.size(zscale) >= len(indices) else np.ones(len(indices)))
    image = (volume[:, :, indices] * scale).sum(axis=2) / len(indices)
    for other in extra_volumes:
        image = image + (np.asarray(other, np.float64)[:, :, indices] * scale).sum(axis=2) / len(indices)
    image = image * power_ratio
    if mask is not None:
        image = image * np.asarray(mask, np.float64)
    return image


def blurred_background(volume, indices, kernel, *, power_ratio=1.0, mask=None, zscale=None, extra_volumes=(),
                       frequency_size=None):
    """movie.py:69-102.  ``kernel`` is the spatial kernel; with
    ``frequency_size`` (the (S0, S1) of the reference's ``psf_fft`` spectrum)
    the frequency-domain branch is restated: a circular convolution of size S
    cropped from ceil((S - X - 1) / 2)."""
    image = background_image(volume, indices, power_ratio=power_ratio, mask=mask, zscale=zscale,
                             extra_volumes=extra_volumes)
    indices = np.asarray(indices, int).ravel()
    k = np.asarray(kernel, np.float64)
    if k.ndim == 3:
        k = k[:, :, indices].mean(axis=2) if k.shape[2] > 1 else k[:, :, 0]
    if frequency_size is None:
        return conv2_same(image, k)
    S = tuple(int(s) for s in frequency_size)
    X, Y = image.shape
    spec = sfft.fft2(k, s=S)
    circ = sfft.ifft2(sfft.fft2(image, s=S) * spec).real
    start = np.ceil((np.asarray(S) - np.asarray((X, Y)) - 1) / 2).astype(int)
    return circ[start[0]:start[0] + X, start[1]:start[1] + Y]
