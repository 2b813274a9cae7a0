"""Stage geometry shared by every propagation entry point.

Mirrors maomi/_propagation.py:9-61: window sizes ``n``/``n2``, pupil and
tissue pitches ``d1``/``d2``, the z-planes of stages A (pupil side), B (focal
slab) and C (bottom tail), the top-tail cut and the crops.  Scalars keep the
reference's float32 roundings (``fl``, ``d1``, ``d2``, ``wvl``, ``nr``) so the
transfer functions built from them describe the same optical system.
"""

from types import SimpleNamespace

import numpy as np

from ._optical_math import gaussian_beam_size


def center_slice(n, m):
    """Centred slice of length ``m`` inside ``n`` (both of equal parity)."""
    if m > n or (n - m) % 2:
        raise ValueError(f"Incompatible centered grids {n},{m}")
    lo = (n - m) // 2
    return slice(lo, lo + m)


def geometry(config, raw_fields):
    """Window sizes, pitches, plane positions and crops for ``config``.

    ``raw_fields`` only contributes the number of screens of each stage (its
    arrays' last axis), exactly like _propagation.py:41."""
    v, p = config.parameters()
    r, ss = config.vres, config.ss
    n = int(round((v.vasc_sz[0] - v.vol_sz[0]) * r * ss))
    if config.propcrop:
        n2 = int(round(min(max(gaussian_beam_size(p, config.psf_um[2] / 2, 3)) * r * 2 * ss, n)))
    else:
        n2 = n
    if n % 2 and not n2 % 2:
        n2 -= 1
    fl = np.float32(config.focal_length_mm / 1000)
    d1 = np.float32(max(gaussian_beam_size(p, float(fl * 1e6))) / 1e6 / n)
    d2 = np.float32(1e-6 / r / ss)
    za = r * (config.depth_um + config.volume_um[2] / 2 - config.psf_um[2] / 2)
    slab = config.prop_um * r
    na, nb, nc = [np.shape(f)[-1] for f in raw_fields]
    part = za % slab
    if part:
        z_a = np.concatenate(([0.0], np.arange(na) + part / slab))
    else:
        z_a = np.arange(na + 1, dtype=float)
    planes = [
        z_a * config.prop_um * 1e-6,
        np.arange(nb + 1) / r * 1e-6,
        np.concatenate((np.arange(nc) * config.prop_um, [config.tail_um])) * 1e-6,
    ]
    cut = max(0, int(np.ceil((za - config.tail_um * r) / slab)))
    if cut >= len(planes[0]) - 1:
        raise ValueError("Top tail has no extent")
    focal_shape = np.round(np.array(config.psf_um[:2]) * r * ss).astype(int)
    return SimpleNamespace(
        n=n, n2=n2, fl=fl, d1=d1, d2=d2,
        wvl=np.float32(config.wavelength_um * 1e-6), nr=np.float32(config.n),
        z=planes, cut=cut, focal_shape=focal_shape,
        crop=center_slice(n, n2),
        focal_crop=tuple(center_slice(n2, int(k)) for k in focal_shape),
    )


def edge_window_1d(size):
    """One axis of the order-16 super-Gaussian edge window, exp(-(x/0.47n)^16),
    evaluated in FP64 on x = -n/2 .. n/2-1 and rounded once to float32."""
    x = np.arange(-size / 2, size / 2, dtype=np.float64) / (0.47 * size)
    return np.exp(-(x ** 16)).astype(np.float32)


def edge_apodization(size, device="cuda", dtype=None):
    """Separable edge window (size x size) as a device tensor (_propagation.py:59-61)."""
    import torch
    e = torch.as_tensor(edge_window_1d(size), device=device)
    w = e[:, None] * e[None, :]
    return w if dtype is None else w.to(dtype)
