"""Scattering-field generation on the GPU: the raw A/B/C refractive-index
occupancy fields the optical stage propagates through.

Drop-in for ``maomi.optics.prepare_fields`` (optics.py:120-197) and
``maomi._optical_math.masked_3DGP_test`` (_optical_math.py:20-67) with
``device="cuda"``: same shapes, scales, slab factors and vessel occupancy
combination, returned as CUDA float32 tensors that ``fixed.stage_device`` /
``fixed.run_stages`` take directly.

A Gaussian-process draw is two hand-written kernels around the inverse 3-D
DFT: ``mm_gp_spectrum`` shapes complex white noise with sqrt(sum of
separable squared-exponential spectra) and applies the first ifftshift; the
transform is cuFFT's complex-to-complex inverse (``torch.fft.ifftn``, the
library transform of a 768 x 768 x 46 grid); ``mm_gp_finish`` applies the
second ifftshift, takes the scaled real part and the partial-slab factor.

Noise: by default drawn on the device by a torch generator seeded with
``config.seed`` (real grid, then imaginary grid, field after field, as the
reference draws on its device); like the reference's backends, device and CPU
draws differ.  ``noise=`` takes explicit (real, imaginary) grids per field,
which is how the tests feed the reference's own CPU draws.
"""

import numpy as np

from . import _lib
from .fixed import field_shapes

WMX = np.pi / 2


def _grid2(n):
    """linspace(-pi/2, pi/2, n)^2 in float32, formed as the reference forms it."""
    import torch
    return torch.linspace(-WMX, WMX, int(n), dtype=torch.float32).pow(2)


def _scale_tables(l_scale, l_weights, device):
    import torch
    ls = np.asarray(l_scale.cpu() if hasattr(l_scale, "cpu") else l_scale, np.float32).reshape(-1, 3)
    k = ls.shape[0]
    w = np.ones(k, np.float32) if l_weights is None else np.asarray(
        l_weights.cpu() if hasattr(l_weights, "cpu") else l_weights, np.float32).reshape(-1)
    if w.shape[0] != k:
        raise ValueError(f"{k} length scales but {w.shape[0]} weights")
    l2 = (ls * ls).astype(np.float32)
    prod_l = ((ls[:, 0] * ls[:, 1]).astype(np.float32) * ls[:, 2]).astype(np.float32)
    w2 = (w * w).astype(np.float32)
    return [torch.as_tensor(a, device=device) for a in (l2.reshape(-1), prod_l, w2)] + [k]


def _noise_pair(noise, shape, generator, device):
    import torch
    if noise is None:
        re = torch.randn(shape, generator=generator, device=device, dtype=torch.float32)
        im = torch.randn(shape, generator=generator, device=device, dtype=torch.float32)
        return re, im
    out = []
    for a in noise:
        t = torch.as_tensor(a, dtype=torch.float32)
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"noise of shape {tuple(t.shape)} for a {tuple(shape)} grid")
        out.append(t.to(device, non_blocking=True).contiguous())
    return out


def _gp(shape, l_scale, p_scale, l_weights, noise, generator, device, first=1.0, last=1.0, bin_mask=1, mu=0):
    import torch
    nx, ny, nz = (int(v) for v in shape)
    stream = _lib.stream_of(device)
    g2 = [_grid2(n).to(device) for n in (nx, ny, nz)]
    l2, prod_l, w2, k = _scale_tables(l_scale, l_weights, device)
    re, im = _noise_pair(noise, (nx, ny, nz), generator, device)
    spec = torch.empty((nx, ny, nz), dtype=torch.complex64, device=device)
    _lib.call("mm_gp_spectrum", nx, ny, nz, _lib.ptr(g2[0]), _lib.ptr(g2[1]), _lib.ptr(g2[2]), k, _lib.ptr(l2),
              _lib.ptr(prod_l), _lib.ptr(w2), _lib.ptr(re), _lib.ptr(im), _lib.ptr(spec), stream)
    y = torch.fft.ifftn(spec, dim=(0, 1, 2))
    out = torch.empty((nx, ny, nz), dtype=torch.float32, device=device)
    scalar_mask = np.ndim(bin_mask) == 0 and not hasattr(bin_mask, "shape")
    scale = 2 * p_scale * (bin_mask if scalar_mask else 1) * np.sqrt(nx * ny * nz)
    _lib.call("mm_gp_finish", _lib.ptr(y), nx, ny, nz, float(np.float32(scale)), float(first), float(last),
              _lib.ptr(out), stream)
    if not scalar_mask:
        out = out * torch.as_tensor(bin_mask, dtype=torch.float32, device=device)
    if mu:
        out = out + mu
    return out


def masked_3DGP_test(grid_sz, l_scale, p_scale, mu=0, bin_mask=1, l_weights=None, device="cuda", *, noise=None,
                     generator=None):
    """One Gaussian-process draw (_optical_math.py:20-67) on the GPU.

    ``noise`` = (real, imaginary) float32 grids of ``grid_sz`` replaces the
    draw from ``generator`` (torch's default CUDA generator when None)."""
    _lib.require_cuda(device)
    return _gp([int(x) for x in grid_sz], l_scale, float(p_scale), l_weights, noise, generator, device,
               bin_mask=bin_mask, mu=mu)


def field_extents(config):
    """(shapes, za, zb, pc, nc, n, n2) of optics.py:127-144."""
    r = config.vres
    shapes = field_shapes(config)
    za = int(round((config.depth_um + config.volume_um[2] / 2 - config.psf_um[2] / 2) * r))
    zb = int(round(config.psf_um[2] * r))
    pc = int(round(config.prop_um * r))
    nc = int(round(config.tail_um * r))
    xy = np.round(np.asarray(config.volume_um[:2]) * r).astype(int)
    return shapes, za, zb, pc, nc, shapes[0][0] - int(xy[0]), shapes[1][0] - int(xy[0])


def _slab_bounds(za, zb, pc, nc):
    """Vessel-plane ranges of the A, B and C slabs (optics.py:183-193)."""
    a, start, end = [0], 0, (za % pc or pc)
    while start < za:
        a.append(end)
        start, end = end, min(za, end + pc)
    b = list(range(za, za + zb + 1))
    c = [za + zb]
    for z in range(za + zb, za + zb + nc, pc):
        c.append(min(z + pc, za + zb + nc))
    return a, b, c


def prepare_fields(config, vessels=None, *, device="cuda", scatter=True, noise=None, generator=None):
    """Raw A/B/C occupancy fields (optics.py:120-197) as CUDA float32 tensors.

    ``noise``: optional list of three (real, imaginary) grids; otherwise a
    device generator seeded with ``config.seed`` draws them."""
    import torch
    _lib.require_cuda(device)
    shapes, za, zb, pc, nc, n, n2 = field_extents(config)
    r = config.vres
    if scatter and noise is None and generator is None:
        generator = torch.Generator(device=device).manual_seed(int(config.seed))
    scales = np.repeat(np.asarray(config.scatter_scales_um, np.float32)[:, None], 3, 1) * np.float32(r)
    raw = []
    for i, shape in enumerate(shapes):
        first = (za % pc) / pc if i == 0 and za % pc else 1.0
        last = (nc % pc) / pc if i == 2 and nc % pc else 1.0
        if scatter:
            ls = scales.copy()
            scale = 1 if i == 1 else pc
            ls[:, 2] /= np.float32(scale)
            raw.append(_gp(shape, ls, float(scale), config.scatter_weights, None if noise is None else noise[i],
                           generator, device, first=first, last=last))
        else:
            raw.append(torch.zeros(shape, dtype=torch.float32, device=device))
    if vessels is not None:
        v = torch.as_tensor(vessels, dtype=torch.float32).to(device).contiguous()
        required = (shapes[0][0], shapes[0][1], za + zb + nc)
        if v.ndim != 3 or any(a < b for a, b in zip(v.shape, required)):
            raise ValueError(f"Padded vessels need at least {required}, got {tuple(v.shape)}")
        off = (n - n2) // 2
        stream = _lib.stream_of(device)
        for i, (bounds, x0, denom) in enumerate(zip(_slab_bounds(za, zb, pc, nc), (0, off, 0), (pc, 1, pc))):
            f = raw[i]
            _lib.call("mm_vessel_combine", _lib.ptr(v), v.shape[0], v.shape[1], v.shape[2], x0, x0,
                      _lib.host_array(bounds, _lib.c_int), float(denom), _lib.ptr(f), f.shape[0], f.shape[1],
                      f.shape[2], stream)
    return raw
