"""CPU restatement of the scattering-field generator (TEST INFRASTRUCTURE ONLY).

Follows maomi/_optical_math.py:20-67 (``masked_3DGP_test``) and
maomi/optics.py:120-197 (``prepare_fields``): a Gaussian-process draw made by
shaping complex white noise with the square root of a sum of separable
squared-exponential spectra, inverse 3-D DFT between two ifftshifts, the real
part scaled by 2 * p_scale * sqrt(N); then partial end slabs scaled by their
optical thickness and, with vessels, the occupancy combination.

The noise is an input here: the reference draws it with torch's generator
(real parts of the whole grid, then imaginary parts, field after field from
one seed), and the tests draw it the same way so both sides see the same
numbers.  Arithmetic follows the reference's float32 spectrum; the inverse
transform is numpy's FP64 FFT.
"""

import numpy as np

WMX = np.pi / 2


def spectrum(grid_sz, l_scale, l_weights=None):
    """sqrt(sum_i prod(l_i) * (kx ky kz)^2 * w_i^2) on the unshifted grid, float32
    (_optical_math.py:26-53)."""
    import torch
    grid_sz = [int(x) for x in grid_sz]
    l_scale = np.asarray(l_scale, np.float32)
    w = np.ones(l_scale.shape[0], np.float32) if l_weights is None else np.asarray(l_weights, np.float32)
    g = [torch.linspace(-WMX, WMX, n, dtype=torch.float32).pow(2).numpy() for n in grid_sz]
    gx, gy, gz = g[0][:, None, None], g[1][None, :, None], g[2][None, None, :]
    acc = np.zeros(grid_sz, np.float32)
    for i in range(l_scale.shape[0]):
        kx = np.exp(-gx * np.float32(l_scale[i, 0] ** 2)).astype(np.float32)
        ky = np.exp(-gy * np.float32(l_scale[i, 1] ** 2)).astype(np.float32)
        kz = np.exp(-gz * np.float32(l_scale[i, 2] ** 2)).astype(np.float32)
        prod_l = np.float32(l_scale[i, 0] * l_scale[i, 1] * l_scale[i, 2])
        k3 = (kx * ky * kz).astype(np.float32)
        acc += (prod_l * (k3 ** 2) * np.float32(w[i] ** 2)).astype(np.float32)
    return np.sqrt(acc)


def gp_sample(grid_sz, l_scale, p_scale, noise_re, noise_im, l_weights=None, mu=0.0, bin_mask=1.0):
    """masked_3DGP_test with the noise given (_optical_math.py:55-67)."""
    s = spectrum(grid_sz, l_scale, l_weights).astype(np.float64)
    g = (np.asarray(noise_re, np.float64) + 1j * np.asarray(noise_im, np.float64)) * s
    g = np.fft.ifftshift(np.fft.ifftn(np.fft.ifftshift(g)))
    n_elem = g.size
    return 2 * p_scale * bin_mask * np.sqrt(n_elem) * np.real(g) + mu


def torch_noise(shapes, seed):
    """The reference's draws for prepare_fields: one generator seeded once,
    per field a real and an imaginary standard-normal grid (float32)."""
    import torch
    gen = torch.Generator().manual_seed(int(seed))
    out = []
    for shape in shapes:
        re = torch.randn(tuple(int(v) for v in shape), generator=gen, dtype=torch.float32).numpy()
        im = torch.randn(tuple(int(v) for v in shape), generator=gen, dtype=torch.float32).numpy()
        out.append((re, im))
    return out


def field_extents(config):
    """(shapes, za, zb, pc, nc) as optics.py:127-144 forms them."""
    from maomi_b200.fixed import field_shapes
    r = config.vres
    za = int(round((config.depth_um + config.volume_um[2] / 2 - config.psf_um[2] / 2) * r))
    zb = int(round(config.psf_um[2] * r))
    pc = int(round(config.prop_um * r))
    nc = int(round(config.tail_um * r))
    return field_shapes(config), za, zb, pc, nc


def prepare_fields(config, noise, vessels=None):
    """Raw A/B/C fields (optics.py:145-196) from the given per-field noise."""
    shapes, za, zb, pc, nc = field_extents(config)
    r = config.vres
    raw = []
    for i, shape in enumerate(shapes):
        ls = np.repeat(np.asarray(config.scatter_scales_um, np.float32)[:, None], 3, 1) * np.float32(r)
        scale = 1 if i == 1 else pc
        ls[:, 2] /= np.float32(scale)
        raw.append(gp_sample(shape, ls, scale, noise[i][0], noise[i][1], config.scatter_weights))
    if za % pc:
        raw[0][..., 0] *= (za % pc) / pc
    if nc % pc:
        raw[2][..., -1] *= (nc % pc) / pc
    if vessels is not None:
        v = np.asarray(vessels, np.float64)
        n = shapes[0][0] - int(round(config.volume_um[0] * r))
        n2 = shapes[1][0] - int(round(config.volume_um[0] * r))
        xs, ys = slice(0, shapes[0][0]), slice(0, shapes[0][1])
        edges = list(range(0, za, pc)) if za % pc == 0 else [0] + list(range(za % pc, za, pc))
        occ_a = np.stack([v[xs, ys, a:b].sum(-1) for a, b in zip(edges, edges[1:] + [za])], -1)
        off = (n - n2) // 2
        occ_b = v[off:off + shapes[1][0], off:off + shapes[1][1], za:za + zb]
        occ_c = np.stack([v[xs, ys, z:min(z + pc, za + zb + nc)].sum(-1) for z in range(za + zb, za + zb + nc, pc)],
                         -1)
        for i, occ in enumerate((occ_a, occ_b, occ_c)):
            raw[i] = occ + raw[i] * (1 - occ / (1 if i == 1 else pc))
    return raw
