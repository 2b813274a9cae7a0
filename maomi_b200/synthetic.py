"""Seeded synthetic inputs for the optical stage and the local-PSF renderer.

The workloads have no public dataset: refractive-index perturbations, pupil
aberrations, fluorescence volumes and PSF banks are generated here from fixed
seeds (NumPy PCG64 streams, bit-reproducible across machines).

Refractive-index screens: seeded uniform noise, Gaussian-filtered (periodic)
with ``sigma`` voxels, scaled to the requested RMS of Delta-n over the
background index.  MaoMi's propagation consumes raw occupancy fields whose
phase per voxel is ``raw * n_diff * 2*pi / (lambda_um * vres)``
(optics.py:232), so a slab of ``t`` voxels with perturbation ``dn`` has
``raw = t * dn / n_diff`` (the perturbation is held constant through each
slab's thickness).
"""

from dataclasses import replace

import numpy as np
from scipy import ndimage

#: Zernike modes (Noll-style index of the reference's ``zernike``) aberrated at benchmark size
ZERNIKE_MODES = tuple(range(4, 12))


def unit_noise(shape2d, sigma, rng):
    """Zero-mean, unit-RMS, Gaussian-correlated 2-D noise (float64)."""
    a = rng.random(shape2d) - 0.5
    a = ndimage.gaussian_filter(a, sigma, mode="wrap")
    a -= a.mean()
    return a / np.sqrt(np.mean(a * a))


def raw_fields(config, shapes, *, sigma, rms, seed):
    """Raw A/B/C occupancy fields (float32, shapes from ``field_shapes``).

    Stage A and C screens are slabs of ``prop_um * vres`` voxels, stage B
    screens one voxel; each screen gets an independent noise draw."""
    rng = np.random.default_rng(seed)
    pc = int(round(config.prop_um * config.vres))
    out = []
    for part, shape in enumerate(shapes):
        thick = 1 if part == 1 else pc
        field = np.empty(shape, np.float32)
        for z in range(shape[2]):
            field[..., z] = (unit_noise(shape[:2], sigma, rng) * (thick * rms / config.n_diff)).astype(np.float32)
        out.append(field)
    return out


def zernike_weights(config, seed, rms_rad=0.1, modes=ZERNIKE_MODES):
    """Per-mode weights (``OpticalConfig.zernike_weights``) whose phase is
    N(0, rms_rad) radians: the pupil phase is 2*pi*n*w*Z (_optical_math.py:183,251)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(max(modes))
    w[np.array(modes) - 1] = rng.normal(0.0, rms_rad, len(modes)) / (2 * np.pi * config.n)
    return tuple(float(v) for v in w)


def small_stage_config(cls):
    """128x128-window stage: 3x3 sites, 16 screens (4+10+... mapped geometry)."""
    return cls(volume_um=(64.0, 64.0, 8.0), vres=2.0, ss=1, depth_um=24.5,
               psf_um=(10.0, 10.0, 5.0), prop_um=10.0, tail_um=30.0, propcrop=False)


def benchmark_stage_config(cls, *, zernike_seed=11):
    """256x256-window stage: 65x65 = 4,225 sites, 60 screens (10 + 46 + 4),
    512x512 mask, circular pupil with Zernike modes 4-11 of N(0, 0.1 rad)."""
    cfg = cls(volume_um=(256.0, 256.0, 30.0), vres=2.0, ss=1, depth_um=42.5,
              psf_um=(20.0, 20.0, 23.0), prop_um=5.0, tail_um=20.0, propcrop=False)
    return replace(cfg, zernike_weights=zernike_weights(cfg, zernike_seed))


def somata_volume(shape=(256, 256, 16), count=400, seed=3, voxel_um=(1.0, 1.0, 1.0),
                  radii_um=(4.0, 7.0), background=0.05):
    """Fluorescence volume of seeded ellipsoidal somata (log-normal brightness,
    mu=0, sigma=0.5) on a constant background, float32."""
    rng = np.random.default_rng(seed)
    vol = np.full(shape, background, np.float64)
    grid = np.meshgrid(*[(np.arange(s) + 0.5) * v for s, v in zip(shape, voxel_um)], indexing="ij")
    extent = np.array(shape) * np.array(voxel_um)
    for _ in range(count):
        c = rng.uniform(0, extent)
        r = rng.uniform(*radii_um, 3)
        b = rng.lognormal(0.0, 0.5)
        lo = np.maximum(((c - r) / voxel_um).astype(int), 0)
        hi = np.minimum(((c + r) / voxel_um).astype(int) + 1, shape)
        sl = tuple(slice(a, b_) for a, b_ in zip(lo, hi))
        d = sum(((g[sl] - ci) / ri) ** 2 for g, ci, ri in zip(grid, c, r))
        vol[sl] += b * (d <= 1.0)
    return vol.astype(np.float32)


def psf_bank_kernels(nodes=(16, 16), kernel=(33, 33, 9), depths=4, seed=5):
    """Positive, smoothly varying local PSF kernels (depths, X, Y, kx, ky, kz):
    an anisotropic Gaussian focus whose width, tilt and gain vary across the
    field and with depth (a stand-in for propagated excitation PSFs)."""
    rng = np.random.default_rng(seed)
    kx, ky, kz = [np.arange(k) - k // 2 for k in kernel]
    X, Y, Z = np.meshgrid(kx, ky, kz, indexing="ij")
    out = np.empty((depths,) + tuple(nodes) + tuple(kernel), np.float64)
    for d in range(depths):
        phase = rng.uniform(0, 2 * np.pi, 4)
        for i in range(nodes[0]):
            for j in range(nodes[1]):
                u, v = i / max(nodes[0] - 1, 1), j / max(nodes[1] - 1, 1)
                sx = 3.0 + 1.5 * np.sin(2 * np.pi * u + phase[0]) + 0.3 * d
                sy = 3.0 + 1.5 * np.cos(2 * np.pi * v + phase[1]) + 0.3 * d
                sz = 2.0 + 0.5 * np.sin(2 * np.pi * (u + v) + phase[2])
                tilt = 0.3 * np.sin(2 * np.pi * u * v + phase[3])
                gain = 1.0 + 0.5 * u - 0.3 * v + 0.1 * d
                xr = X + tilt * Z
                out[d, i, j] = gain * np.exp(-(xr / sx) ** 2 - (Y / sy) ** 2 - (Z / sz) ** 2) + 1e-6
    return out.astype(np.float32)


def propagated_psf_bank(cls, *, nodes=16, kernel=(33, 33, 9), depths_um=(0.0, 16.0 / 3, 32.0 / 3, 16.0),
                        fov_um=256.0, base_depth_um=30.0, sigma=3.0, rms=0.015, seed=21, device="cuda"):
    """Depth bank of local excitation PSFs made by the optical stage itself.

    For each bank depth d the stage runs on a tissue block of ``fov_um`` x
    ``fov_um`` x 16 um at 1 um voxels (vres 1, no supersampling) focused at ``base_depth_um + d``,
    with scattering screens of the benchmark recipe (``sigma`` voxels, RMS
    ``rms``), over a ``nodes`` x ``nodes`` lattice of sites; each site's focal
    |E|^4 PSF (``kernel[0] + 1`` x ``kernel[1] + 1`` x ``kernel[2]`` at 1 um)
    is trimmed by its first row and column to ``kernel``, which keeps the
    focus at index ``kernel // 2``.  Returns (kernels (depths, nodes, nodes,
    kx, ky, kz) float64, node positions in um (shared by x and y), depths)."""
    from .fixed import field_shapes, run_stage
    kx, ky, kz = kernel
    ticks = np.round(np.linspace(0.0, fov_um, nodes))
    pts = np.stack(np.meshgrid(ticks, ticks, indexing="ij"), -1).reshape(-1, 2)
    out = np.empty((len(depths_um), nodes, nodes, kx, ky, kz))
    for k, d in enumerate(depths_um):
        cfg = cls(volume_um=(fov_um, fov_um, 16.0), vres=1.0, ss=1, depth_um=base_depth_um + float(d),
                  psf_um=(float(kx + 1), float(ky + 1), float(kz)), prop_um=5.0, tail_um=20.0, propcrop=False)
        raw = raw_fields(cfg, field_shapes(cfg), sigma=sigma, rms=rms, seed=seed + k)
        psf = run_stage(cfg, raw, pts, device=device, tails=False)["psf_3d"]
        out[k] = np.maximum(psf[:, 1:, 1:, :kz], 0.0).reshape(nodes, nodes, kx, ky, kz)
    return out, ticks, np.asarray(depths_um, float)
