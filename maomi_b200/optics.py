"""Optical configuration, the pupil and the CUDA optical stage entry point.

``OpticalConfig`` carries the same fields, defaults and derived parameters as
maomi/optics.py:21-72.  ``pupil`` (optics.py:90-117) evaluates the Gaussian
beam, aperture, focusing phase and Zernike or custom phase in FP64 on the GPU
and returns complex64.  ``propagate`` (optics.py:200-381) returns the same
result dictionary as the reference's CPU stage, computed by the CUDA path.
"""

from dataclasses import dataclass

import numpy as np

from . import _lib
from ._optical_math import PsfParams, VolParams, gaussian_beam_size, zernike_terms
from .excitation import excitation_order


@dataclass
class OpticalConfig:
    volume_um: tuple = (32.0, 32.0, 10.0)
    depth_um: float = 30.0
    vres: float = 1.0
    NA: float = 0.6
    objNA: float = 0.8
    n: float = 1.35
    wavelength_um: float = 0.92
    focal_length_mm: float = 4.5
    ss: int = 2
    psf_um: tuple = (8.0, 8.0, 10.0)
    prop_um: float = 5.0
    tail_um: float = 20.0
    n_diff: float = 0.02
    hemoabs: float = 0.0155194235
    propcrop: bool = True
    scatter_scales_um: tuple = (0.51, 1.56, 4.52, 14.78)
    scatter_weights: tuple = (0.57, 0.29, 0.19, 0.15)
    seed: int = 20260927
    scaling: str = "two-photon"
    temporal_length_um: float = 10.0
    zernike_weights: tuple = ()

    def parameters(self):
        """(VolParams, PsfParams) with the padded vascular extent ``vasc_sz``."""
        excitation_order(self)
        if not np.isfinite(self.temporal_length_um) or self.temporal_length_um <= 0:
            raise ValueError("Positive temporal length required")
        p = PsfParams(NA=self.NA, objNA=self.objNA, n=self.n, lambda_exc=self.wavelength_um,
                      obj_fl=self.focal_length_mm, ss=self.ss, psf_sz=np.array(self.psf_um),
                      prop_sz=self.prop_um, taillength=self.tail_um, n_diff=self.n_diff,
                      propcrop=self.propcrop, fastmask=False,
                      zernikeWt=(np.asarray(self.zernike_weights, dtype=float).ravel()
                                 if len(self.zernike_weights) else None))
        v = VolParams(vol_sz=np.array(self.volume_um), vres=self.vres, vol_depth=self.depth_um, verbose=0)
        v.vasc_sz = (gaussian_beam_size(p, self.depth_um + self.volume_um[2] / 2) + v.vol_sz
                     + np.array([0, 0, self.depth_um]))
        return v, p


def locations(volume_um, count_per_axis):
    """Explicit (X, Y) microns; one sample is the FOV centre (optics.py:75-87)."""
    axes = [np.linspace(0, volume_um[i], count_per_axis) if count_per_axis > 1 else np.array([volume_um[i] / 2])
            for i in (0, 1)]
    return np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 2)


def _pupil_grid(config):
    """(n, D1, rad, objrad, k, fl) of _optical_math.generate_ba:242-251."""
    v, p = config.parameters()
    fl = float(config.focal_length_mm / 1000.0)
    d2 = float(1e-6 * (1.0 / config.vres) / config.ss)
    npts = np.float32(1e-6 * (v.vasc_sz[:2] - v.vol_sz[:2]) / d2)
    beam = gaussian_beam_size(p, fl * 1e6)
    d1 = float(max(beam) / 1e6 / min(npts))
    nre = float(config.n)
    rad = float(np.tan(np.arcsin(config.NA / nre)) * fl)
    objrad = float(np.tan(np.arcsin(config.objNA / nre)) * fl)
    k = 2 * nre * np.pi / float(config.wavelength_um * 1e-6)
    return int(npts[0]), d1, rad, objrad, k, fl


def pupil(config, *, custom_phase=None, phase_units="radians", phase_aperture="objective", device="cuda"):
    """Input pupil field (complex64, on ``device``), FP64 arithmetic on the GPU.

    Zernike weights come from ``config.zernike_weights`` (mode j uses weight
    j-1, phase 2*pi*n*w*Z_j); a ``custom_phase`` replaces them and is sampled
    nearest-neighbour over the objective or excitation aperture."""
    import torch
    _lib.require_cuda(device)
    if custom_phase is not None and (phase_units not in ("radians", "waves")
                                     or phase_aperture not in ("objective", "excitation")):
        raise ValueError("Explicit phase_units / phase_aperture required")
    n, d1, rad, objrad, k, fl = _pupil_grid(config)
    desc = _lib.PupilDesc(n=n, pitch=d1, beam_radius=rad, aperture=objrad, k=k, focal_length=fl)
    if custom_phase is None and len(config.zernike_weights):
        abb = np.asarray(config.zernike_weights, dtype=float).ravel() * config.wavelength_um * 1e-6
        modes = [int(i) for i in np.nonzero(abb)[0]]
        if len(modes) > 32:
            raise ValueError("At most 32 nonzero Zernike modes are supported")
        coef, mm, mcos, ntm, tcoef, tpow = [], [], [], [], [], []
        for i in modes:
            norm, m, use_cos, terms = zernike_terms(i + 1)
            coef.append(abb[i] * norm)
            mm.append(m)
            mcos.append(int(use_cos))
            ntm.append(len(terms))
            tcoef += [c for c, _ in terms]
            tpow += [e for _, e in terms]
        arrays = [_lib.host_array(coef, _lib.c_double), _lib.host_array(mm, _lib.c_int),
                  _lib.host_array(mcos, _lib.c_int), _lib.host_array(ntm, _lib.c_int),
                  _lib.host_array(tcoef, _lib.c_double), _lib.host_array(tpow, _lib.c_int)]
        desc.nmodes = len(modes)
        (desc.mode_coef, desc.mode_m, desc.mode_cos, desc.mode_nterms, desc.term_coef, desc.term_pow) = arrays
    if custom_phase is not None:
        ph = _lib.upload(np.ascontiguousarray(custom_phase, np.float32), device)
        if ph.ndim != 2:
            raise ValueError("custom_phase must be a 2-D array")
        na = config.objNA if phase_aperture == "objective" else config.NA
        desc.custom_phase = ph.data_ptr()
        desc.custom_h, desc.custom_w = ph.shape
        desc.custom_radius = float(np.tan(np.arcsin(na / config.n)) * fl)
        desc.custom_scale = 2 * np.pi if phase_units == "waves" else 1.0
    out = torch.empty((n, n), dtype=torch.complex64, device=device)
    scratch = torch.empty(n * n + 2 * 1024 + 8, dtype=torch.float64, device=device)
    # mm_pupil copies the host tables into the launch parameters before it
    # returns, and the device buffers are stream-ordered: no synchronisation
    _lib.check(_lib.load().mm_pupil(desc, _lib.ptr(out), _lib.ptr(scratch), _lib.stream_of(device)), "pupil")
    return out


def propagate(config, raw_fields, points_um, *, uin=None, device="cuda", save_full=False, phase_mode="auto",
              phase_memory_limit_mb=256):
    """The optical stage on the GPU with the result dictionary of
    maomi/optics.py:200-381 (``psf_3d``, ``psf``, ``mask``, ``psfT``/``psfB``...).

    ``save_full`` and ``phase_mode`` are accepted for signature compatibility:
    the CUDA path always keeps full phase volumes on the device and never
    stores untouched planes."""
    from .fixed import run_stage
    if phase_mode not in ("auto", "full", "window"):
        raise ValueError("phase_mode must be auto/full/window")
    res = run_stage(config, raw_fields, points_um, uin=uin, device=device, tails=True)
    res["mask_mode"] = "explicit_full_paths_v4"
    res["scattering_replay"] = "provided_raw_fields"
    res["phase_mode"] = "full"
    return res


def _collection_disks(config, vessel_shape):
    """(start, disk) per slab of ``pc`` vessel planes: the normalised disk of
    the collection cone at the slab's mid depth (optics.py:390-404), or None
    where the reference skips the slab (cone apex above it, or no pixel)."""
    r = config.vres
    pc = int(round(config.prop_um * r))
    slope = np.tan(np.arcsin(config.objNA / config.n))
    x = np.arange(-vessel_shape[0] / 2, vessel_shape[0] / 2)[:, None]
    y = np.arange(-vessel_shape[1] / 2, vessel_shape[1] / 2)[None, :]
    out = []
    for start in range(0, vessel_shape[-1], pc):
        radius = r * slope * (config.depth_um + config.volume_um[2] / 2 - (start / pc + 0.5) * config.prop_um)
        inside = (x * x + y * y <= radius * radius) if radius > 0 else np.zeros((1, 1), bool)
        rows, cols = np.nonzero(inside.any(1))[0], np.nonzero(inside.any(0))[0]
        if not len(rows):
            out.append((start, None))
            continue
        disk = inside[rows[0]:rows[-1] + 1, cols[0]:cols[-1] + 1].astype(np.float32)
        out.append((start, disk / disk.sum()))
    return out


def collection_mask(vessels, config, *, device=None):
    """NAOMi's depth-dependent collection disk and hemoglobin absorption
    (maomi/optics.py:384-409) on the GPU.

    Every slab of ``pc`` vessel planes is summed and convolved ('same',
    centred as SciPy does) with the normalised disk of the collection cone at
    the slab's depth; the slabs' disks share one kernel stack (each placed so
    that one crop serves all), so the sum over slabs is one pass of the
    plane-convolution engine; the centre crop of the FOV becomes the
    transmission 10^(-total / vres * hemoabs).  Float32 like the reference;
    NumPy vessels give a NumPy mask, device tensors a device tensor."""
    import torch
    from ._scan import KernelSpectrum, as_device, transform_size
    dev = device if device is not None else (vessels.device if isinstance(vessels, torch.Tensor) and vessels.is_cuda
                                             else "cuda")
    _lib.require_cuda(dev)
    v = as_device(vessels, dev, torch.float32)
    if v.ndim != 3:
        raise ValueError("vessels must be an X,Y,Z volume")
    r = config.vres
    pc = int(round(config.prop_um * r))
    shape = np.round(np.array(config.volume_um[:2]) * r).astype(int)
    off = (np.array(v.shape[:2]) - shape) // 2
    disks = _collection_disks(config, tuple(v.shape))
    live = [d for _, d in disks if d is not None]
    if not live:
        ones = torch.ones(tuple(int(s) for s in shape), dtype=torch.float32, device=dev)
        return ones if isinstance(vessels, torch.Tensor) else ones.cpu().numpy()
    # one crop for every slab: disk (dx, dy) with SciPy's 'same' start
    # (d - 1)//2 sits at offset C - (d - 1)//2 of a common frame
    cx = max((d.shape[0] - 1) // 2 for d in live)
    cy = max((d.shape[1] - 1) // 2 for d in live)
    kx = max(cx - (d.shape[0] - 1) // 2 + d.shape[0] for d in live)
    ky = max(cy - (d.shape[1] - 1) // 2 + d.shape[1] for d in live)
    stack = np.zeros((kx, ky, len(disks)), np.float32)
    for s, (_, d) in enumerate(disks):
        if d is not None:
            ox, oy = cx - (d.shape[0] - 1) // 2, cy - (d.shape[1] - 1) // 2
            stack[ox:ox + d.shape[0], oy:oy + d.shape[1], s] = d
    crop = (cx + int(off[0]), cy + int(off[1]))
    X, Y = int(shape[0]), int(shape[1])
    # every source row must fit the transform as well as the kept window
    fx = transform_size(max(crop[0] + X, v.shape[0] + kx - 1 - crop[0], v.shape[0]))
    fy = transform_size(max(crop[1] + Y, v.shape[1] + ky - 1 - crop[1], v.shape[1]))
    spec = KernelSpectrum(_lib.upload(stack, dev), fx, fy)
    total = torch.empty((X, Y), dtype=torch.float32, device=dev)
    spec.convolve(v, zrule=_lib.MM_SCAN_SUM_Z, out=total, crop=crop, out_shape=(X, Y), out_planes=1, group=pc)
    mask = torch.pow(10.0, -total / r * config.hemoabs)
    return mask if isinstance(vessels, torch.Tensor) else mask.cpu().numpy()
