"""CPU restatement of MaoMi's optical stage (TEST INFRASTRUCTURE ONLY).

Every function restates one reference routine; the reference location is given
as ``path:line`` inside the MaoMi 0.8.0b1 source tree.  Arithmetic follows the
reference's own order of operations so that the FP32 restatement reproduces the
reference's FP32 rounding (PyTorch casts Python/NumPy scalars to the tensor
dtype before each operation; the helpers ``_s`` below do the same), and the
FP64 restatement reproduces the reference's FP64 run (pupil built under a
float64 default dtype, complex128 ``uin`` and float64 raw fields).

The array type of the input pupil selects the precision: complex64 -> FP32
oracle, complex128 -> FP64 oracle.  FFTs use ``scipy.fft`` (pocketfft, the
same library family the reference reaches through ``torch.fft`` on CPU).
"""

from math import factorial
from types import SimpleNamespace

import numpy as np
from scipy import fft as sfft
from scipy.spatial.distance import cdist

ORDERS = {"one-photon": 1, "two-photon": 2, "three-photon": 3, "temporal-focusing": 2}

#: worker threads used by the FFTs (set by the CPU baseline; 1 in tests)
FFT_WORKERS = 1


def _s(dtype, value):
    """Cast a scalar the way PyTorch does before a tensor-scalar operation."""
    return np.asarray(value).astype(dtype)[()]


def _rdiv(rdt, z, value):
    """complex tensor / Python scalar: PyTorch multiplies by the reciprocal."""
    return z * _s(rdt, 1 / value)


def _cdt(rdt):
    return np.complex64 if np.dtype(rdt) == np.float32 else np.complex128


def _cis(arg):
    """exp(1j*arg) for a real array, in the matching complex precision."""
    return np.exp(arg.astype(_cdt(arg.dtype)) * 1j).astype(_cdt(arg.dtype))


# ---------------------------------------------------------------- geometry --

def gaussian_beam_size(objNA, nidx, dist, apod=2.0):
    """_optical_math.py:116-118."""
    radius = np.ceil(np.tan(np.arcsin(objNA / nidx)) * dist * 1.5) * apod
    return np.array([radius, radius, 0], dtype=np.float32)


def excitation_order(cfg):
    """excitation.py:8-11."""
    if cfg.scaling not in ORDERS:
        raise ValueError(f"Unknown excitation scaling: {cfg.scaling}")
    return ORDERS[cfg.scaling]


def temporal_profile(size, length_um, dz_um, *, legacy_offset=0.0):
    """excitation.py:14-29."""
    rayleigh = length_um / (dz_um * 2 * np.sqrt(3))
    indices = np.ceil(size / 2) - np.arange(1, size + 1) + legacy_offset * dz_um
    return 1 / np.sqrt(1 + (indices / rayleigh) ** 2)


def axial_profile(cfg, size, part="focus"):
    """excitation.py:32-49."""
    if cfg.scaling != "temporal-focusing":
        return np.ones(size, np.float32)
    if part == "focus":
        dz, offset = 1 / cfg.vres, 0.0
    else:
        pp = cfg.prop_um * cfg.vres
        depth = cfg.psf_um[2] * cfg.vres
        dz = pp / cfg.vres
        offset = ((depth * cfg.vres + 2 * pp) / (pp * pp) if part == "top"
                  else -depth * cfg.vres / (pp * pp))
    return temporal_profile(size, cfg.temporal_length_um, dz, legacy_offset=offset).astype(np.float32)


def center_slice(n, m):
    """_propagation.py:9-12."""
    if m > n or (n - m) % 2:
        raise ValueError(f"Incompatible centered grids {n},{m}")
    return slice((n - m) // 2, (n + m) // 2)


def field_shapes(cfg):
    """fixed.py:36-56 (raw A/B/C occupancy shapes)."""
    r = cfg.vres
    n = int(round(gaussian_beam_size(cfg.objNA, cfg.n, cfg.depth_um + cfg.volume_um[2] / 2)[0] * r))
    n2 = (int(round(min(max(gaussian_beam_size(cfg.objNA, cfg.n, cfg.psf_um[2] / 2, 3)) * r * 2, n)))
          if cfg.propcrop else n)
    za = int(round((cfg.depth_um + cfg.volume_um[2] / 2 - cfg.psf_um[2] / 2) * r))
    zb = int(round(cfg.psf_um[2] * r))
    pc = int(round(cfg.prop_um * r))
    nc = int(round(cfg.tail_um * r))
    xy = np.round(np.asarray(cfg.volume_um[:2]) * r).astype(int)
    return [(int(xy[0] + n), int(xy[1] + n), int(np.ceil(za / pc))),
            (int(xy[0] + n2), int(xy[1] + n2), zb),
            (int(xy[0] + n), int(xy[1] + n), int(np.ceil(nc / pc)))]


def geometry(cfg, raw_shapes):
    """_propagation.py:15-56."""
    r, ss = cfg.vres, cfg.ss
    vol = np.array(cfg.volume_um)
    vasc = (gaussian_beam_size(cfg.objNA, cfg.n, cfg.depth_um + cfg.volume_um[2] / 2)
            + vol + np.array([0, 0, cfg.depth_um]))
    n = int(round((vasc[0] - vol[0]) * r * ss))
    n2 = (int(round(min(max(gaussian_beam_size(cfg.objNA, cfg.n, cfg.psf_um[2] / 2, 3)) * r * 2 * ss, n)))
          if cfg.propcrop else n)
    if n % 2 and not n2 % 2:
        n2 -= 1
    fl = np.float32(cfg.focal_length_mm / 1000)
    d1 = np.float32(max(gaussian_beam_size(cfg.objNA, cfg.n, float(fl * 1e6))) / 1e6 / n)
    d2 = np.float32(1e-6 / r / ss)
    za = r * (cfg.depth_um + cfg.volume_um[2] / 2 - cfg.psf_um[2] / 2)
    pc = cfg.prop_um * r
    a, b, c = [s[-1] for s in raw_shapes]
    positions = [
        (np.r_[0, np.arange(a) + (za % pc) / pc] if za % pc else np.arange(a + 1)) * cfg.prop_um * 1e-6,
        np.arange(b + 1) / r * 1e-6,
        np.r_[np.arange(c) * cfg.prop_um, cfg.tail_um] * 1e-6,
    ]
    cut = max(0, int(np.ceil((za - cfg.tail_um * r) / pc)))
    if cut >= len(positions[0]) - 1:
        raise ValueError("Top tail has no extent")
    focal_shape = np.round(np.array(cfg.psf_um[:2]) * r * ss).astype(int)
    return SimpleNamespace(n=n, n2=n2, fl=fl, d1=d1, d2=d2,
                           wvl=np.float32(cfg.wavelength_um * 1e-6), nr=np.float32(cfg.n),
                           z=positions, cut=cut, focal_shape=focal_shape,
                           crop=center_slice(n, n2),
                           focal_crop=tuple(center_slice(n2, int(k)) for k in focal_shape))


def edge_apodization(size, rdt):
    """_propagation.py:59-61 (super-Gaussian order-16 edge window)."""
    axis = np.arange(-size / 2, size / 2, dtype=rdt) / _s(rdt, 0.47 * size)
    return np.exp(-axis[:, None] ** 16) * np.exp(-axis[None, :] ** 16)


# ------------------------------------------------------------------- pupil --

def _zidx(i, j):
    """_optical_math.py:150-157."""
    idx = int(np.ceil(np.sqrt(0.25 + 2 * i) - 1.5))
    if j == 1:
        return idx
    t = i - (idx + 1) * idx / 2
    return int(((idx + 1) % 2) * 2 * np.floor(t / 2) + (idx % 2) * (2 * np.ceil(t / 2) - 1))


def _zrf(n, m, r):
    """_optical_math.py:137-147."""
    out = np.zeros_like(r)
    for s in range(int((n - m) / 2) + 1):
        num = ((-1) ** s) * factorial(int(n - s))
        den = factorial(int(s)) * factorial(int((n + m) / 2 - s)) * factorial(int((n - m) / 2 - s))
        out += _s(r.dtype, num / den) * (r ** (n - 2 * s))
    return out


def zernike(i, x, y):
    """_optical_math.py:160-173."""
    theta = np.arctan2(y, x)
    r = np.sqrt(x ** 2 + y ** 2)
    n, m = _zidx(i, 1), _zidx(i, 2)
    if m == 0:
        return _s(x.dtype, np.sqrt(n + 1)) * _zrf(n, 0, r)
    trig = np.cos(_s(x.dtype, m) * theta) if i % 2 == 0 else np.sin(_s(x.dtype, m) * theta)
    return _s(x.dtype, np.sqrt(2 * (n + 1))) * _zrf(n, m, r) * trig


def generate_ba(cfg, rdt, *, zernike_weights="config"):
    """_optical_math.py:232-296 for the Gaussian beam (generate_gaussian_profile
    :121-134, apply_zernike :187-197).  ``rdt`` plays the role of the
    reference's default torch dtype."""
    vasc = gaussian_beam_size(cfg.objNA, cfg.n, cfg.depth_um + cfg.volume_um[2] / 2) + np.array(cfg.volume_um)
    fl = float(cfg.focal_length_mm / 1000.0)
    D2 = float(1e-6 * (1.0 / cfg.vres) / cfg.ss)
    N = np.float32(1e-6 * (vasc[:2] - np.array(cfg.volume_um)[:2]) / D2)
    beam = gaussian_beam_size(cfg.objNA, cfg.n, fl * 1e6)
    D1 = float(max(beam) / 1e6 / min(N))
    nre = float(cfg.n)
    rad = float(np.tan(np.arcsin(cfg.NA / nre)) * fl)
    objrad = float(np.tan(np.arcsin(cfg.objNA / nre)) * fl)
    k = 2 * nre * np.pi / float(cfg.wavelength_um * 1e-6)
    xr = np.arange(-N[0] / 2, N[0] / 2, dtype=rdt) * _s(rdt, D1)
    yr = np.arange(-N[1] / 2, N[1] / 2, dtype=rdt) * _s(rdt, D1)
    Y, X = np.meshgrid(yr, xr, indexing="ij")
    rho2 = X ** 2 + Y ** 2
    amp = np.exp(-(X ** 2 + Y ** 2) / _s(rdt, rad ** 2))
    amp = amp * (rho2 < _s(rdt, objrad ** 2)).astype(rdt)
    focus = _s(rdt, -k / (2 * fl)) * rho2
    u = amp.astype(_cdt(rdt)) * _cis(focus)
    w = cfg.zernike_weights if zernike_weights == "config" else zernike_weights
    if w is not None and len(w):
        abb = np.asarray(w, dtype=float).ravel() * cfg.wavelength_um * 1e-6
        if np.any(abb != 0):
            xs, ys = X / _s(rdt, objrad), Y / _s(rdt, objrad)
            # The reference accumulates this phase in a float32 buffer in both
            # precisions (_optical_math.py:190), so the factor is complex64.
            phase = np.zeros(xs.shape, np.float32)
            for i in np.nonzero(abb)[0]:
                phase = (phase.astype(rdt) + _s(rdt, abb[i]) * zernike(i + 1, xs, ys)).astype(np.float32)
            phase = phase - phase.mean(dtype=np.float32)
            u = u * _cis(np.float32(k) * phase)
    return u


def pupil(cfg, rdt=np.float64, *, custom_phase=None, phase_units="radians", phase_aperture="objective"):
    """optics.py:90-117 (custom phases are sampled nearest-neighbour on the
    objective or excitation aperture, align_corners=True, zero padding)."""
    if custom_phase is None:
        return generate_ba(cfg, rdt)
    if phase_units not in ("radians", "waves") or phase_aperture not in ("objective", "excitation"):
        raise ValueError("Explicit phase_units / phase_aperture required")
    u = generate_ba(cfg, rdt, zernike_weights=None)
    h, w = u.shape
    fl = cfg.focal_length_mm / 1000
    d1 = max(gaussian_beam_size(cfg.objNA, cfg.n, fl * 1e6)) / 1e6 / min(h, w)
    na = cfg.objNA if phase_aperture == "objective" else cfg.NA
    rad = np.tan(np.arcsin(na / cfg.n)) * fl
    y, x = np.meshgrid(np.arange(-h / 2, h / 2, dtype=rdt) * _s(rdt, d1),
                       np.arange(-w / 2, w / 2, dtype=rdt) * _s(rdt, d1), indexing="ij")
    gx, gy = x / _s(rdt, rad), y / _s(rdt, rad)
    ph = np.asarray(custom_phase, dtype=rdt)
    H, W = ph.shape
    ix = np.rint(((gx + _s(rdt, 1)) / _s(rdt, 2)) * _s(rdt, W - 1))
    iy = np.rint(((gy + _s(rdt, 1)) / _s(rdt, 2)) * _s(rdt, H - 1))
    inside = (ix >= 0) & (ix <= W - 1) & (iy >= 0) & (iy <= H - 1)
    sampled = np.zeros_like(gx)
    sampled[inside] = ph[iy[inside].astype(int), ix[inside].astype(int)]
    scale = 2 * np.pi if phase_units == "waves" else 1
    return u * _cis(sampled * _s(rdt, scale))


# --------------------------------------------------------------- numerics --

def _cubic(x):
    """numerics.py:8-12 (Keys cubic, a = -0.5)."""
    a = np.abs(x)
    return (((1.5 * a - 2.5) * a * a + 1) * (a <= 1)
            + (((-0.5 * a + 2.5) * a - 4) * a + 2) * ((a > 1) & (a < 2)))


def resize_plan(n, scale):
    """Index/weight table of numerics.py:15-39 for one axis (float64)."""
    m = int(np.ceil(n * scale))
    u = (np.arange(m) + 0.5) / scale - 0.5
    width = 4 / min(scale, 1)
    left = np.floor(u - width / 2).astype(int)
    idx = left[:, None] + np.arange(int(np.ceil(width)) + 2)[None, :]
    weights = _cubic((u[:, None] - idx) * min(scale, 1)) * min(scale, 1)
    weights /= weights.sum(1, keepdims=True)
    idx %= 2 * n
    idx = np.where(idx < n, idx, 2 * n - 1 - idx)
    return idx, weights


def resize_xy(a, scale):
    """numerics.py:15-39 (MATLAB imresize bicubic with antialiasing, XY only)."""
    out = a
    rdt = np.asarray(a).real.dtype
    for axis in (0, 1):
        idx, weights = resize_plan(out.shape[axis], scale)
        moved = np.moveaxis(out, axis, 0)
        wt = weights.astype(rdt).reshape(weights.shape + (1,) * (moved.ndim - 1))
        out = np.moveaxis((moved[idx] * wt).sum(1), 0, axis)
    return out


def _shift_axis(a, axis, shift):
    size = a.shape[axis]
    src = np.arange(size) - shift
    lo = np.floor(src).astype(int)
    f = (src - lo).astype(a.dtype)
    moved = np.moveaxis(a, axis, 0)
    res = np.zeros_like(moved)
    shape = (-1,) + (1,) * (moved.ndim - 1)
    ok0 = (lo >= 0) & (lo < size)
    ok1 = (lo + 1 >= 0) & (lo + 1 < size)
    res[ok0] += moved[lo[ok0]] * (1 - f[ok0]).reshape(shape)
    res[ok1] += moved[lo[ok1] + 1] * f[ok1].reshape(shape)
    return np.moveaxis(res, 0, axis)


def translate_xy(a, shift):
    """numerics.py:79-90: imtranslate (bilinear, same view, zero fill);
    output(i, j) samples the input at (i - shift, j - shift)."""
    if shift == 0:
        return a.copy()
    return _shift_axis(_shift_axis(a, 0, shift), 1, shift)


def resample_matrix(n, ss):
    """backends/cuda/native.py:27-48: imresize(1/ss) composed with
    imtranslate(ss/2-0.5) as one dense (ceil(n/ss), n) matrix."""
    scale = 1 / ss
    m = int(np.ceil(n * scale))
    shift = ss / 2 - 0.5
    u = (np.arange(m) + 0.5) / scale - 0.5
    width = 4 / scale
    idx = np.floor(u - width / 2).astype(int)[:, None] + np.arange(int(np.ceil(width)) + 2)[None]
    weights = _cubic((u[:, None] - idx) * scale) * scale
    weights /= weights.sum(1, keepdims=True)
    idx %= 2 * n
    idx = np.where(idx < n, idx, 2 * n - 1 - idx)
    matrix = np.zeros((m, n))
    for i in range(m):
        for j, w in zip(idx[i], weights[i]):
            a = int(np.floor(j - shift))
            f = j - shift - a
            if 0 <= a < n:
                matrix[i, a] += w * (1 - f)
            if 0 <= a + 1 < n:
                matrix[i, a + 1] += w * f
    return matrix


def _green(x, y):
    d = np.sqrt(((x[:, None, :] - y[None, :, :]) ** 2).sum(-1))
    with np.errstate(divide="ignore", invalid="ignore"):
        g = d * d * (np.log(d) - 1)
    g[d == 0] = 0
    return g


def v4_coefficients(points, values):
    """numerics.py:122-129: dense FP64 solve of the v4 Green system."""
    p, v = np.asarray(points, float), np.asarray(values, float)
    return np.linalg.solve(_green(p, p), v)


def v4_evaluate(points, coef, queries, chunk=16384):
    """numerics.py:140-153: evaluate r^2(0.5 log r^2 - 1) against coefficients."""
    p = np.asarray(points, float)
    q = np.asarray(queries, float)
    coef = np.asarray(coef, float)
    flat = q.reshape(-1, 2)
    result = np.empty((len(flat),) + coef.shape[1:], dtype=np.float64)
    chunk = min(chunk, max(1, 8_388_608 // len(p)))
    for start in range(0, len(flat), chunk):
        d2 = cdist(flat[start:start + chunk], p, "sqeuclidean")
        with np.errstate(divide="ignore", invalid="ignore"):
            basis = np.log(d2)
            basis *= 0.5
            basis -= 1
            basis *= d2
        basis[d2 == 0] = 0
        result[start:start + chunk] = basis @ coef
    return result.reshape(q.shape[:-1] + coef.shape[1:])


def v4_interpolate(points, values, queries, chunk=16384):
    """numerics.py:93-153 (MATLAB 'v4' biharmonic spline, FP64)."""
    p, v, q = np.asarray(points, float), np.asarray(values, float), np.asarray(queries, float)
    if p.ndim != 2 or p.shape[1] != 2 or not len(p):
        raise ValueError("points must be a nonempty (N, 2) array")
    shape = q.shape[:-1] + v.shape[1:]
    if len(p) == 1:
        return np.broadcast_to(v[0], shape).copy()
    if not q.reshape(-1, 2).shape[0]:
        return np.empty(shape, dtype=np.float64)
    return v4_evaluate(p, v4_coefficients(p, v), q, chunk)


def _fft2(a):
    return sfft.fft2(a, axes=(-2, -1), workers=FFT_WORKERS)


def _ifft2(a):
    return sfft.ifft2(a, axes=(-2, -1), workers=FFT_WORKERS)


def fresnel(u, wavelength, dx, z, phi, nidx, *, crop=None, save_from=0, return_all=False):
    """numerics.py:156-210: scaled multi-screen Fresnel propagation.

    u: (..., H, W) complex; phi: (..., H, W, screens)."""
    dx, z = np.asarray(dx, float).ravel(), np.asarray(z, float).ravel()
    if len(z) < 2 or len(dx) != len(z) or np.any(np.diff(z) <= 0):
        raise ValueError("Need increasing z and one dx per plane")
    if phi.shape[-1] not in (len(z), len(z) - 1):
        raise ValueError("Wrong number of phase screens")
    h, w = u.shape[-2:]
    rdt = u.real.dtype
    x = np.arange(-h / 2, h / 2, dtype=rdt)[:, None]
    y = np.arange(-w / 2, w / 2, dtype=rdt)[None, :]
    lam = float(wavelength) / float(nidx)
    k = 2 * np.pi / lam
    dz = np.diff(z)
    sc = dx[1:] / dx[:-1]
    t = (x * _s(rdt, dx[0])) ** 2 + (y * _s(rdt, dx[0])) ** 2
    arg = _rdiv(rdt, (_s(rdt, k) * t) * _s(rdt, 1 - sc[0]), 2 * dz[0])
    u = u * _cis(arg) * phi[..., 0]
    saved = []

    def keep(i, field):
        if return_all and i >= save_from:
            saved.append(field[..., crop[0], crop[1]].copy() if crop else field.copy())

    keep(0, u)
    cache = {}
    axes = (-2, -1)
    for i in range(len(dz)):
        key = (float(dz[i]), float(dx[i]), float(sc[i]))
        if key not in cache:
            c = -np.pi * lam * dz[i]
            t = (x / _s(rdt, h * dx[i])) ** 2 + (y / _s(rdt, w * dx[i])) ** 2
            cache[key] = _cis(_rdiv(rdt, _s(rdt, c) * t, sc[i]))
        f = sfft.fftshift(_fft2(sfft.fftshift(_rdiv(rdt, u, sc[i]), axes=axes)), axes=axes)
        u = sfft.ifftshift(_ifft2(sfft.ifftshift(cache[key] * f, axes=axes)), axes=axes)
        if i + 1 < phi.shape[-1]:
            u = u * phi[..., i + 1]
        keep(i + 1, u)
    c = 1 / 2 * k * (sc[-1] - 1) / (sc[-1] * dz[-1])
    t = (x * _s(rdt, dx[-1])) ** 2 + (y * _s(rdt, dx[-1])) ** 2
    out = u * _cis(_s(rdt, c) * t)
    return (out, np.stack(saved, axis=-1)) if return_all else out


def base_field(cfg, g, u, sg):
    """optics.py:222-231: pupil -> tissue top (pitch d1 -> d2), unit L2 norm."""
    rdt = u.real.dtype
    z1 = np.float32(g.fl - (cfg.depth_um + cfg.volume_um[2] / 2) * 1e-6)
    base = fresnel(u, g.wvl, [g.d1, g.d2], [0, z1], np.stack((sg, sg), -1), g.nr)
    return base / _s(rdt, np.linalg.norm(base))


def phase_screens(cfg, raw_fields, rdt):
    """optics.py:232-249 (full phase mode): exp(1j*resize(raw,ss)*scale), (H,W,Z)."""
    scale = cfg.n_diff * 2 * np.pi / (cfg.wavelength_um * cfg.vres)
    return [_cis(resize_xy(np.asarray(a, dtype=rdt), cfg.ss) * _s(rdt, scale)) for a in raw_fields]


# -------------------------------------------------------------- propagate --

def propagate_sites(cfg, raw_fields, points_um, uin, *, phases=None):
    """Per-site loop of optics.py:256-340.

    Returns the raw per-site products: psfs (P,X,Y,Z), per-tail lists of
    profiles (P,planes), weights (P,), convmask images (P,h,w)."""
    r, ss = cfg.vres, cfg.ss
    g = geometry(cfg, [np.shape(a) for a in raw_fields])
    n, n2, wvl, nr = g.n, g.n2, g.wvl, g.nr
    u = np.asarray(uin)
    rdt = u.real.dtype
    order = excitation_order(cfg)
    sg, sg2 = edge_apodization(n, rdt), edge_apodization(n2, rdt)
    base = base_field(cfg, g, u, sg)
    phase = phase_screens(cfg, raw_fields, rdt) if phases is None else phases
    za_pos, zb_pos, zc_pos = g.z
    cut, c, fc = g.cut, g.crop, g.focal_crop
    outputs, tails, weights, profiles = [], [[], []], [[], []], [[], []]
    pts = np.asarray(points_um, float)
    if np.any(pts < 0) or np.any(pts > np.array(cfg.volume_um[:2])):
        raise ValueError("PSF coordinates outside FOV")
    psf_scale = _s(rdt, r * (1e6 * wvl) ** 1.5)
    psf_den = _s(rdt, np.pi * nr)
    for xy in pts:
        offset = xy * r * ss
        if not np.allclose(offset, np.round(offset)):
            raise ValueError("Locations must land on the supersampled grid")
        x, y = np.round(offset).astype(int)
        pa = phase[0][x:x + n, y:y + n] * sg[..., None]
        pb = phase[1][x:x + n2, y:y + n2] * sg2[..., None]
        pcf = phase[2][x:x + n, y:y + n] * sg[..., None]
        ua, top = fresnel(base, wvl, np.full(len(za_pos), g.d2), za_pos, pa, nr,
                          return_all=True, crop=(c, c), save_from=cut)
        ub, focus = fresnel(ua[c, c], wvl, np.full(len(zb_pos), g.d2), zb_pos, pb, nr,
                            return_all=True, crop=fc)
        pad = (n - n2) // 2
        padded = np.pad(ub, ((pad, pad), (pad, pad)))
        _, bottom = fresnel(padded, wvl, np.full(len(zc_pos), g.d2), zc_pos, pcf, nr,
                            return_all=True, crop=(c, c))
        inten = _s(rdt, ss ** 2) * np.abs(focus[..., :-1]) ** (2 * order)
        inten = inten * axial_profile(cfg, inten.shape[-1]).astype(rdt)
        final = (_s(rdt, ss ** 2) * resize_xy(translate_xy(inten, ss / 2 - 0.5), 1 / ss)
                 * psf_scale) / psf_den
        outputs.append(final)
        for j, field in enumerate((top, bottom)):
            inten = _s(rdt, ss ** 2) * np.abs(field) ** (2 * order)
            inten = inten * axial_profile(cfg, field.shape[-1], "top" if j == 0 else "bottom").astype(rdt)
            profiles[j].append(inten.sum((0, 1)))
            inten[..., 0] *= _s(rdt, 0.5)
            inten[..., -1] *= _s(rdt, 0.5)
            weights[j].append(float(inten.sum()) * cfg.prop_um)
            tails[j].append(_s(rdt, ss ** 2) * resize_xy(translate_xy(inten.sum(-1), ss / 2 - 0.5), 1 / ss))
    return dict(psfs=np.stack(outputs), profiles=[np.stack(p) for p in profiles],
                weights=[np.asarray(w) for w in weights], convmasks=[np.stack(t) for t in tails],
                geometry=g, points_um=pts)


def finish(cfg, sites):
    """optics.py:341-381: energies, v4 masks, averaged tails and psfZ."""
    r = cfg.vres
    g = sites["geometry"]
    pts = sites["points_um"]
    psfs = sites["psfs"]
    energies = psfs.sum((1, 2, 3), dtype=np.float64)
    xyshape = np.round(np.array(cfg.volume_um[:2]) * r).astype(int)
    q = np.stack(np.meshgrid(np.arange(xyshape[0]) + 0.5, np.arange(xyshape[1]) + 0.5, indexing="ij"), -1)
    values = np.stack([energies, sites["weights"][0], sites["weights"][1]], 1)
    masks = v4_interpolate(pts * r, values, q)
    mask = masks[..., 0]
    mean = float(mask.mean())
    result = {
        "psf_3d": psfs,
        "psf_raw": psfs.mean(0),
        "psf": np.abs(psfs).mean(0),
        "mask_raw": mask,
        "mask_mean": mean,
        "mask": mask / mean if mean > 0 else mask,
        "points_um": pts,
        "energies": energies,
        "negative_resampling_mass_fraction": float(
            -np.minimum(psfs, 0).sum(dtype=np.float64) / np.abs(psfs).sum(dtype=np.float64)),
    }
    za_pos, _, zc_pos = g.z
    for j, name in enumerate(("psfT", "psfB")):
        profile = sites["profiles"][j].sum(0)
        actual_z = (za_pos[g.cut:] - za_pos[g.cut]) if j == 0 else zc_pos
        out_z = np.arange(round(actual_z[-1] * 1e6 * r) + 1) / r
        interp = np.interp(out_z, actual_z * 1e6, profile)
        tail_mask = masks[..., j + 1]
        tail_mean = float(tail_mask.mean())
        result[name] = {
            "convmask": np.mean(sites["convmasks"][j], 0),
            "weight": float(np.mean(sites["weights"][j])),
            "psfZ": interp / interp.mean() if interp.mean() > 0 else interp,
            "mask_raw": tail_mask,
            "mask_mean": tail_mean,
            "mask": tail_mask / tail_mean if tail_mean > 0 else tail_mask,
            "weights_per_point": sites["weights"][j],
            "profiles_per_point": sites["profiles"][j],
        }
    return result


def propagate(cfg, raw_fields, points_um, uin):
    """optics.py:200-381 (full phase mode): the reference's CPU optical stage."""
    return finish(cfg, propagate_sites(cfg, raw_fields, points_um, uin))


def fixed_locations(cfg, count_per_axis=65):
    """fixed.py:15-33."""
    ticks = np.asarray(cfg.volume_um[:2], float) * cfg.vres * cfg.ss
    axes = [np.round(np.linspace(0, int(round(n)), count_per_axis)) / (cfg.vres * cfg.ss) for n in ticks]
    return np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 2)


def locations(volume_um, count_per_axis):
    """optics.py:75-87."""
    x = np.linspace(0, volume_um[0], count_per_axis) if count_per_axis > 1 else np.array([volume_um[0] / 2])
    y = np.linspace(0, volume_um[1], count_per_axis) if count_per_axis > 1 else np.array([volume_um[1] / 2])
    return np.stack(np.meshgrid(x, y, indexing="ij"), -1).reshape(-1, 2)


def collection_disks(cfg, vessel_shape):
    """Normalised collection disks per slab of ``pc`` vessel planes, or None
    for slabs the reference skips (optics.py:384-404): (start, disk) pairs."""
    r = cfg.vres
    pc = int(round(cfg.prop_um * r))
    out = []
    for start in range(0, vessel_shape[-1], pc):
        depth = (start / pc + 0.5) * cfg.prop_um
        radius = r * np.tan(np.arcsin(cfg.objNA / cfg.n)) * (cfg.depth_um + cfg.volume_um[2] / 2 - depth)
        if radius <= 0:
            out.append((start, None))
            continue
        x = np.arange(-vessel_shape[0] / 2, vessel_shape[0] / 2)[:, None]
        y = np.arange(-vessel_shape[1] / 2, vessel_shape[1] / 2)[None, :]
        disk = (x * x + y * y <= radius * radius).astype(np.float64)
        nz = np.argwhere(disk)
        if len(nz) == 0:
            out.append((start, None))
            continue
        lo, hi = nz.min(0), nz.max(0) + 1
        disk = disk[lo[0]:hi[0], lo[1]:hi[1]]
        out.append((start, disk / disk.sum()))
    return out


def collection_mask(vessels, cfg):
    """optics.py:384-409 in float64: per slab, the vessel occupancy summed over
    the slab convolved ('same', SciPy's centring) with the normalised disk of
    the collection cone at the slab's depth; the centre FOV crop of the sum,
    as hemoglobin transmission 10^(-total / vres * hemoabs)."""
    from scipy.signal import fftconvolve
    a = np.asarray(vessels, np.float64)
    r = cfg.vres
    pc = int(round(cfg.prop_um * r))
    total = np.zeros(a.shape[:2])
    for start, disk in collection_disks(cfg, a.shape):
        if disk is not None:
            total += fftconvolve(a[..., start:start + pc].sum(-1), disk, mode="same")
    shape = np.round(np.array(cfg.volume_um[:2]) * r).astype(int)
    off = (np.array(total.shape) - shape) // 2
    total = total[off[0]:off[0] + shape[0], off[1]:off[1] + shape[1]]
    return 10 ** (-total / r * cfg.hemoabs)
