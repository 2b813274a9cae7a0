"""Per-frame scan operators on the GPU: ``conv2_same``, ``psf_fft``,
``single_scan`` and ``blurred_background``.

Drop-ins for maomi/movie.py:14-102 with the same signatures and error types.
Arrays are X, Y, Z.  Inputs may be NumPy arrays or tensors; NumPy inputs give
NumPy results (copied back once), device tensors give device tensors.  The
frequency-domain objects (``psf_fft``'s result) stay on the device and are
accepted by ``single_scan(frequency_psf=...)`` and
``blurred_background(..., frequency=True)`` exactly where the reference
accepts its NumPy spectra; their ``shape`` is the reference's spectrum shape.

All four run through the plane-convolution engine (``csrc/scan.cu``):
``single_scan`` is the sum over (grouped) planes of the 2-D convolutions,
evaluated as one inverse DFT of the per-bin sum; ``blurred_background``
forms the scaled plane mean on the device (``mm_scan_background``) and
convolves it once.
"""

import numpy as np

from . import _lib
from ._scan import KernelSpectrum, as_device, mask_tensor, real_dtype, transform_size


def _smooth_length(n):
    """movie.py:22-29: the smallest m >= n with no prime factor above 7 (the
    reference's FFT length, which fixes the frequency-domain background crop)."""
    while True:
        m = n
        for prime in (2, 3, 5, 7):
            while m % prime == 0:
                m //= prime
        if m == 1:
            return n
        n += 1


def _check_group(count):
    if isinstance(count, bool) or not isinstance(count, (int, np.integer)) or count < 1:
        raise ValueError("scan_avg must be a positive integer")
    return int(count)


def _device_of(*arrays):
    import torch
    for a in arrays:
        if isinstance(a, torch.Tensor) and a.is_cuda:
            return a.device
    return torch.device("cuda", torch.cuda.current_device())


def _result(t, like):
    import torch
    if isinstance(like, torch.Tensor):
        return t
    return t.cpu().numpy()


class FrequencyPSF:
    """Device spectra of a (grouped) PSF for volumes of one XY shape
    (the object ``psf_fft`` returns; movie.py:37-42).

    ``shape`` is the shape of the reference's spectrum (its FFT lengths and
    the grouped depth); ``kernel`` holds the device half spectra."""

    def __init__(self, volume_shape, psf, scan_avg, device):
        p = as_device(psf, device)
        if not p.is_floating_point():
            p = p.float()
        if p.ndim == 2:
            p = p[..., None]
        if p.ndim != 3:
            raise ValueError("PSF must be X,Y or X,Y,Z")
        real_dtype(p)
        self.scan_avg = _check_group(scan_avg)
        X, Y = int(volume_shape[0]), int(volume_shape[1])
        a, b = int(p.shape[0]), int(p.shape[1])
        self.volume_xy = (X, Y)
        self.shape = (_smooth_length(X + a - 1), _smooth_length(Y + b - 1), -(-int(p.shape[2]) // self.scan_avg))
        # kept windows: floor(k/2) (single_scan, conv2_same) and the
        # frequency-domain background's ceil((S - n - 1)/2)
        cb = [int(np.ceil((s - n - 1) / 2)) for s, n in zip(self.shape[:2], (X, Y))]
        fx = transform_size(max(X + a // 2, X + a - 1 - a // 2, cb[0] + X, X + a - 1 - cb[0]))
        fy = transform_size(max(Y + b // 2, Y + b - 1 - b // 2, cb[1] + Y, Y + b - 1 - cb[1]))
        self.background_crop = tuple(cb)
        self.kernel = KernelSpectrum(p.contiguous(), fx, fy, group=self.scan_avg)
        self.dtype = p.dtype
        self.device = p.device
        self.ndim = 3


def psf_fft(volume_shape, psf, scan_avg=1, *, device=None):
    """Spectra of the PSF grouped by ``scan_avg`` for volumes of
    ``volume_shape`` (movie.py:37-42), kept on the device."""
    dev = device if device is not None else _device_of(psf)
    _lib.require_cuda(dev)
    return FrequencyPSF(volume_shape, psf, scan_avg, dev)


def single_scan(volume, psf, *, scan_avg=1, frequency_psf=None, rana=None, z_start=0, device=None):
    """One XY frame: the sum of the axial slice convolutions, with optional
    grouped Z (movie.py:48-66)."""
    import torch
    if rana is not None and rana is not False:
        return rana.scan_slab(volume, scan_avg=scan_avg, z_start=z_start)
    dev = device if device is not None else _device_of(volume, psf)
    _lib.require_cuda(dev)
    v = as_device(volume, dev)
    if not v.is_floating_point():
        v = v.float()
    p = as_device(psf, dev)
    if v.ndim != 3 or p.ndim != 3 or v.shape[2] != p.shape[2]:
        raise ValueError("Volume slab and PSF must have the same axial length")
    g = _check_group(scan_avg)
    freq = psf_fft(v.shape, p.to(v.dtype), g, device=dev) if frequency_psf is None else frequency_psf
    if not isinstance(freq, FrequencyPSF):
        raise ValueError("frequency_psf must be the result of maomi_b200.movie.psf_fft")
    if freq.shape[2] != -(-int(v.shape[2]) // g):
        raise ValueError("Wrong grouped PSF depth")
    if freq.dtype != v.dtype:
        raise ValueError("frequency_psf was built for another floating type")
    X, Y = int(v.shape[0]), int(v.shape[1])
    a, b = int(p.shape[0]), int(p.shape[1])
    out = torch.empty((X, Y), dtype=v.dtype, device=dev)
    freq.kernel.convolve(v, zrule=_lib.MM_SCAN_SUM_Z, out=out, crop=(a // 2, b // 2), out_shape=(X, Y),
                         out_planes=1, group=g)
    return _result(out, volume)


def conv2_same(image, kernel, *, device=None):
    """Full 2-D convolution cropped at floor(k/2) (movie.py:14-19)."""
    import torch
    dev = device if device is not None else _device_of(image, kernel)
    _lib.require_cuda(dev)
    im = as_device(image, dev)
    if not im.is_floating_point():
        im = im.double()
    k = as_device(kernel, dev, im.dtype)
    if im.ndim != 2 or k.ndim != 2:
        raise ValueError("conv2_same expects 2-D image and kernel")
    X, Y = int(im.shape[0]), int(im.shape[1])
    a, b = int(k.shape[0]), int(k.shape[1])
    spec = KernelSpectrum(k[..., None].contiguous(), transform_size(X + max(a // 2, a - 1 - a // 2)),
                          transform_size(Y + max(b // 2, b - 1 - b // 2)))
    out = torch.empty((X, Y), dtype=im.dtype, device=dev)
    spec.convolve(im[..., None], zrule=_lib.MM_SCAN_EACH_Z, out=out, crop=(a // 2, b // 2), out_shape=(X, Y),
                  out_planes=1)
    return _result(out, image)


def blurred_background(volume, indices, kernel, *, power_ratio=1.0, mask=None, zscale=None, extra_volumes=(),
                       frequency=False, device=None):
    """Port of blurredBackComp2 (movie.py:69-102); indices are zero-based.

    The scaled plane mean is formed on the device, then convolved with the
    spatial kernel (crop floor(k/2)) or, with ``frequency=True``, with the
    spectrum ``psf_fft(volume.shape, kernel)`` returned (crop
    ceil((S - n - 1)/2) of the reference's FFT length S).  The result has
    the volume's floating type."""
    import torch
    dev = device if device is not None else _device_of(volume, kernel)
    _lib.require_cuda(dev)
    v = as_device(volume, dev)
    if not v.is_floating_point():
        v = v.float()
    real_dtype(v)
    idx = np.asarray(indices, int).ravel()
    if idx.size == 0:
        raise ValueError("Background requires at least one axial slice")
    if np.any(idx < 0) or np.any(idx >= v.shape[2]):
        raise ValueError("Invalid background indices")
    scale = (np.asarray(zscale, np.float64).ravel()[:len(idx)]
             if zscale is not None and np.size(zscale) >= len(idx) else np.ones(len(idx)))
    vols = [v] + [as_device(o, dev, v.dtype) for o in extra_volumes]
    vols = [t.contiguous() for t in vols]
    if len(vols) > 4 or any(tuple(t.shape) != tuple(v.shape) for t in vols):
        raise ValueError("extra_volumes must be at most three volumes of the volume's shape")
    X, Y = int(v.shape[0]), int(v.shape[1])
    m = mask_tensor(mask, (X, Y), dev, v.dtype)
    image = torch.empty((X, Y), dtype=v.dtype, device=dev)
    ptrs = (_lib.c_void_p * len(vols))(*[t.data_ptr() for t in vols])
    idx_d = _lib.upload(idx.astype(np.int32), dev)
    scale_d = _lib.upload(scale.astype(np.float64), dev)
    s = vols[0].stride()
    _lib.call("mm_scan_background", int(v.dtype == torch.float64), ptrs, len(vols), s[0], s[1], s[2], X, Y,
              int(v.shape[2]), _lib.ptr(idx_d), _lib.ptr(scale_d), len(idx), float(power_ratio), _lib.ptr(m),
              _lib.ptr(image), _lib.stream_of(dev))
    out = torch.empty((X, Y), dtype=v.dtype, device=dev)
    if frequency:
        if not isinstance(kernel, FrequencyPSF):
            raise ValueError("frequency=True expects the result of maomi_b200.movie.psf_fft")
        if tuple(kernel.volume_xy) != (X, Y):
            raise ValueError("background spectrum was built for another volume shape")
        if kernel.dtype != v.dtype:
            raise ValueError("background spectrum was built for another floating type")
        spec = kernel.kernel
        if spec.planes > 1:
            raise ValueError("frequency-domain background expects a 2-D kernel spectrum")
        spec.convolve(image[..., None], zrule=_lib.MM_SCAN_EACH_Z, out=out, crop=kernel.background_crop,
                      out_shape=(X, Y), out_planes=1)
        return _result(out, volume)
    k = as_device(kernel, dev, v.dtype)
    if k.ndim == 3:
        k = k[:, :, torch.as_tensor(idx, device=dev)].mean(dim=2) if k.shape[2] > 1 else k[:, :, 0]
    if k.ndim != 2:
        raise ValueError("Background kernel must be X,Y or X,Y,Z")
    a, b = int(k.shape[0]), int(k.shape[1])
    spec = KernelSpectrum(k[..., None].contiguous(), transform_size(X + max(a // 2, a - 1 - a // 2)),
                          transform_size(Y + max(b // 2, b - 1 - b // 2)))
    spec.convolve(image[..., None], zrule=_lib.MM_SCAN_EACH_Z, out=out, crop=(a // 2, b // 2), out_shape=(X, Y),
                  out_planes=1)
    return _result(out, volume)


class FrameScanner:
    """The optical part of one frame of the reference's planar movie loop
    (maomi/movie.py:601-679), on the device: the focal slab of the frame's
    activity volume plus the static base, convolved with the PSF over
    ``scan_avg`` plane groups (``single_scan``); the optional extra blur
    (``conv2_same`` of the frame onto itself); and both out-of-focus tails as
    blurred backgrounds of the planes above and below the slab
    (``blurred_background`` with the frequency-domain kernels).  The spectra
    of the PSF, the tail kernels and the blur are built once for the volume
    shape; each frame is then one engine pass for the slab (the base is added
    in the read) and one per tail.  Motion, binning and detector noise follow
    in the reference loop and are not part of this class.

    ``tails``: up to two dicts (top, bottom) with ``kernel`` (2-D, already
    normalised to unit sum), ``weight``, ``mask`` (2-D) and ``zscale``.
    """

    def __init__(self, shape, psf, *, scan_avg=2, tails=(), blur=None, device=None):
        import torch
        dev = device if device is not None else _device_of(psf)
        _lib.require_cuda(dev)
        p = as_device(psf, dev, torch.float32)
        if p.ndim != 3 or len(shape) != 3:
            raise ValueError("FrameScanner needs an X,Y,Z volume shape and an X,Y,Z PSF")
        self.shape, self.depth, self.device = tuple(int(s) for s in shape), int(p.shape[2]), dev
        self.scan_avg = _check_group(scan_avg)
        self.psf_xy = (int(p.shape[0]), int(p.shape[1]))
        self.freq = FrequencyPSF(self.shape, p, self.scan_avg, dev)
        if len(tails) not in (0, 2):
            raise ValueError("Both optical tails are required")
        X, Y = self.shape[:2]
        self.tails = []
        for spec in tails:
            mask = None if spec.get("mask") is None else mask_tensor(spec["mask"], (X, Y), dev, torch.float32)
            zs = spec.get("zscale")
            self.tails.append({"kernel": FrequencyPSF(self.shape, as_device(spec["kernel"], dev, torch.float32), 1,
                                                      dev),
                               "weight": float(spec["weight"]), "mask": mask,
                               "zscale": None if zs is None else np.asarray(zs, np.float64).ravel()})
        self.blur = None
        if blur is not None:
            k = as_device(blur, dev, torch.float32)
            a, b = int(k.shape[0]), int(k.shape[1])
            self.blur = (KernelSpectrum(k[..., None].contiguous(), transform_size(X + max(a // 2, a - 1 - a // 2)),
                                        transform_size(Y + max(b // 2, b - 1 - b // 2))), (a // 2, b // 2))

    def frame(self, temp, base, z, *, scale=1.0, sf=2.0):
        """The optical frame (X, Y) device tensor for focal slab planes
        [z, z + depth): movie.py:650-679 before the row motion."""
        import torch
        t = as_device(temp, self.device, torch.float32).contiguous()
        b = as_device(base, self.device, torch.float32).contiguous()
        X, Y, nz = self.shape
        if tuple(t.shape) != self.shape or tuple(b.shape) != self.shape:
            raise ValueError(f"frame volumes must have shape {self.shape}")
        z = int(z)
        if z < 0 or z + self.depth > nz:
            raise ValueError("Motion places focal slab outside volume")
        out = torch.empty((X, Y), dtype=torch.float32, device=self.device)
        a, bb = self.psf_xy
        self.freq.kernel.convolve(t[:, :, z:z + self.depth], zrule=_lib.MM_SCAN_SUM_Z, out=out, crop=(a // 2, bb // 2),
                                  out_shape=(X, Y), out_planes=1, group=self.scan_avg, alpha=scale / (2 * sf * sf),
                                  add=b[:, :, z:z + self.depth])
        if self.blur is not None:
            spec, crop = self.blur
            spec.convolve(out[..., None], zrule=_lib.MM_SCAN_EACH_Z, out=out, crop=crop, out_shape=(X, Y),
                          out_planes=1, accumulate=True)
        for j, spec in enumerate(self.tails):
            idx = np.arange(z) if j == 0 else np.arange(z + self.depth, nz)
            zs = spec["zscale"]
            if len(idx) == 0:
                idx, zs = np.arange(nz), None
            scl = zs[:len(idx)] if zs is not None and zs.size >= len(idx) else np.ones(len(idx))
            image = torch.empty((X, Y), dtype=torch.float32, device=self.device)
            ptrs = (_lib.c_void_p * 2)(t.data_ptr(), b.data_ptr())
            s = t.stride()
            # both tables stay referenced until the launch is queued: a table
            # freed early would hand its block to the next upload, whose copy
            # (queued before the launch) would overwrite it
            idx_d = _lib.upload(idx.astype(np.int32), self.device)
            scl_d = _lib.upload(scl.astype(np.float64), self.device)
            _lib.call("mm_scan_background", 0, ptrs, 2, s[0], s[1], s[2], X, Y, nz, _lib.ptr(idx_d), _lib.ptr(scl_d),
                      len(idx), spec["weight"], _lib.ptr(spec["mask"]), _lib.ptr(image), _lib.stream_of(self.device))
            k = spec["kernel"]
            k.kernel.convolve(image[..., None], zrule=_lib.MM_SCAN_EACH_Z, out=out, crop=k.background_crop,
                              out_shape=(X, Y), out_planes=1, accumulate=True, alpha=scale / (sf * sf))
        return out
