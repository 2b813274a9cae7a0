"""Host side of the plane-convolution engine (``csrc/scan.cu``) shared by
``maomi_b200.scanning`` (zstack) and ``maomi_b200.movie`` (single_scan,
blurred_background, conv2_same, psf_fft).

Every operator here is a linear 2-D convolution of real planes with real
kernel planes, evaluated through zero-padded DFTs of power-of-two sizes and
cropped to the window the reference keeps.  The transform size of an axis
only has to keep that window alias free: for a source of extent ``e``, a
kernel of extent ``k`` and a first kept index ``c`` the linear convolution
ends at ``e + k - 1``, so ``f >= max(c + out, e + k - 1 - c)``.
"""

import ctypes

import numpy as np

from . import _lib

MIN_SIZE, MAX_SIZE = 64, 1024
# transform sizes of one axis: 384 = 48 x 8 and 768 = 48 x 16 lines serve
# FP32 planes (a float64 spectrum asked for them runs at 512 / 1024, see
# KernelSpectrum)
SIZES = (64, 128, 256, 384, 512, 768, 1024)


def transform_size(need):
    """Smallest supported transform size >= ``need``."""
    for n in SIZES:
        if n >= need:
            return n
    raise ValueError(f"plane convolution needs a transform of {need} samples; this build supports up to "
                     f"{MAX_SIZE} (volumes up to about {MAX_SIZE} pixels across with small kernels)")


def real_dtype(t):
    """float32 and float64 planes are convolved in their own precision."""
    import torch
    if t.dtype == torch.float64:
        return 1
    if t.dtype == torch.float32:
        return 0
    raise ValueError(f"plane convolution supports float32 and float64 data, got {t.dtype}")


def planes_record(t, *, group=1, masks=(None, None), add=None):
    """ScanPlanes of a 3-D device tensor (any strides), optional XY masks and
    an optional second tensor of the same shape and strides added to it."""
    s = t.stride()
    m0, m1 = masks
    if add is not None and (tuple(add.shape) != tuple(t.shape) or add.stride() != t.stride()
                            or add.dtype != t.dtype):
        raise ValueError("the added volume must share the source's shape, strides and type")
    return _lib.ScanPlanes(t.data_ptr(), s[0], s[1], s[2], t.shape[0], t.shape[1], t.shape[2], int(group),
                           None if m0 is None else m0.data_ptr(), None if m1 is None else m1.data_ptr(),
                           None if add is None else add.data_ptr())


class KernelSpectrum:
    """Device half spectra of (grouped) kernel planes at one transform size.

    ``fx``, ``fy``: transform sizes; ``kx``, ``ky``: kernel plane extents;
    ``planes``: kernel transform planes (after grouping); ``fp64``.  A
    float64 kernel asked for a 384- or 768-point axis gets 512 or 1024 (the
    48-point line transform is FP32 only); any size at least the one asked for
    is alias-free.
    Every convolution and spectrum buffer takes its sizes from ``desc``."""

    def __init__(self, kernel, fx, fy, *, group=1):
        import torch
        self.device = kernel.device
        self.fp64 = real_dtype(kernel)
        self.dtype = kernel.dtype
        self.fx, self.fy = int(fx), int(fy)
        if self.fp64:
            self.fx, self.fy = ({384: 512, 768: 1024}.get(f, f) for f in (self.fx, self.fy))
        self.kx, self.ky = int(kernel.shape[0]), int(kernel.shape[1])
        self.group = int(group)
        self.planes = -(-int(kernel.shape[2]) // self.group)
        self.desc = _lib.ScanDesc(self.fp64, self.fx, self.fy, self.kx, self.ky, self.planes)
        lib = _lib.load()
        nbytes = lib.mm_scan_spectrum_bytes(ctypes.byref(self.desc))
        if nbytes == 0:
            _lib.check(_lib.MM_ERR_UNSUPPORTED, _lib.last_error() or "scan descriptor rejected")
        self.data = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        work = workspace(self.desc, self.planes, self.device)
        rec = planes_record(kernel, group=self.group)
        _lib.check(lib.mm_scan_kernel_spectrum(ctypes.byref(self.desc), ctypes.byref(rec), _lib.ptr(self.data),
                                               _lib.ptr(work), work.numel(), _lib.stream_of(self.device)),
                   "kernel spectrum")
        self._keep = kernel  # the kernel stays alive until the stream has read it

    def convolve(self, src, *, zrule, out, crop, out_shape, out_planes, zoff=0, group=1, masks=(None, None),
                 wrap=None, accumulate=False, alpha=1.0, src_spectra=None, out_spectra=None, out_weight=None,
                 add=None):
        """One engine pass of ``src`` (3-D device tensor) into ``out``.

        ``src_spectra``: the source's packed spectra (``forward_spectra``),
        reused instead of transforming ``src`` again; ``out_spectra``: store
        (or, with ``accumulate``, add) the packed output spectra there and
        skip the inverse; ``out_weight``: (out_x, out_y) weights of the kept
        window."""
        lib = _lib.load()
        if src.dtype != self.dtype or (out is not None and out.dtype != self.dtype):
            raise ValueError("source, kernel and output must share one floating type")
        rec = planes_record(src, group=group, masks=masks, add=add)
        nin = -(-int(src.shape[2]) // int(group))
        conv = conv_record(src, rec, wrap, zrule, zoff, out_planes, crop, out_shape, out, accumulate, alpha)
        conv.src_spectra = None if src_spectra is None else src_spectra.data_ptr()
        conv.out_spectra = None if out_spectra is None else out_spectra.data_ptr()
        conv.out_weight = None if out_weight is None else out_weight.data_ptr()
        planes = 0 if (src_spectra is not None and out_spectra is not None) else (
            int(out_planes) if src_spectra is not None else max(nin, int(out_planes)))
        work = workspace(self.desc, planes, self.device) if planes else None
        _lib.check(lib.mm_scan_convolve(ctypes.byref(self.desc), ctypes.byref(conv), _lib.ptr(self.data),
                                        _lib.ptr(work), 0 if work is None else work.numel(),
                                        _lib.stream_of(self.device)), "plane convolution")
        return out


def conv_record(src, rec, wrap, zrule, zoff, out_planes, crop, out_shape, out, accumulate, alpha):
    if wrap is None:
        wrap_flag, wx0, wy0, ext_x, ext_y = 0, 0, 0, int(src.shape[0]), int(src.shape[1])
    else:
        wrap_flag, (wx0, wy0), (ext_x, ext_y) = 1, wrap[0], wrap[1]
    if out is None:
        ptr, o = None, (0, 0, 0)
    else:
        ptr, o = out.data_ptr(), (out.stride() if out.dim() == 3 else (out.stride(0), out.stride(1), 0))
    return _lib.ScanConv(rec, wrap_flag, int(wx0), int(wy0), int(ext_x), int(ext_y), int(zrule), int(zoff),
                         int(out_planes), int(crop[0]), int(crop[1]), int(out_shape[0]), int(out_shape[1]), ptr,
                         o[0], o[1], o[2], int(bool(accumulate)), float(alpha))


def spectra_buffer(desc, planes, device):
    """Packed spectra of ``planes`` transform planes (complex pairs, fx x fy)."""
    return workspace(desc, planes, device)


def forward_spectra(desc, src, *, masks=(None, None), group=1):
    """Packed spectra of the planes of ``src`` at the transform sizes of ``desc``."""
    planes = -(-int(src.shape[2]) // int(group))
    buf = spectra_buffer(desc, planes, src.device)
    rec = planes_record(src, group=group, masks=masks)
    conv = conv_record(src, rec, None, 0, 0, planes, (0, 0), (1, 1), None, False, 1.0)
    _lib.check(_lib.load().mm_scan_forward(ctypes.byref(desc), ctypes.byref(conv), _lib.ptr(buf),
                                           _lib.stream_of(src.device)), "plane transform")
    return buf


def inverse_spectra(desc, spectra, out, *, crop, out_shape, out_planes, accumulate=False, alpha=1.0,
                    out_weight=None):
    """Inverse passes of packed spectra (overwritten) into ``out``."""
    dummy = out if out.dim() == 3 else out[..., None]
    rec = planes_record(dummy)
    conv = conv_record(dummy, rec, None, 0, 0, out_planes, crop, out_shape, out, accumulate, alpha)
    conv.out_weight = None if out_weight is None else out_weight.data_ptr()
    _lib.check(_lib.load().mm_scan_inverse(ctypes.byref(desc), ctypes.byref(conv), _lib.ptr(spectra),
                                           _lib.stream_of(out.device)), "inverse plane transform")
    return out


def workspace(desc, planes, device):
    import torch
    nbytes = _lib.load().mm_scan_workspace_size(ctypes.byref(desc), int(planes))
    if nbytes == 0:
        _lib.check(_lib.MM_ERR_UNSUPPORTED, _lib.last_error() or "scan descriptor rejected")
    return torch.empty(nbytes, dtype=torch.uint8, device=device)


def as_device(a, device, dtype=None):
    """Host or device array -> device tensor (no copy when already there)."""
    import torch
    if isinstance(a, torch.Tensor):
        t = a.to(device=device, dtype=dtype if dtype is not None else a.dtype)
    else:
        arr = np.asarray(a)
        t = _lib.upload(arr, device) if arr.size else torch.as_tensor(arr, device=device)
        if dtype is not None:
            t = t.to(dtype)
    return t


def mask_tensor(m, shape, device, dtype):
    if m is None:
        return None
    t = as_device(m, device, dtype)
    if tuple(t.shape) != tuple(shape):
        raise ValueError("Mask must match volume XY")
    return t.contiguous()
