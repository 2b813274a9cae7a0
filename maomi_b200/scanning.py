"""``zstack``: the static scan operator on the GPU.

Drop-in for maomi/scanning.py:8-53.  Arrays are X, Y, Z; the result is a
device tensor of the volume's floating type, like the reference's.

``matlab_convn`` is MATLAB ``convn(..., 'same')``: zero extension on every
axis, convolution on every axis, crop from ``floor(k/2)``.
``legacy_circular`` is periodic in XY, zero extended in Z and a correlation
along Z, cropped from ``k - 1 - k//2`` (the July Python scan).  Both run
through the plane-convolution engine (``csrc/scan.cu``): 2-D DFTs of every
(masked) volume plane, the per-bin convolution (or correlation) along Z
against the kernel spectra, inverse DFTs of the kept rows and columns only.
The periodic XY case reads the volume with a wrap-around so that a linear
convolution of the periodic extension gives the circular one.
"""

from . import _lib
from ._scan import KernelSpectrum, as_device, mask_tensor, real_dtype, transform_size


def zstack(volume, psf, *, device="cuda", mode="matlab_convn", mask=None, collection_mask=None, rana=None):
    """FFT implementation of MATLAB convn(...,'same') or the July Python scan
    (maomi/scanning.py:8-53).  Optional masks modulate the source volume
    before convolution; device transfers happen inside this call."""
    import torch
    _lib.require_cuda(device)
    v = as_device(volume, device)
    if not v.is_floating_point():
        v = v.float()
    p = as_device(psf, device, v.dtype)
    if v.ndim != 3 or p.ndim != 3:
        raise ValueError("Expected X,Y,Z arrays")
    real_dtype(v)
    m0 = mask_tensor(mask, v.shape[:2], device, v.dtype)
    m1 = mask_tensor(collection_mask, v.shape[:2], device, v.dtype)
    if rana is not None and rana is not False:
        if mode != "matlab_convn":
            raise ValueError("RANA uses zero-extended local optics; legacy_circular is a different boundary model")
        src = v
        for m in (m0, m1):
            if m is not None:
                src = src * m[..., None]
        return torch.as_tensor(rana.static(src), device=device, dtype=v.dtype)
    X, Y, Z = (int(s) for s in v.shape)
    a, b, k = (int(s) for s in p.shape)
    if mode == "matlab_convn":
        cx, cy = a // 2, b // 2
        fx, fy = transform_size(X + cx), transform_size(Y + cy)
        spec = KernelSpectrum(p.contiguous(), fx, fy)
        out = torch.empty((X, Y, Z), dtype=v.dtype, device=device)
        return spec.convolve(v, zrule=_lib.MM_SCAN_CONV_Z, zoff=k // 2, out=out, crop=(cx, cy), out_shape=(X, Y),
                             out_planes=Z, masks=(m0, m1))
    if mode == "legacy_circular":
        if a > X or b > Y:
            raise ValueError("Legacy operator requires PSF XY <= image XY")
        # circular XY convolution with the kernel rolled by (-a//2, -b//2):
        # the linear convolution of the periodic extension read from row
        # (i + wx0) mod X, kept from a - 1 (see csrc/scan.cu)
        wx0 = (-((-a) // 2) - a + 1) % X
        wy0 = (-((-b) // 2) - b + 1) % Y
        fx, fy = transform_size(X + a - 1), transform_size(Y + b - 1)
        spec = KernelSpectrum(p.contiguous(), fx, fy)
        out = torch.empty((X, Y, Z), dtype=v.dtype, device=device)
        return spec.convolve(v, zrule=_lib.MM_SCAN_CORR_Z, zoff=k // 2, out=out, crop=(a - 1, b - 1),
                             out_shape=(X, Y), out_planes=Z, masks=(m0, m1),
                             wrap=((wx0, wy0), (X + a - 1, Y + b - 1)))
    raise ValueError(f"Unknown operator: {mode}")
