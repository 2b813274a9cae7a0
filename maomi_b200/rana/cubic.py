"""Global cubic-RBF full-field renderer on the GPU.

Drop-in for ``CubicFullFieldRenderer`` (maomi/rana/fields.py:113-276): the
complete local effective kernels of a ``FullFieldPSF`` are interpolated over
XY with an affine-augmented r^3 radial basis, and the image is the exact
basis decomposition

    excitation:  image(x) = sum_i w_i(x) * (density corr K_i)(x)
    detection:   image    = sum_i (density * w_i) conv K_i

with w_i the basis functions at the pixel centres (|p - node_i|^3, 1, p_x,
p_y) and K_i the basis coefficients (kernel-shaped).  Each term is one pass
of the plane-convolution engine (``csrc/scan.cu``, FP64): for excitation the
density is transformed once and every term reuses its spectra, applying its
weight plane in the inverse pass; for detection the weighted density of each
term is transformed and the terms are summed in the frequency domain, with
one inverse at the end.  Bitwise-uniform fields reduce exactly to the
constant basis term (one pass), as in the reference.

The interpolation system (nodes + 3 affine terms, FP64) is solved on the GPU
and the interpolated kernel at every pixel centre is checked before use, with
the reference's acceptance rules and messages.
"""

import numpy as np

from .. import _lib
from .._scan import KernelSpectrum, forward_spectra, inverse_spectra, spectra_buffer, transform_size
from .fields import FullFieldPSF


def _cuda_device(device):
    if not str(device).startswith("cuda"):
        raise ValueError("maomi_b200 renders on CUDA only (device='cuda[:index]'); the reference renders on CPU")
    _lib.require_cuda(device)
    return device


def _dist(a, b):
    """Euclidean distances formed from coordinate differences (no Gram-matrix
    shortcut, which cancels badly near the nodes)."""
    import torch
    return torch.cdist(a, b, compute_mode="donot_use_mm_for_euclid_dist")


class CubicFullFieldRenderer:
    """Affine-augmented r^3 interpolation of complete local effective kernels."""

    def __init__(self, psf_field, shape, *, voxel_size_um, origin_um=(0., 0.), device="cuda"):
        import torch
        if not isinstance(psf_field, FullFieldPSF):
            raise TypeError("RANA Mode requires FullFieldPSF; a shared PSF is not accepted")
        dims = psf_field.kernels.ndim - 2
        if len(shape) != dims or any(isinstance(n, bool) or int(n) != n or n < 1 for n in shape):
            raise ValueError("Image shape must contain positive integers matching kernel dimensions")
        self.shape = tuple(int(n) for n in shape)
        pitch = np.asarray(voxel_size_um, dtype=float)
        origin = np.asarray(origin_um, dtype=float)
        if (pitch.shape != (dims,) or not np.isfinite(pitch).all() or (pitch <= 0).any()
                or not np.allclose(pitch, psf_field.voxel_size_um, rtol=1e-12, atol=0)):
            raise ValueError("Image and kernel voxel pitches must match; resample explicitly")
        if origin.shape != (2,) or not np.isfinite(origin).all():
            raise ValueError("origin_um must contain two finite XY lower-edge coordinates")
        lower = np.array([psf_field.x_um[0], psf_field.y_um[0]])
        upper = np.array([psf_field.x_um[-1], psf_field.y_um[-1]])
        end = origin + np.array(self.shape[:2]) * pitch[:2]
        if (origin < lower - 1e-12).any() or (end > upper + 1e-12).any():
            raise ValueError("PSF field must cover the entire FOV including edges; extrapolation is forbidden")
        self.device = _cuda_device(device)
        self.field = psf_field
        self._lower, self._span = lower, upper - lower
        nodes = (np.stack(np.meshgrid(psf_field.x_um, psf_field.y_um, indexing="ij"), -1).reshape(-1, 2)
                 - lower) / self._span
        self._nodes = nodes
        n = len(nodes)
        self.kernel_shape = tuple(int(k) for k in psf_field.kernels.shape[2:])
        kprod = int(np.prod(self.kernel_shape))
        dev = self.device
        f64 = torch.float64
        nodes_d = torch.as_tensor(nodes, dtype=f64, device=dev)
        self._nodes_d = nodes_d
        kern = torch.as_tensor(np.array(psf_field.kernels, np.float64), device=dev).reshape(n, kprod)
        # exact input symmetry: bitwise identical kernels use the constant basis only
        self._uniform_xy = bool(np.array_equal(psf_field.kernels, np.broadcast_to(psf_field.kernels[0, 0],
                                                                                  psf_field.kernels.shape)))
        coeff = torch.zeros((n + 3, kprod), dtype=f64, device=dev)
        if self._uniform_xy:
            coeff[n] = kern[0]
        else:
            system = torch.zeros((n + 3, n + 3), dtype=f64, device=dev)
            system[:n, :n] = _dist(nodes_d, nodes_d) ** 3
            poly = torch.cat([torch.ones((n, 1), dtype=f64, device=dev), nodes_d], 1)
            system[:n, n:] = poly
            system[n:, :n] = poly.T
            rhs = torch.cat([kern, torch.zeros((3, kprod), dtype=f64, device=dev)], 0)
            coeff = torch.linalg.solve(system, rhs)
        if not bool(torch.isfinite(coeff).all()):
            raise ValueError("Ill-conditioned cubic PSF field")
        self._coeff = coeff
        axes = [origin[i] + (np.arange(self.shape[i]) + .5) * pitch[i] for i in range(2)]
        pixels = (np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 2) - lower) / self._span
        self._pixels_d = torch.as_tensor(pixels, dtype=f64, device=dev)
        self._chunk = max(1, min(1024, 2_000_000 // (coeff.shape[0] + coeff.shape[1])))
        worst, gain = np.inf, np.inf
        if self._uniform_xy:
            blocks = [kern[:1]]
        else:
            blocks = (self._basis(self._pixels_d[s:s + self._chunk]) @ coeff
                      for s in range(0, len(pixels), self._chunk))
        for local in blocks:
            self._check_local(local)
            worst = min(worst, float(local.min()))
            gain = min(gain, float(local.sum(1).min()))
        self.validation = {"checked_xy_positions": len(pixels), "minimum_interpolated_value": worst,
                           "minimum_local_gain": gain, "exact_uniform_xy": self._uniform_xy,
                           "shared_psf_fallback": False}
        detection = psf_field.operator == "detection"
        self._centers = [k // 2 if detection else k - 1 - k // 2 for k in self.kernel_shape]
        self._crop = tuple(slice(c, c + s) for c, s in zip(self._centers, self.shape))
        X, Y = self.shape[:2]
        kx, ky = self.kernel_shape[:2]
        cx, cy = self._centers[:2]
        self._fx = transform_size(max(cx + X, X + kx - 1 - cx))
        self._fy = transform_size(max(cy + Y, Y + ky - 1 - cy))
        self._terms = (coeff.abs().amax(1) > 0).nonzero().flatten().tolist()

    def _basis(self, q):
        import torch
        return torch.cat([_dist(q, self._nodes_d) ** 3, torch.ones((len(q), 1), dtype=q.dtype, device=q.device), q], 1)

    @staticmethod
    def _check_local(local):
        scale = local.abs().amax(1)
        if (not bool(local.isfinite().all()) or bool((local.sum(1) <= 0).any())
                or bool((local.amin(1) < -1e-10 * scale).any())):
            raise ValueError("Cubic interpolation produced nonphysical local PSFs; "
                             "refine or revise the supplied field. No shared-PSF fallback is allowed")

    def local_psfs(self, xy_um):
        """Interpolated effective kernels at covered physical positions (host array)."""
        import torch
        xy = np.asarray(xy_um, dtype=float)
        if xy.ndim != 2 or xy.shape[1] != 2 or not np.isfinite(xy).all():
            raise ValueError("xy_um must be a finite (N, 2) array")
        q = (xy - self._lower) / self._span
        if (q < 0).any() or (q > 1).any():
            raise ValueError("PSF extrapolation is forbidden")
        if len(q) == 0:
            return np.empty((0, *self.kernel_shape))
        qd = torch.as_tensor(q, dtype=torch.float64, device=self.device)
        blocks = []
        for s in range(0, len(q), self._chunk):
            local = self._basis(qd[s:s + self._chunk]) @ self._coeff
            self._check_local(local)
            blocks.append(local.reshape(-1, *self.kernel_shape))
        return torch.cat(blocks).cpu().numpy()

    def _weight(self, index):
        """Basis function ``index`` at the pixel centres, an (X, Y) device plane."""
        import torch
        n = len(self._nodes)
        p = self._pixels_d
        if index < n:
            values = torch.linalg.vector_norm(p - self._nodes_d[index], dim=1) ** 3
        elif index == n:
            values = torch.ones(len(p), dtype=p.dtype, device=p.device)
        else:
            values = p[:, index - n - 1].contiguous()
        return values.reshape(self.shape[0], self.shape[1])

    def __call__(self, density):
        import torch
        if np.iscomplexobj(density) or (isinstance(density, torch.Tensor) and density.is_complex()):
            raise ValueError("Fluorescence density must be real")
        src = (density.to(device=self.device, dtype=torch.float64) if isinstance(density, torch.Tensor)
               else _lib.upload(np.asarray(density, dtype=float), self.device))
        if (tuple(src.shape) != self.shape or not bool(torch.isfinite(src).all())
                or bool((src < 0).any())):
            raise ValueError("Density must be finite, nonnegative and match the prepared shape")
        return self.render_device(src).cpu().numpy()

    def render_device(self, src, *, checks=True):
        """The image of a validated FP64 device density (device tensor)."""
        import torch
        src3 = (src if src.ndim == 3 else src[..., None]).contiguous()
        X, Y, Z = (int(v) for v in src3.shape)
        ks = self.kernel_shape + ((1,) if len(self.kernel_shape) == 2 else ())
        cz = self._centers[2] if len(self._centers) == 3 else 0
        out = torch.zeros((X, Y, Z), dtype=torch.float64, device=self.device)
        excitation = self.field.operator == "excitation"
        acc = None
        src_spec = None
        for j, i in enumerate(self._terms):
            kernel = self._coeff[i].reshape(ks)
            if excitation:
                kernel = torch.flip(kernel, dims=(0, 1, 2))  # correlation
            spec = KernelSpectrum(kernel.contiguous(), self._fx, self._fy)
            common = dict(zrule=_lib.MM_SCAN_CONV_Z, zoff=cz, crop=tuple(self._centers[:2]), out_shape=(X, Y),
                          out_planes=Z)
            weight = self._weight(i)
            if excitation:
                if src_spec is None:
                    src_spec = forward_spectra(spec.desc, src3)
                spec.convolve(src3, out=out, accumulate=True, src_spectra=src_spec, out_weight=weight, **common)
            else:
                if acc is None:
                    acc = spectra_buffer(spec.desc, Z, self.device)
                spec.convolve(src3, out=None, accumulate=j > 0, out_spectra=acc, masks=(weight, None), **common)
        if not excitation and acc is not None:
            inverse_spectra(spec.desc, acc, out, crop=tuple(self._centers[:2]), out_shape=(X, Y), out_planes=Z)
        result = out if src.ndim == 3 else out[..., 0]
        if not checks:
            return result
        if not bool(torch.isfinite(result).all()):
            raise FloatingPointError("Nonfinite full-field image")
        scale = max(float(result.abs().max()), np.finfo(float).tiny)
        if float(result.min()) < -1e-9 * scale:
            raise FloatingPointError("Full-field image has material negative intensity")
        return torch.clamp(result, min=0.0)  # only floating-point cancellation, after the checks
