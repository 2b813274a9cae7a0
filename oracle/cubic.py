"""CPU restatement of MaoMi's global cubic-RBF renderers (TEST INFRASTRUCTURE ONLY).

Restates CubicFullFieldRenderer (maomi/rana/fields.py:113-276) and
DepthFullFieldRenderer (maomi/rana/depth.py:72-104) in float64 NumPy/SciPy:
the affine-augmented r^3 interpolation system over the normalised field
nodes, the exact basis decomposition of the spatially varying operator, and
the linear depth weights.  Inputs are plain arrays (kernels (nx, ny, *k),
node axes, pitch, operator), so the checker does not depend on the product's
classes.
"""

import numpy as np
from scipy import fft
from scipy.linalg import lu_factor, lu_solve
from scipy.spatial.distance import cdist


def cubic_coefficients(kernels, x_um, y_um):
    """(normalised nodes, lower, span, coefficients (n + 3, prod(k))) of
    fields.py:150-170."""
    lower = np.array([x_um[0], y_um[0]], float)
    span = np.array([x_um[-1], y_um[-1]], float) - lower
    nodes = (np.stack(np.meshgrid(x_um, y_um, indexing="ij"), -1).reshape(-1, 2) - lower) / span
    n = len(nodes)
    rhs = np.r_[kernels.reshape(n, -1), np.zeros((3, int(np.prod(kernels.shape[2:]))))]
    if np.array_equal(kernels, np.broadcast_to(kernels[0, 0], kernels.shape)):
        coeff = np.zeros_like(rhs)
        coeff[n] = kernels[0, 0].ravel()
        return nodes, lower, span, coeff
    poly = np.c_[np.ones(n), nodes]
    system = np.block([[cdist(nodes, nodes) ** 3, poly], [poly.T, np.zeros((3, 3))]])
    return nodes, lower, span, lu_solve(lu_factor(system), rhs)


def cubic_render(kernels, x_um, y_um, pitch, operator, density, origin=(0.0, 0.0)):
    """fields.py:237-276: the image of ``density`` through the interpolated
    local kernels (no clamping, for comparison before the final max(., 0))."""
    kernels = np.asarray(kernels, float)
    a = np.asarray(density, float)
    shape, kshape = a.shape, kernels.shape[2:]
    nodes, lower, span, coeff = cubic_coefficients(kernels, x_um, y_um)
    axes = [origin[i] + (np.arange(shape[i]) + .5) * pitch[i] for i in range(2)]
    pixels = (np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 2) - lower) / span
    n = len(nodes)
    fshape = tuple(n_ + k - 1 for n_, k in zip(shape, kshape))
    centers = [k // 2 if operator == "detection" else k - 1 - k // 2 for k in kshape]
    crop = tuple(slice(c, c + s) for c, s in zip(centers, shape))
    tail = (1,) if len(shape) == 3 else ()

    def weight(i):
        if i < n:
            w = np.linalg.norm(pixels - nodes[i], axis=1) ** 3
        elif i == n:
            w = np.ones(len(pixels))
        else:
            w = pixels[:, i - n - 1]
        return w.reshape(*shape[:2], *tail)

    excitation = operator == "excitation"
    spectrum = fft.rfftn(a, s=fshape) if excitation else None
    acc = None
    for i, flat in enumerate(coeff):
        k = flat.reshape(kshape)
        if not np.any(k):
            continue
        if excitation:
            r = fft.irfftn(spectrum * fft.rfftn(np.flip(k), s=fshape), s=fshape)[crop] * weight(i)
        else:
            r = fft.rfftn(a * weight(i), s=fshape) * fft.rfftn(k, s=fshape)
        acc = r if acc is None else acc + r
    return acc if excitation else fft.irfftn(acc, s=fshape)[crop]


def depth_render(depths_um, kernel_sets, x_um, y_um, pitch, operator, density, origin=(0.0, 0.0), z_origin=0.0):
    """depth.py:72-104: linear depth weights over per-depth cubic renders."""
    a = np.asarray(density, float)
    z = z_origin + (np.arange(a.shape[2]) + .5) * pitch[2]
    eye = np.eye(len(depths_um))
    out = np.zeros(a.shape)
    for i, kernels in enumerate(kernel_sets):
        w = np.interp(z, depths_um, eye[i])
        if not np.any(w):
            continue
        if operator == "detection":
            out += np.maximum(cubic_render(kernels, x_um, y_um, pitch, operator, a * w[None, None, :], origin), 0)
        else:
            out += np.maximum(cubic_render(kernels, x_um, y_um, pitch, operator, a, origin), 0) * w[None, None, :]
    return out
