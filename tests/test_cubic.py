"""Global cubic-RBF renderers: oracle pins (CPU) and the CUDA engine (GPU).

Fixtures (``tests/golden/cubic.npz``) are the reference's own
``CubicFullFieldRenderer`` (maomi/rana/fields.py:113-276) and
``DepthFullFieldRenderer`` (maomi/rana/depth.py:72-104) outputs.  The
renderer is float64 on every backend; the reference checks its CUDA path
against direct sums at 1e-12 absolute (tests/test_enhanced.py:122-127).
Here: 1e-11 relative L2 for the small fields, 1e-9 for the 16 x 16-node
field, whose interpolation system is solved by a different LU.
"""

import numpy as np
import pytest

from conftest import golden, rel_l2
from oracle import cubic as C


def _case(d, i):
    k, a, op = d[f"k{i}_kernels"], d[f"k{i}_density"], str(d[f"k{i}_op"])
    org = tuple(d[f"k{i}_origin"]) if f"k{i}_origin" in d.files else (0.0, 0.0)
    return k, d[f"k{i}_x"], d[f"k{i}_y"], a, op, org


def _tol(k):
    return 1e-9 if k.shape[0] * k.shape[1] > 9 else 1e-11


def test_oracle_cubic_pin():
    d = golden("cubic")
    for i in range(int(d["cases"])):
        k, x, y, a, op, org = _case(d, i)
        got = np.maximum(C.cubic_render(k, x, y, (1.0,) * a.ndim, op, a, org), 0)
        assert rel_l2(got, d[f"k{i}_image"]) < 1e-12, i


def test_oracle_depth_pin():
    d = golden("cubic")
    for name in ("uniform", "varying"):
        for op in ("detection", "excitation"):
            got = C.depth_render(d["d_depths"], list(d[f"d_{name}_{op}_kernels"]), d["d_x"], d["d_y"],
                                 (1.0, 1.0, 1.0), op, d[f"d_{name}_{op}_density"])
            assert rel_l2(got, d[f"d_{name}_{op}_image"]) < 1e-12, (name, op)


@pytest.mark.gpu
def test_cubic_renderer_gpu_matches_reference():
    from maomi_b200.rana import CubicFullFieldRenderer, FullFieldPSF
    d = golden("cubic")
    for i in range(int(d["cases"])):
        k, x, y, a, op, org = _case(d, i)
        f = FullFieldPSF(k, x, y, (1.0,) * a.ndim, 920.0, op)
        r = CubicFullFieldRenderer(f, a.shape, voxel_size_um=(1,) * a.ndim, origin_um=org)
        got = r(a)
        assert got.shape == a.shape and got.dtype == np.float64
        assert rel_l2(got, d[f"k{i}_image"]) < _tol(k), (i, rel_l2(got, d[f"k{i}_image"]))
        assert r.validation["checked_xy_positions"] == a.shape[0] * a.shape[1]
        assert not r.validation["shared_psf_fallback"]


@pytest.mark.gpu
def test_cubic_local_psfs_reproduce_the_nodes():
    from maomi_b200.rana import CubicFullFieldRenderer, FullFieldPSF
    d = golden("cubic")
    k, x, y, a, op, _ = _case(d, 8)  # the non-affine knot
    f = FullFieldPSF(k, x, y, (1, 1), 920, op)
    r = CubicFullFieldRenderer(f, a.shape, voxel_size_um=(1, 1))
    nodes = np.stack(np.meshgrid(x, y, indexing="ij"), -1).reshape(-1, 2)
    np.testing.assert_allclose(r.local_psfs(nodes), k.reshape(-1, *k.shape[2:]), atol=1e-12)
    assert r.local_psfs(np.empty((0, 2))).shape == (0,) + k.shape[2:]
    with pytest.raises(ValueError, match="extrapolation"):
        r.local_psfs([[5.01, 2]])


@pytest.mark.gpu
def test_depth_renderer_gpu_matches_reference():
    from maomi_b200.rana import DepthFullFieldRenderer, DepthPSFBank, FullFieldPSF
    d = golden("cubic")
    for name in ("uniform", "varying"):
        for op in ("detection", "excitation"):
            kern = d[f"d_{name}_{op}_kernels"]
            bank = DepthPSFBank(d["d_depths"], tuple(FullFieldPSF(kk, d["d_x"], d["d_y"], (1., 1., 1.), 920., op)
                                                     for kk in kern))
            a = d[f"d_{name}_{op}_density"]
            r = DepthFullFieldRenderer(bank, a.shape, voxel_size_um=(1., 1., 1.))
            assert rel_l2(r(a), d[f"d_{name}_{op}_image"]) < 1e-11, (name, op)
            assert all(v["exact_uniform_xy"] == (name == "uniform") for v in r.validation["fields"])


@pytest.mark.gpu
def test_cubic_renderer_contracts():
    from maomi_b200.rana import CubicFullFieldRenderer, FullFieldPSF
    d = golden("cubic")
    k, x, y, a, op, _ = _case(d, 1)
    f = FullFieldPSF(k, x, y, (1, 1), 920, "excitation")
    for shape, pitch, origin in [((6, 4), (1, 1), (0, 0)), ((5, 4), (1, 1), (-.1, 0)), ((5, 4), (.5, 1), (0, 0))]:
        with pytest.raises(ValueError):
            CubicFullFieldRenderer(f, shape, voxel_size_um=pitch, origin_um=origin)
    with pytest.raises(TypeError):
        CubicFullFieldRenderer(np.ones((3, 3)), (5, 4), voxel_size_um=(1, 1))
    with pytest.raises(ValueError, match="CUDA"):
        CubicFullFieldRenderer(f, (5, 4), voxel_size_um=(1, 1), device="cpu")
    over = np.ones((3, 3, 2, 2)) * .01
    over[0, 0] = 100
    with pytest.raises(ValueError, match="nonphysical"):
        CubicFullFieldRenderer(FullFieldPSF(over, [0, 4, 8], [0, 4, 8], (1, 1), 920, "detection"), (8, 8),
                               voxel_size_um=(1, 1))
    r = CubicFullFieldRenderer(f, (5, 4), voxel_size_um=(1, 1))
    for bad in (-np.ones((5, 4)), np.ones((5, 3)), np.full((5, 4), np.nan)):
        with pytest.raises(ValueError):
            r(bad)
    with pytest.raises(ValueError, match="real"):
        r(np.ones((5, 4), complex))
    shifted = FullFieldPSF(k, x + 11, y - 3, (1, 1), 920, "excitation")
    np.testing.assert_allclose(CubicFullFieldRenderer(shifted, (5, 4), voxel_size_um=(1, 1), origin_um=(11, -3))(
        np.ones((5, 4))), r(np.ones((5, 4))), atol=1e-12)
