"""Local-PSF (RANA) renderer: oracle pins (CPU) and the CUDA operator (GPU).

Tolerances follow the reference's own tests: the operator is float64 on both
of its backends and its CUDA-vs-CPU test allows 2e-13 absolute
(tests/test_rana_addon.py:238-247); relative 1e-11 here covers FFT vs direct
summation order on these magnitudes."""

import numpy as np
import pytest

from conftest import golden, rel_l2
from oracle import local_fft as L

RTOL = 1e-11


def test_axis_weights_pin():
    d = golden("local_fft")
    np.testing.assert_allclose(L.axis_weights(d["c_nodes"], d["c_pos"]), d["c_weights"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("op", ["excitation", "detection"])
def test_oracle_small_field(op):
    d = golden("local_fft")
    vol, k = d["a_volume"], d["a_kernels"]
    args = ([k], [0, 12], [0, 14], (1., 1., 1.))
    assert rel_l2(L.static(*args, vol, operator=op), d[f"a_{op}_static"]) < RTOL
    assert rel_l2(L.static(*args, vol, operator=op, native=True), d[f"a_{op}_native_static"]) < RTOL
    for avg in (1, 2):
        got = L.scan_slab(*args, vol[..., :3], operator=op, scan_avg=avg)
        assert rel_l2(got, d[f"a_{op}_slab{avg}"]) < RTOL


@pytest.mark.parametrize("op", ["excitation", "detection"])
def test_oracle_depth_bank(op):
    d = golden("local_fft")
    kern = [d["b_kernels"][0], d["b_kernels"][1]]
    args = (kern, d["b_x"], d["b_y"], (1., 1., 1.))
    assert rel_l2(L.static(*args, d["b_volume"], operator=op, depths=d["b_depths"]), d[f"b_{op}_static"]) < RTOL
    got = L.scan_slab(*args, d["b_volume"][..., 2:7], operator=op, depths=d["b_depths"], z_start=2)
    assert rel_l2(got, d[f"b_{op}_slab"]) < RTOL


@pytest.mark.gpu
@pytest.mark.parametrize("op", ["excitation", "detection"])
def test_cuda_operator_matches_reference(op):
    from maomi_b200.rana import DepthPSFBank, FullFieldPSF, RanaOperator
    d = golden("local_fft")
    vol, k = d["a_volume"], d["a_kernels"]
    f = FullFieldPSF(k, [0, 12], [0, 14], (1., 1., 1.), 920., op)
    R = RanaOperator(f, device="cuda")
    assert rel_l2(R.static(vol), d[f"a_{op}_static"]) < RTOL
    assert rel_l2(RanaOperator(f, native=True, device="cuda").static(vol), d[f"a_{op}_native_static"]) < RTOL
    for avg in (1, 2):
        assert rel_l2(R.scan_slab(vol[..., :3], scan_avg=avg), d[f"a_{op}_slab{avg}"]) < RTOL
    fields = tuple(FullFieldPSF(d["b_kernels"][i], d["b_x"], d["b_y"], (1., 1., 1.), 920., op) for i in range(2))
    R = RanaOperator(DepthPSFBank(d["b_depths"], fields), device="cuda")
    assert rel_l2(R.static(d["b_volume"]), d[f"b_{op}_static"]) < RTOL
    assert rel_l2(R.scan_slab(d["b_volume"][..., 2:7], z_start=2), d[f"b_{op}_slab"]) < RTOL


@pytest.mark.gpu
def test_cuda_operator_large_kernels_vs_oracle():
    """33x33x9 kernels (the benchmark bank's shape) on a 64x64x16 volume, 4x4
    nodes, two depths: the CUDA direct sum against the oracle's FFT path."""
    from maomi_b200 import synthetic
    from maomi_b200.rana import DepthPSFBank, FullFieldPSF, RanaOperator
    vol = synthetic.somata_volume((64, 64, 16), count=30, seed=2)
    kern = synthetic.psf_bank_kernels(nodes=(4, 4), kernel=(33, 33, 9), depths=2, seed=4).astype(np.float64)
    xs = ys = np.linspace(0, 64, 4)
    depths = np.array([0.0, 16.0])
    for op in ("excitation", "detection"):
        fields = tuple(FullFieldPSF(kern[i], xs, ys, (1., 1., 1.), 920., op) for i in range(2))
        got = RanaOperator(DepthPSFBank(depths, fields), device="cuda").static(vol)
        ref = L.static([kern[0], kern[1]], xs, ys, (1., 1., 1.), vol, operator=op, depths=depths)
        assert rel_l2(got, ref) < RTOL, op


@pytest.mark.gpu
@pytest.mark.parametrize("xs,ys", [(np.array([0., 1.5, 2.0, 9.0, 40.0]), np.linspace(0, 36, 7)),
                                   (np.linspace(0, 40, 3), np.array([0., 3., 4., 30., 36.]))])
def test_cuda_operator_uneven_and_dense_nodes(xs, ys):
    """Irregular node grids: intervals from 0.5 to 31 pixels (tiles split to
    <= 18 pixels, one-pixel tiles, single-node pixels), 9x7x5 kernels with
    even and odd extents, every operator mode, static and scan slabs."""
    from maomi_b200.rana import DepthPSFBank, FullFieldPSF, RanaOperator
    rng = np.random.default_rng(17)
    vol = rng.uniform(0, 1, (40, 36, 7))
    kern = rng.uniform(0.05, 1, (2, len(xs), len(ys), 9, 6, 5))
    depths = np.array([0.0, 7.0])
    for op in ("excitation", "detection"):
        fields = tuple(FullFieldPSF(kern[i], xs, ys, (1., 1., 1.), 920., op) for i in range(2))
        for native in (False, True):
            R = RanaOperator(DepthPSFBank(depths, fields), native=native, device="cuda")
            ref = L.static([kern[0], kern[1]], xs, ys, (1., 1., 1.), vol, operator=op, depths=depths, native=native)
            assert rel_l2(R.static(vol), ref) < RTOL, (op, native)
            for avg in (1, 2):
                got = R.scan_slab(vol[..., 1:6], z_start=1, scan_avg=avg)
                ref = L.scan_slab([kern[0], kern[1]], xs, ys, (1., 1., 1.), vol[..., 1:6], operator=op,
                                  depths=depths, z_start=1, native=native, scan_avg=avg)
                assert rel_l2(got, ref) < RTOL, (op, native, avg)


@pytest.mark.gpu
@pytest.mark.parametrize("plane", [False, True])
@pytest.mark.parametrize("detection,correlate", [(False, True), (False, False), (True, False)])
def test_local_fft_plan_drop_in(plane, detection, correlate):
    """LocalFFTPlan called directly (the reference's plan API) against the
    oracle's restatement of the same plan."""
    from maomi_b200.rana import LocalFFTPlan
    from maomi_b200.rana.operator import _axis_weights
    rng = np.random.default_rng(5)
    shape = (30, 26, 5)
    kern = rng.uniform(0.1, 1, (3, 4, 7, 5, 5))
    w = (_axis_weights(np.linspace(0, 30, 3), np.arange(30) + .5),
         _axis_weights(np.linspace(0, 26, 4), np.arange(26) + .5))
    src = rng.uniform(0, 1, shape)
    plan = LocalFFTPlan(shape, kern, w, plane=plane, detection=detection, correlate=correlate, device="cuda")
    got = plan(src).cpu().numpy()
    again = plan(src).cpu().numpy()
    ref = L.local_fft(shape, kern, w, src, plane=plane, detection=detection, correlate=correlate)
    assert got.shape == ref.shape
    assert rel_l2(got, ref) < RTOL
    np.testing.assert_array_equal(again, got)
    assert plan.stats == {"kernel_fft_builds": 0, "cache_hits": 1} and plan.cache_bytes == 0
