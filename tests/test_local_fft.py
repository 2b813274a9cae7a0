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
