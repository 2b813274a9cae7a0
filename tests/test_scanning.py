"""Static and per-frame scan operators: oracle pins (CPU) and the CUDA engine (GPU).

The fixtures in ``tests/golden/scanning.npz`` were produced by the reference's
own ``zstack`` (maomi/scanning.py:8-53), ``single_scan`` / ``psf_fft``
(maomi/movie.py:37-66) and ``blurred_background`` (movie.py:69-102).

Tolerances: the FP64 oracle reproduces the reference's FP64 runs to rounding
(1e-12 relative L2).  The GPU path computes in the data's own precision: FP64
planes must agree with the FP64 oracle to 1e-12, FP32 planes to 1e-5 relative
L2 (the reference's own FP32 path is ~1e-7 from FP64 here; its full-image
test allows 2e-6, tests/test_fixed.py:99-109).
"""

import numpy as np
import pytest

from conftest import golden, rel_l2
from oracle import scanning as S

FP64_TOL = 1e-12
FP32_TOL = 1e-5


# ------------------------------------------------------------------ oracle pins
@pytest.mark.parametrize("case", [0, 1, 2])
def test_oracle_zstack_pin(case):
    d = golden("scanning")
    v, p, m1, m2 = (d[f"z{case}_{k}"] for k in ("volume", "psf", "mask", "colmask"))
    assert rel_l2(S.zstack(v, p, mask=m1, collection_mask=m2), d[f"z{case}_convn64"]) < FP64_TOL
    assert rel_l2(S.zstack(v, p), d[f"z{case}_plain64"]) < FP64_TOL
    assert rel_l2(S.zstack(v, p, mode="legacy_circular"), d[f"z{case}_legacy64"]) < FP64_TOL
    # the reference's FP32 run sits at FP32 rounding from the FP64 restatement
    assert rel_l2(S.zstack(v, p, mask=m1, collection_mask=m2), d[f"z{case}_convn32"]) < 1e-6


@pytest.mark.parametrize("case", [0, 1])
@pytest.mark.parametrize("group", [1, 2, 3])
def test_oracle_single_scan_pin(case, group):
    d = golden("scanning")
    got = S.single_scan(d[f"s{case}_volume"], d[f"s{case}_psf"], scan_avg=group)
    assert rel_l2(got, d[f"s{case}_g{group}"]) < 1e-6
    assert rel_l2(got, d[f"s{case}_g{group}_freq"]) < 1e-6


@pytest.mark.parametrize("name, idx", [("top", np.arange(5)), ("bottom", np.arange(9, 14))])
def test_oracle_blurred_background_pin(name, idx):
    d = golden("scanning")
    kw = dict(power_ratio=0.37, mask=d["b_mask"], zscale=d["b_zscale"][:len(idx)], extra_volumes=[d["b_extra"]])
    assert rel_l2(S.blurred_background(d["b_volume"], idx, d["b_kernel"], **kw), d[f"b_{name}_spatial"]) < FP64_TOL
    got = S.blurred_background(d["b_volume"], idx, d["b_kernel"], frequency_size=d[f"b_{name}_freq_shape"][:2], **kw)
    assert rel_l2(got, d[f"b_{name}_freq"]) < 1e-6


def test_oracle_even_kernel_contract():
    """The reference's own known answer (tests/test_reference.py:10-16): an
    impulse convolved with an even kernel lands at MATLAB's floor(k/2) crop."""
    from scipy.signal import convolve
    v = np.zeros((7, 8, 9))
    v[1, 2, 3] = 1
    p = np.arange(24, dtype=np.float64).reshape(2, 3, 4)
    ref = convolve(v, p, mode="full", method="direct")[1:8, 1:9, 2:11]
    np.testing.assert_allclose(S.zstack(v, p), ref, atol=1e-13)


def test_transform_sizes():
    from maomi_b200._scan import transform_size
    assert transform_size(1) == 64
    assert transform_size(64) == 64
    assert transform_size(65) == 128
    assert transform_size(257) == 384  # 48 x 8 lines (FP32 planes)
    assert transform_size(532) == 768  # 48 x 16 lines (FP32 planes)
    assert transform_size(769) == 1024
    with pytest.raises(ValueError):
        transform_size(1025)


# ------------------------------------------------------------------ GPU parity
@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 1, 2])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_zstack_gpu_matches_oracle(case, dtype):
    from maomi_b200.scanning import zstack
    d = golden("scanning")
    v, p, m1, m2 = (d[f"z{case}_{k}"] for k in ("volume", "psf", "mask", "colmask"))
    tol = FP64_TOL if dtype == "float64" else FP32_TOL
    vv, pp = v.astype(dtype), p.astype(dtype)
    got = zstack(vv, pp, mask=m1, collection_mask=m2, device="cuda").cpu().numpy()
    assert got.dtype == np.dtype(dtype)
    assert rel_l2(got, S.zstack(vv, pp, mask=m1, collection_mask=m2)) < tol
    assert rel_l2(zstack(vv, pp, device="cuda").cpu().numpy(), S.zstack(vv, pp)) < tol
    got = zstack(vv, pp, mode="legacy_circular", device="cuda").cpu().numpy()
    assert rel_l2(got, S.zstack(vv, pp, mode="legacy_circular")) < tol
    if dtype == "float64":  # the reference's own outputs
        assert rel_l2(zstack(v, p, mask=m1, collection_mask=m2, device="cuda").cpu().numpy(),
                      d[f"z{case}_convn64"]) < tol
        assert rel_l2(zstack(v, p, mode="legacy_circular", device="cuda").cpu().numpy(), d[f"z{case}_legacy64"]) < tol


@pytest.mark.gpu
def test_zstack_gpu_even_kernel_contract():
    from scipy.signal import convolve
    from maomi_b200.scanning import zstack
    v = np.zeros((7, 8, 9))
    v[1, 2, 3] = 1
    p = np.arange(24, dtype=np.float64).reshape(2, 3, 4)
    ref = convolve(v, p, mode="full", method="direct")[1:8, 1:9, 2:11]
    np.testing.assert_allclose(zstack(v, p, device="cuda").cpu().numpy(), ref, atol=1e-12)


@pytest.mark.gpu
def test_zstack_gpu_benchmark_size():
    """The static scan of run_fixed at the benchmark size: 512 x 512 x 60
    volume, the 40 x 40 x 46 stage PSF, both masks (FP32 like run_fixed).
    Both modes run on 768-point lines in FP32 (transforms of 532 and 551
    samples); FP64 planes take 1024-point lines for the same request."""
    from maomi_b200.scanning import zstack
    rng = np.random.default_rng(11)
    v = rng.uniform(0, 1, (512, 512, 60)).astype(np.float32)
    p = rng.uniform(0, 1, (40, 40, 46)).astype(np.float32)
    m1 = rng.uniform(0.5, 1.5, (512, 512)).astype(np.float32)
    m2 = rng.uniform(0.2, 1.0, (512, 512)).astype(np.float32)
    got = zstack(v, p, mask=m1, collection_mask=m2, device="cuda").cpu().numpy()
    assert rel_l2(got, S.zstack(v, p, mask=m1, collection_mask=m2)) < FP32_TOL
    got = zstack(v, p, mode="legacy_circular", device="cuda").cpu().numpy()
    assert rel_l2(got, S.zstack(v, p, mode="legacy_circular")) < FP32_TOL
    v64, p64 = v[:, :, :8].astype(np.float64), p[:, :, :6].astype(np.float64)
    got = zstack(v64, p64, device="cuda").cpu().numpy()
    assert got.dtype == np.float64 and rel_l2(got, S.zstack(v64, p64)) < FP64_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 1])
@pytest.mark.parametrize("group", [1, 2, 3])
def test_single_scan_gpu(case, group):
    import torch
    from maomi_b200.movie import psf_fft, single_scan
    d = golden("scanning")
    v, p = d[f"s{case}_volume"], d[f"s{case}_psf"]
    ref = S.single_scan(v, p, scan_avg=group)
    got = single_scan(v, p, scan_avg=group)
    assert isinstance(got, np.ndarray) and got.shape == ref.shape
    assert rel_l2(got, ref) < FP32_TOL
    assert rel_l2(got, d[f"s{case}_g{group}"]) < FP32_TOL
    freq = psf_fft(v.shape, p, group)
    assert freq.shape[2] == -(-v.shape[2] // group)
    got = single_scan(torch.as_tensor(v, device="cuda"), p, scan_avg=group, frequency_psf=freq)
    assert got.is_cuda
    assert rel_l2(got.cpu().numpy(), ref) < FP32_TOL
    got64 = single_scan(v.astype(np.float64), p.astype(np.float64), scan_avg=group)
    assert rel_l2(got64, ref) < FP64_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("name, idx", [("top", np.arange(5)), ("bottom", np.arange(9, 14))])
def test_blurred_background_gpu(name, idx):
    from maomi_b200.movie import blurred_background, psf_fft
    d = golden("scanning")
    kw = dict(power_ratio=0.37, mask=d["b_mask"], zscale=d["b_zscale"][:len(idx)], extra_volumes=[d["b_extra"]])
    ref = S.blurred_background(d["b_volume"], idx, d["b_kernel"], **kw)
    assert rel_l2(blurred_background(d["b_volume"], idx, d["b_kernel"], **kw), ref) < FP32_TOL
    spec = psf_fft(d["b_volume"].shape, d["b_kernel"])
    assert tuple(spec.shape) == tuple(d[f"b_{name}_freq_shape"])
    ref = S.blurred_background(d["b_volume"], idx, d["b_kernel"], frequency_size=spec.shape[:2], **kw)
    got = blurred_background(d["b_volume"], idx, spec, frequency=True, **kw)
    assert rel_l2(got, ref) < FP32_TOL
    assert rel_l2(got, d[f"b_{name}_freq"]) < FP32_TOL


@pytest.mark.gpu
def test_zstack_gpu_384_point_lines():
    """A 300 x 330 x 12 FP32 volume with a 21 x 9 x 5 PSF needs transforms of
    310 x 334 samples (MATLAB crop) or 320 x 338 (periodic mode): 384 = 48 x 8
    lines in both directions (FP32); the FP64 volume takes 512-point lines
    for the same request."""
    from maomi_b200._scan import transform_size
    from maomi_b200.scanning import zstack
    assert transform_size(320) == 384 and transform_size(338) == 384
    rng = np.random.default_rng(12)
    v = rng.uniform(0, 1, (300, 330, 12)).astype(np.float32)
    p = rng.uniform(0, 1, (21, 9, 5)).astype(np.float32)
    m1 = rng.uniform(0.5, 1.5, (300, 330)).astype(np.float32)
    got = zstack(v, p, mask=m1, device="cuda").cpu().numpy()
    assert rel_l2(got, S.zstack(v, p, mask=m1)) < FP32_TOL
    got = zstack(v, p, mode="legacy_circular", device="cuda").cpu().numpy()
    assert rel_l2(got, S.zstack(v, p, mode="legacy_circular")) < FP32_TOL
    v64, p64 = v.astype(np.float64), p.astype(np.float64)
    assert rel_l2(zstack(v64, p64, device="cuda").cpu().numpy(), S.zstack(v64, p64)) < FP64_TOL


@pytest.mark.gpu
def test_conv2_same_gpu():
    from maomi_b200.movie import conv2_same
    rng = np.random.default_rng(5)
    for shape, k in (((37, 50), (4, 7)), ((128, 96), (16, 16)), ((20, 20), (21, 3))):
        im = rng.uniform(-1, 1, shape)
        ker = rng.uniform(0, 1, k)
        assert rel_l2(conv2_same(im, ker), S.conv2_same(im, ker)) < FP64_TOL


@pytest.mark.gpu
def test_scan_errors_match_reference_types():
    from maomi_b200.movie import blurred_background, single_scan
    from maomi_b200.scanning import zstack
    v = np.ones((8, 8, 4), np.float32)
    p = np.ones((3, 3, 4), np.float32)
    with pytest.raises(ValueError, match="Mask must match"):
        zstack(v, p, mask=np.ones((7, 8)), device="cuda")
    with pytest.raises(ValueError, match="Unknown operator"):
        zstack(v, p, mode="nope", device="cuda")
    with pytest.raises(ValueError, match="PSF XY"):
        zstack(v, np.ones((9, 3, 2), np.float32), mode="legacy_circular", device="cuda")
    with pytest.raises(ValueError, match="X,Y,Z"):
        zstack(v[..., 0], p, device="cuda")
    with pytest.raises(ValueError, match="axial length"):
        single_scan(v, p[..., :3])
    with pytest.raises(ValueError, match="scan_avg"):
        single_scan(v, p, scan_avg=0)
    with pytest.raises(ValueError, match="at least one"):
        blurred_background(v, [], np.ones((3, 3)))
    with pytest.raises(ValueError, match="Invalid background"):
        blurred_background(v, [4], np.ones((3, 3)))
    with pytest.raises(ValueError, match="cpu|CPU"):
        zstack(v, p, device="cpu")
