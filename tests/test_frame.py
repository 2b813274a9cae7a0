"""The optical part of one movie frame (maomi/movie.py:601-679) on the GPU
against the oracle's restatements of its operators.

The frame is single_scan of the focal slab of (activity + base) with the PSF
over scan_avg groups, the optional extra blur of the frame, and both tails as
frequency-domain blurred backgrounds of the planes outside the slab.  The
oracle composes oracle.scanning's single_scan, conv2_same and
blurred_background (FP64); the GPU computes in FP32: 1e-5 relative L2.
"""

import numpy as np
import pytest

from conftest import rel_l2
from oracle import scanning as S

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _scene(seed=4):
    rng = np.random.default_rng(seed)
    shape = (48, 40, 20)
    temp = rng.uniform(0, 1, shape).astype(np.float32)
    base = rng.uniform(0, .3, shape).astype(np.float32)
    psf = rng.uniform(0, 1, (7, 6, 6)).astype(np.float32)
    tails = []
    for j in range(2):
        k = rng.uniform(0, 1, (16, 16)).astype(np.float32)
        tails.append({"kernel": k / k.sum(), "weight": 0.3 + 0.2 * j,
                      "mask": rng.uniform(0.5, 1.5, shape[:2]).astype(np.float32),
                      "zscale": rng.uniform(0.5, 2.0, 30)})
    blur = rng.uniform(0, .1, (3, 3)).astype(np.float32)
    return shape, temp, base, psf, tails, blur


def _oracle_frame(shape, temp, base, psf, tails, blur, z, scan_avg, scale, sf):
    from maomi_b200.movie import _smooth_length
    depth = psf.shape[2]
    t64, b64 = temp.astype(np.float64), base.astype(np.float64)
    frame = S.single_scan(t64[:, :, z:z + depth] + b64[:, :, z:z + depth], psf, scan_avg=scan_avg) * (
        scale / (2 * sf * sf))
    if blur is not None:
        frame = frame + S.conv2_same(frame, blur)
    X, Y, nz = shape
    for j, spec in enumerate(tails):
        idx = np.arange(z) if j == 0 else np.arange(z + depth, nz)
        zs = spec["zscale"]
        if len(idx) == 0:
            idx, zs = np.arange(nz), None
        k = spec["kernel"]
        size = (_smooth_length(X + k.shape[0] - 1), _smooth_length(Y + k.shape[1] - 1))
        frame = frame + S.blurred_background(t64, idx, k, power_ratio=spec["weight"], mask=spec["mask"],
                                             zscale=zs, extra_volumes=[b64], frequency_size=size) * (scale / (sf * sf))
    return frame


@pytest.mark.parametrize("z", [0, 5, 14])
@pytest.mark.parametrize("with_blur", [False, True])
def test_frame_matches_oracle(z, with_blur):
    from maomi_b200.movie import FrameScanner
    shape, temp, base, psf, tails, blur = _scene()
    blur = blur if with_blur else None
    fs = FrameScanner(shape, psf, scan_avg=2, tails=tails, blur=blur)
    got = fs.frame(temp, base, z, scale=3.5, sf=2.0).cpu().numpy()
    ref = _oracle_frame(shape, temp, base, psf, tails, blur, z, 2, 3.5, 2.0)
    assert got.shape == shape[:2]
    assert rel_l2(got, ref) < TOL


def test_frame_argument_errors():
    from maomi_b200.movie import FrameScanner
    shape, temp, base, psf, tails, blur = _scene()
    fs = FrameScanner(shape, psf, scan_avg=2, tails=tails)
    with pytest.raises(ValueError, match="outside volume"):
        fs.frame(temp, base, 15)
    with pytest.raises(ValueError, match="shape"):
        fs.frame(temp[:-1], base[:-1], 0)
    with pytest.raises(ValueError, match="Both optical tails"):
        FrameScanner(shape, psf, tails=tails[:1])
