"""Scattering-field generation: the oracle against the reference's own draws
(golden fixtures), the CUDA path against both on the same noise, and the
device generator's determinism and statistics."""

import numpy as np
import pytest

from conftest import cfg_from, golden, rel_l2

TOL = 2e-6  # float32 spectrum and FFT against the reference's float32 run


def _ref_noise(shape, seed):
    import torch
    torch.manual_seed(int(seed))
    re = torch.randn(tuple(int(v) for v in shape), dtype=torch.float32)
    im = torch.randn(tuple(int(v) for v in shape), dtype=torch.float32)
    return re.numpy(), im.numpy()


def _vessels(d):
    return (np.random.default_rng(int(d["vessels_seed"])).random((72, 72, 45)) < 0.05).astype(np.float32)


@pytest.mark.parametrize("tag", ["odd", "even"])
def test_oracle_gp_matches_reference_draw(tag):
    from oracle import fields as OF
    d = golden("fields")
    shape = tuple(int(v) for v in d[f"{tag}_shape"])
    re, im = _ref_noise(shape, d[f"{tag}_seed"])
    out = OF.gp_sample(shape, d[f"{tag}_ls"], float(d[f"{tag}_p"]), re, im, d[f"{tag}_w"])
    assert rel_l2(out, d[f"{tag}_out"]) < TOL


def test_oracle_prepare_fields_matches_reference():
    """Scattered fields of the reference's GPU-vs-CPU geometry (stage_reftest)
    and the same geometry with a vessel volume (partial slabs, offsets)."""
    from oracle import fields as OF
    from maomi_b200.optics import OpticalConfig
    d = golden("stage_reftest")
    cfg = cfg_from(d, cls=OpticalConfig)
    shapes = OF.field_extents(cfg)[0]
    raw = OF.prepare_fields(cfg, OF.torch_noise(shapes, cfg.seed))
    assert all(rel_l2(raw[i], d[f"raw{i}"]) < TOL for i in range(3))
    f = golden("fields")
    raw = OF.prepare_fields(cfg, OF.torch_noise(shapes, cfg.seed), _vessels(f))
    assert all(rel_l2(raw[i], f[f"vessel_raw{i}"]) < TOL for i in range(3))


def test_slab_bounds_follow_the_reference_chunking():
    from maomi_b200.fields import _slab_bounds
    a, b, c = _slab_bounds(22, 10, 5, 12)
    assert a == [0, 2, 7, 12, 17, 22] and b == list(range(22, 33)) and c == [32, 37, 42, 44]
    a, _, c = _slab_bounds(20, 10, 5, 10)
    assert a == [0, 5, 10, 15, 20] and c == [30, 35, 40]


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["odd", "even"])
def test_gp_cuda_matches_reference_draw(tag):
    from maomi_b200.fields import masked_3DGP_test
    d = golden("fields")
    shape = tuple(int(v) for v in d[f"{tag}_shape"])
    noise = _ref_noise(shape, d[f"{tag}_seed"])
    out = masked_3DGP_test(shape, d[f"{tag}_ls"], float(d[f"{tag}_p"]), l_weights=d[f"{tag}_w"], noise=noise)
    assert out.is_cuda and out.dtype.is_floating_point
    assert rel_l2(out.cpu().numpy(), d[f"{tag}_out"]) < TOL


@pytest.mark.gpu
def test_prepare_fields_cuda_matches_reference():
    from oracle import fields as OF
    from maomi_b200.fields import prepare_fields
    from maomi_b200.optics import OpticalConfig
    d = golden("stage_reftest")
    cfg = cfg_from(d, cls=OpticalConfig)
    noise = OF.torch_noise(OF.field_extents(cfg)[0], cfg.seed)
    raw = prepare_fields(cfg, noise=noise)
    assert all(rel_l2(raw[i].cpu().numpy(), d[f"raw{i}"]) < TOL for i in range(3))
    f = golden("fields")
    raw = prepare_fields(cfg, _vessels(f), noise=noise)
    assert all(rel_l2(raw[i].cpu().numpy(), f[f"vessel_raw{i}"]) < TOL for i in range(3))
    flat = prepare_fields(cfg, scatter=False)
    assert all(not t.any() for t in flat)
    with pytest.raises(ValueError):
        prepare_fields(cfg, np.zeros((72, 72, 10), np.float32), noise=noise)


@pytest.mark.gpu
def test_gp_cuda_single_plane_and_mask():
    """nz = 1, a mean and an array mask, against the oracle on the same noise."""
    from oracle import fields as OF
    from maomi_b200.fields import masked_3DGP_test
    shape = (9, 6, 1)
    rng = np.random.default_rng(3)
    re, im = rng.normal(size=shape).astype(np.float32), rng.normal(size=shape).astype(np.float32)
    ls = np.array([[1.5, 2.0, 0.5]], np.float32)
    mask = (rng.random(shape) < 0.5).astype(np.float32)
    out = masked_3DGP_test(shape, ls, 2.0, mu=0.25, bin_mask=mask, noise=(re, im)).cpu().numpy()
    ref = OF.gp_sample(shape, ls, 2.0, re, im, mu=0.25, bin_mask=mask)
    assert rel_l2(out, ref) < TOL


@pytest.mark.gpu
def test_gp_cuda_wide_grid_uses_voxel_kernel():
    """A grid whose per-plane factor tables exceed 48 KB of shared memory
    (4 scales x 3,100 rows) takes the per-voxel kernel; same result."""
    from oracle import fields as OF
    from maomi_b200.fields import masked_3DGP_test
    shape = (3, 3100, 2)
    rng = np.random.default_rng(4)
    re, im = rng.normal(size=shape).astype(np.float32), rng.normal(size=shape).astype(np.float32)
    ls = np.array([[1.0, 40.0, 0.5], [2.0, 90.0, 1.0], [0.5, 10.0, 0.2], [3.0, 200.0, 2.0]], np.float32)
    w = np.array([0.5, 0.3, 0.2, 0.1], np.float32)
    out = masked_3DGP_test(shape, ls, 1.5, l_weights=w, noise=(re, im)).cpu().numpy()
    assert rel_l2(out, OF.gp_sample(shape, ls, 1.5, re, im, w)) < TOL


@pytest.mark.gpu
def test_benchmark_fields_device_draws():
    """Benchmark geometry (768 x 768 x 10/46/4): the device generator is
    deterministic per seed, field B matches the oracle on that same device
    noise, and its mean and power are what the spectrum predicts."""
    import torch
    from oracle import fields as OF
    from maomi_b200 import synthetic
    from maomi_b200.fields import prepare_fields, field_extents
    from maomi_b200.optics import OpticalConfig
    cfg = synthetic.benchmark_stage_config(OpticalConfig)
    a = prepare_fields(cfg)
    b = prepare_fields(cfg)
    assert all(torch.equal(x, y) for x, y in zip(a, b))
    shapes = field_extents(cfg)[0]
    assert [tuple(t.shape) for t in a] == [tuple(s) for s in shapes]
    # the device draws for field B, re-made and fed to the oracle
    gen = torch.Generator(device="cuda").manual_seed(int(cfg.seed))
    s0 = tuple(shapes[0])
    torch.randn(s0, generator=gen, device="cuda"), torch.randn(s0, generator=gen, device="cuda")
    s1 = tuple(shapes[1])
    re = torch.randn(s1, generator=gen, device="cuda").cpu().numpy()
    im = torch.randn(s1, generator=gen, device="cuda").cpu().numpy()
    ls = np.repeat(np.asarray(cfg.scatter_scales_um, np.float32)[:, None], 3, 1) * np.float32(cfg.vres)
    got = a[1].cpu().numpy()
    assert rel_l2(got, OF.gp_sample(s1, ls, 1.0, re, im, cfg.scatter_weights)) < TOL
    # statistics of x = 2 sqrt(N) Re(ifft(noise * S)): the sample mean is
    # 2 Re(z_dc) / sqrt(N) with z_dc the noise times S at the spectrum centre;
    # the sample power (1/N) sum x^2 ~ (2/N) sum_k S_k^2 |noise_k|^2 has mean
    # 4 sum(S^2) / N and relative spread sqrt(sum S^4) / sum(S^2)
    S = OF.spectrum(s1, ls, cfg.scatter_weights).astype(np.float64)
    n = S.size
    s_dc = S[tuple(v // 2 for v in s1)]
    assert abs(got.mean(dtype=np.float64)) < 5 * 2 * s_dc / np.sqrt(n)
    power = float((got.astype(np.float64) ** 2).mean())
    expect = 4 * (S ** 2).sum() / n
    spread = np.sqrt((S ** 4).sum()) / (S ** 2).sum()
    assert abs(power / expect - 1) < 5 * spread + 1e-3
