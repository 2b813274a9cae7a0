"""The surrogate's BF16 tensor-core GEMM against an FP32 product of the same
BF16 operands."""

import numpy as np
import pytest

from conftest import rel_l2


def _gemm(a, b, check=True):
    import torch
    from maomi_b200 import _lib
    m, k = a.shape
    n = b.shape[0]
    d = torch.full((m, n), float("nan"), dtype=torch.float32, device=a.device)
    err = torch.zeros(1, dtype=torch.int32, device=a.device)
    _lib.check(_lib.load().mm_gemm_bf16_tn(a.data_ptr(), b.data_ptr(), d.data_ptr(), m, n, k, err.data_ptr(),
                                           int(check), _lib.stream_of(a.device)), "gemm")
    return d


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,k", [(128, 32, 64), (300, 256, 4096), (576, 32, 4096), (4096, 32, 576),
                                   (200, 16, 32), (130, 96, 80), (5120, 2048, 192)])
def test_gemm_bf16_matches_fp32_product(m, n, k):
    import torch
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n + k)
    a = torch.randn((m, k), generator=g, device="cuda").to(torch.bfloat16)
    b = torch.randn((n, k), generator=g, device="cuda").to(torch.bfloat16)
    d = _gemm(a, b)
    ref = a.double() @ b.double().T
    assert torch.isfinite(d).all()
    # FP32 accumulation over k products: ~sqrt(k) * 2^-24 relative
    assert rel_l2(d.cpu().numpy(), ref.cpu().numpy()) < 3e-5


# ------------------------------------------------------------------ surrogate
def _random_problem(S, seed):
    rng = np.random.default_rng(seed)
    X = np.zeros((S, 4096, 32))
    X[..., :18] = rng.normal(size=(S, 4096, 18))
    T = np.zeros((S, 4096, 16))
    T[..., :9] = np.abs(rng.normal(size=(S, 4096, 9)))
    T /= T.sum((1, 2), keepdims=True)
    return X, T


def test_oracle_gradients_match_finite_differences():
    """The FP64 restatement's hand-written backward pass against central
    differences along random directions, for every parameter tensor."""
    from oracle import surrogate as Sg
    X, T = _random_problem(2, 1)
    rng = np.random.default_rng(2)
    p = Sg.init_params(3, base=np.abs(rng.normal(size=(4096, 16))) * 1e-4)
    for k in p:
        if k.startswith("b") and k != "base":
            p[k] = rng.normal(size=p[k].shape) * 1e-3
    p["Wp"][:9] = rng.normal(size=(9, 32)) * 1e-3
    mats = Sg.spectral_matrices()
    y, cache = Sg.forward(p, X, mats)
    g = Sg.backward(p, cache, y, T, mats)
    eps = 1e-6
    for k in g:
        d = rng.normal(size=p[k].shape)
        if k in ("Wp", "bp"):
            d[9:] = 0.0
        q = dict(p)
        q[k] = p[k] + eps * d
        lp = Sg.loss(Sg.forward(q, X, mats)[0], T)
        q[k] = p[k] - eps * d
        lm = Sg.loss(Sg.forward(q, X, mats)[0], T)
        fd, an = (lp - lm) / (2 * eps), float((g[k] * d).sum())
        assert abs(fd - an) <= 1e-5 * max(abs(an), 1e-3), (k, fd, an)


def test_surrogate_host_tables():
    from maomi_b200 import surrogate as S
    off = S._layout()
    sizes = [int(np.prod(S.PARAM_SHAPES[n])) for n in S.PARAM_NAMES]
    assert [b - a for a, b in zip(off[:-1], off[1:])] == sizes
    g = S.screen_groups(60)
    assert g[0] == 0 and g[-1] == 60 and len(g) == 17 and set(np.diff(g)) == {3, 4}
    idx = S.plane_index(46)
    assert len(idx) == 9 and idx.min() >= 0 and idx.max() < 46 and np.all(np.diff(idx) > 0)


def _model_and_batch(S, seed):
    import torch
    from maomi_b200.surrogate import PSFSurrogate
    X, T = _random_problem(S, seed)
    model = PSFSurrogate(device="cuda", seed=seed)
    rng = np.random.default_rng(seed + 1)
    with torch.no_grad():
        model.base.copy_(torch.as_tensor(np.abs(rng.normal(size=(4096, 16))) * 1e-4, dtype=torch.float32))
        for name in ("bl", "b0", "b1", "b2", "b3"):
            model.view(name).copy_(torch.as_tensor(rng.normal(size=32) * 1e-2, dtype=torch.float32))
        model.view("Wp")[:9] = torch.as_tensor(rng.normal(size=(9, 32)) * 1e-3, dtype=torch.float32)
        for l in range(4):
            for k in ("Rr", "Ri"):
                model.view(f"{k}{l}").mul_(16.0)
    xb = torch.as_tensor(X, dtype=torch.float32).to(torch.bfloat16)
    xp = xb.reshape(-1, 32).cuda().contiguous()
    xc = xb.permute(0, 2, 1).reshape(-1, 4096).cuda().contiguous()
    t = torch.as_tensor(T, dtype=torch.float32).cuda()
    Xq = xb.double().numpy()
    return model, xp, xc, t, Xq, T


@pytest.mark.gpu
def test_surrogate_forward_and_gradients_match_fp64_oracle():
    """BF16 tensor-core forward and backward of the network against the FP64
    NumPy definition on the same weights and inputs (8 sites).  BF16 operands
    (8-bit mantissa) bound the agreement: 2 % on the prediction's deviation
    from the base PSF, 5 % on each gradient tensor."""
    from oracle import surrogate as Sg
    model, xp, xc, t, Xq, T = _model_and_batch(8, 4)
    y = model.forward(xp, xc, check=True)
    loss = float(model.backward(xp, xc, t, check=True)[0])
    p = model.numpy_params()
    mats = Sg.spectral_matrices()
    yo, cache = Sg.forward(p, Xq, mats)
    go = Sg.backward(p, cache, yo, T, mats)
    yg = y.cpu().numpy().astype(np.float64)
    assert rel_l2(yg - p["base"], yo - p["base"]) < 2e-2
    assert abs(loss - Sg.loss(yo, T)) < 2e-2 * Sg.loss(yo, T)
    gg = model.numpy_grads()
    errs = {k: rel_l2(gg[k], go[k]) for k in go}
    assert all(v < 5e-2 for v in errs.values()), errs


@pytest.mark.gpu
def test_surrogate_predict_planes():
    """Inference writes the clipped PSF planes from the projection epilogue:
    the same values as the training-path forward followed by the plane
    reshuffle (FP32 sums in another order: 1e-6), and the FP64 definition
    (2 %, as above) on 45 sites: a partial 8-site group and more layer tiles
    (192) than SMs, so each persistent CTA reuses both accumulators."""
    import torch
    from maomi_b200 import _lib
    from maomi_b200.surrogate import targets_to_planes
    from oracle import surrogate as Sg
    model, xp, xc, t, Xq, T = _model_and_batch(45, 6)
    planes = model.predict(xp, xc).cpu().numpy()
    y = model.forward(xp, xc, check=True, train=False)
    ref = torch.empty((45, 9, 64, 64), dtype=torch.float32, device="cuda")
    _lib.check(_lib.load().mm_surrogate_planes(y.data_ptr(), ref.data_ptr(), 45, _lib.stream_of("cuda")), "planes")
    assert planes.shape == (45, 9, 64, 64) and planes.min() >= 0.0
    assert rel_l2(planes, ref.cpu().numpy()) < 1e-6
    p = model.numpy_params()
    yo, _ = Sg.forward(p, Xq[:4], Sg.spectral_matrices())
    po = np.maximum(targets_to_planes(torch.as_tensor(yo)).numpy(), 0.0)
    base = np.maximum(targets_to_planes(torch.as_tensor(np.broadcast_to(p["base"], yo.shape).copy())).numpy(), 0.0)
    assert rel_l2(planes[:4] - base, po - base) < 2e-2


@pytest.mark.gpu
def test_surrogate_inputs_pool_and_window():
    """Site inputs: 16 screen groups, 4x4 pooled, scaled, the site's 64 x 64
    window, then two coordinate channels (checked against NumPy)."""
    import torch
    from maomi_b200 import surrogate as S
    rng = np.random.default_rng(5)
    raw = [rng.normal(size=(320, 288, z)).astype(np.float32) for z in (3, 9, 2)]
    off = np.array([[0, 0], [64, 32], [64, 28]], np.int32)
    xp, xc, pooled = S.site_inputs(raw, off, scale=0.5, device="cuda")
    vol = np.concatenate(raw, axis=2).astype(np.float64)
    g = S.screen_groups(14)
    ref = np.stack([vol[..., a:b].sum(2) for a, b in zip(g[:-1], g[1:])])
    ref = ref.reshape(16, 80, 4, 72, 4).sum((2, 4)) * 0.5 / 16
    np.testing.assert_allclose(pooled.cpu().numpy(), ref, rtol=1e-5, atol=1e-5)
    x = xp.float().cpu().numpy().reshape(3, 64, 64, 32)
    for s, (ox, oy) in enumerate(off):
        np.testing.assert_allclose(x[s, ..., :16], np.moveaxis(ref[:, ox // 4:ox // 4 + 64, oy // 4:oy // 4 + 64], 0, -1),
                                   rtol=1e-2, atol=1e-2)
    grid = (np.arange(64) - 31.5) / 32
    np.testing.assert_allclose(x[0, :, 0, 16], grid, atol=1e-2)
    np.testing.assert_allclose(x[0, 0, :, 17], grid, atol=1e-2)
    assert not x[..., 18:].any()
    assert torch.equal(xc.view(3, 32, 4096).permute(0, 2, 1), xp.view(3, 4096, 32))
    with pytest.raises(ValueError):
        S.site_inputs(raw, np.array([[2, 0]], np.int32), device="cuda")


@pytest.mark.gpu
def test_surrogate_training_gains_over_mean_psf():
    """Trained on plain-propagator PSFs of 20,000 sites from five tissue blocks
    (weak scattering, RMS dn 0.004; ~25 s on one B200), the network predicts
    held-out sites of another block better than the method without it (the
    training-set mean PSF): 0.135 against 0.19 median relative L2 when this
    was written."""
    import torch
    from maomi_b200 import synthetic, surrogate as S
    from maomi_b200.fixed import field_shapes, fixed_locations
    from maomi_b200.optics import OpticalConfig
    cfg = synthetic.benchmark_stage_config(OpticalConfig)
    data = S.training_set(cfg, 20000, seeds=[201, 202, 203, 204, 205], rms=0.004, device="cuda")
    model = S.PSFSurrogate(device="cuda", seed=0, input_scale=data["scale"])
    hist = model.fit(data, epochs=40, batch=64, lr=1e-3, lr_final=5e-5)
    assert hist[-1] < hist[0]
    raw = synthetic.raw_fields(cfg, field_shapes(cfg), sigma=3.0, rms=0.004, seed=7)
    pts = fixed_locations(cfg)[::7]
    t, _, off = S.plain_targets(cfg, raw, pts, device="cuda")
    xp, xc, _ = S.site_inputs(raw, off, scale=data["scale"], device="cuda")
    ref = S.targets_to_planes(t)
    e_net = float(S.rel_l2_per_site(model.predict(xp, xc), ref).median())
    base = S.targets_to_planes(data["base"][None]).expand_as(ref).contiguous()
    e_base = float(S.rel_l2_per_site(base, ref).median())
    assert e_net < 0.85 * e_base, (e_net, e_base)


@pytest.mark.gpu
def test_surrogate_stage_gate():
    """The plain propagator checks a seeded 5 % of the sites: a sample error
    above the tolerance replaces the whole output by the plain PSFs; below it
    the surrogate output stands."""
    import torch
    from maomi_b200 import synthetic, surrogate as S
    from maomi_b200.fixed import field_shapes, fixed_locations
    from maomi_b200.optics import OpticalConfig
    cfg = synthetic.benchmark_stage_config(OpticalConfig)
    raw = synthetic.raw_fields(cfg, field_shapes(cfg), sigma=3.0, rms=0.015, seed=7)
    pts = fixed_locations(cfg)[:400]
    model = S.PSFSurrogate(device="cuda", seed=0)
    strict = S.SurrogateStage(model, gate_fraction=0.05, tolerance=0.01, seed=3).run(cfg, raw, pts)
    assert len(strict["gate"]["sites"]) == 20 and not strict["gate"]["passed"] and strict["source"] == "plain"
    plain, _, _ = S.plain_targets(cfg, raw, pts, device="cuda")
    assert rel_l2(strict["psfs"].cpu().numpy(), S.targets_to_planes(plain).cpu().numpy()) < 1e-6
    loose = S.SurrogateStage(model, gate_fraction=0.05, tolerance=1e9, seed=3).run(cfg, raw, pts)
    assert loose["gate"]["passed"] and loose["source"] == "surrogate"
    np.testing.assert_array_equal(loose["gate"]["sites"], strict["gate"]["sites"])
    assert abs(loose["gate"]["rel_l2"] - strict["gate"]["rel_l2"]) < 1e-9
    # the gate predicts its own sites first; the full prediction of a passed
    # gate reproduces the gate's sample error on those sites
    g = torch.as_tensor(loose["gate"]["sites"], device="cuda")
    ref_g = S.targets_to_planes(plain)[g]
    full = float(S.rel_l2_per_site(loose["psfs"][g].reshape(1, -1), ref_g.reshape(1, -1))[0])
    assert abs(full - loose["gate"]["rel_l2"]) < 1e-6 * max(1.0, full)
