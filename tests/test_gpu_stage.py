"""CUDA optical stage vs the CPU oracle and the reference's golden outputs.

Tolerance (north star): relative L2 <= 1e-5 against the FP64 reference for
PSFs, masks and tails.  The CUDA path forms every large phase argument in
FP64 and rounds once; FFT arithmetic is FP32."""

import numpy as np
import pytest

from conftest import cfg_from, golden, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def small():
    from oracle import optics as O
    from maomi_b200 import synthetic
    d = golden("stage_small")
    cfg = cfg_from(d)
    raw = synthetic.raw_fields(cfg, O.field_shapes(cfg), sigma=float(d["raw_sigma"]), rms=float(d["raw_rms"]),
                               seed=int(d["raw_seed"]))
    return d, cfg, raw


def _stage_errors(out, d, prefix="f64_"):
    errs = {k: rel_l2(out[k], d[prefix + k]) for k in ("psf_3d", "psf", "psf_raw", "mask_raw", "energies")}
    for t in ("psfT", "psfB"):
        for k in ("convmask", "weight", "psfZ", "mask_raw"):
            errs[f"{t}.{k}"] = rel_l2(out[t][k], d[f"{prefix}{t}_{k}"])
    return errs


def test_pupil_fp64_zernike():
    from maomi_b200.optics import pupil
    d = golden("numerics")
    cfg = cfg_from(d, "zcfg_")
    u = pupil(cfg).cpu().numpy()
    assert rel_l2(u, d["zpupil64"]) < 1e-6


def test_small_stage_matches_reference_fp64(small):
    from maomi_b200.fixed import run_stage
    d, cfg, raw = small
    out = run_stage(cfg, raw, d["points"])
    errs = _stage_errors(out, d)
    bad = {k: v for k, v in errs.items() if not v < TOL}
    assert not bad, errs


@pytest.mark.parametrize("schedule", ["persistent", "batched"])
def test_schedules_agree(small, schedule):
    from maomi_b200.fixed import run_stage
    d, cfg, raw = small
    ref = run_stage(cfg, raw, d["points"], schedule="persistent", slots=4)
    out = run_stage(cfg, raw, d["points"], schedule=schedule, slots=2)
    np.testing.assert_array_equal(out["psf_3d"], ref["psf_3d"])
    assert rel_l2(out["psfT"]["convmask"], ref["psfT"]["convmask"]) < 1e-6
    assert rel_l2(out["mask_raw"], ref["mask_raw"]) < 1e-12


def test_evaluate_per_site_matches_oracle(small):
    """OpticalPlan.evaluate schema and per-site products vs the FP64 oracle."""
    from oracle import optics as O
    from maomi_b200.backends.cuda.batched import OpticalPlan
    d, cfg, raw = small
    plan = OpticalPlan(cfg, raw)
    out = plan.evaluate(d["points"], batch_size=4, tails=True)
    ref = O.propagate_sites(cfg, [np.asarray(a, np.float64) for a in raw], d["points"], O.pupil(cfg, np.float64))
    assert out["psfs"].shape == ref["psfs"].shape and out["psfs"].dtype == np.float32
    assert rel_l2(out["psfs"], ref["psfs"]) < TOL
    for j, name in enumerate(("top", "bottom")):
        assert rel_l2(out[name]["convmask"], ref["convmasks"][j]) < TOL
        assert rel_l2(out[name]["weight"], ref["weights"][j]) < TOL
        assert rel_l2(out[name]["profile"], ref["profiles"][j]) < TOL
    assert plan.paths_evaluated == len(d["points"])


def test_evaluate_graph_replays_a_captured_focal_batch(small):
    """prepare_graph / evaluate_graph (reference batched.py:103-146): the focal
    path of a fixed 4-site batch is captured once in a CUDA graph and replayed
    per chunk of the 9 sites, the last chunk padded with window (0, 0) sites.
    The PSFs equal evaluate's bit for bit (same kernels on the same inputs),
    the padding is reported, only the caller's sites are counted, and a second
    call reuses the captured graph."""
    from maomi_b200.backends.cuda.batched import OpticalPlan
    d, cfg, raw = small
    plan = OpticalPlan(cfg, raw)
    ref = OpticalPlan(cfg, raw).evaluate(d["points"], batch_size=4)
    out = plan.evaluate_graph(d["points"], batch_size=4)
    assert out["graph_padding_slots"] == 3 and out["tails_computed"] is False
    np.testing.assert_array_equal(out["psfs"], ref["psfs"])
    graph = plan.graphs[4]["graph"]
    again = plan.evaluate_graph(d["points"][::-1], batch_size=4)
    assert plan.graphs[4]["graph"] is graph
    np.testing.assert_array_equal(again["psfs"], ref["psfs"][::-1])
    assert plan.paths_evaluated == 2 * len(d["points"])
    with pytest.raises(ValueError, match="Outside FOV"):
        plan.evaluate_graph([[-1.0, 0.0]], batch_size=4)


@pytest.fixture(scope="module")
def bench_sites():
    from oracle import optics as O
    from maomi_b200 import synthetic
    d = golden("stage_bench_sites")
    cfg = cfg_from(d)
    raw = synthetic.raw_fields(cfg, O.field_shapes(cfg), sigma=float(d["raw_sigma"]), rms=float(d["raw_rms"]),
                               seed=int(d["raw_seed"]))
    return d, cfg, raw


@pytest.mark.parametrize("precision", ["compensated", "compensated-full", "mixed", "fp64"])
def test_benchmark_geometry_matches_reference_fp64(bench_sites, precision):
    """256x256 windows, 60 screens, Zernike pupil: three sites vs the reference.

    All-FP32 line transforms sit at ~1.2e-5 here: the rounding of the DFT
    rotation constants is the same in all 240 line transforms of a site, so
    it adds up coherently.  Carrying those constants as hi + lo float pairs
    (compensated: 1.8e-6; with the twiddle tables too, compensated-full:
    4.6e-7), the inverse half in FP64 (mixed: 6e-6) or everything in FP64
    stays inside 1e-5."""
    from maomi_b200.backends.cuda.batched import OpticalPlan
    d, cfg, raw = bench_sites
    plan = OpticalPlan(cfg, raw, precision=precision)
    out = plan.evaluate(d["points"], batch_size=3, tails=True)
    assert rel_l2(out["psfs"], d["f64_psf_3d"]) < TOL
    assert rel_l2(out["psfs"].sum((1, 2, 3), dtype=np.float64), d["f64_energies"]) < TOL


def test_benchmark_geometry_fp32_error_is_reported(bench_sites):
    """The all-FP32 mode is kept for speed; its error stays below 3e-5."""
    from maomi_b200.backends.cuda.batched import OpticalPlan
    d, cfg, raw = bench_sites
    out = OpticalPlan(cfg, raw, precision="fp32").evaluate(d["points"], batch_size=3)
    assert rel_l2(out["psfs"], d["f64_psf_3d"]) < 3e-5


def test_reference_test_geometry_dense_windows():
    """n=112 / n2=72 windows (ss=2, custom pupil phase, three photon orders):
    the circular-convolution line path against the reference's FP64 run."""
    from dataclasses import replace
    from maomi_b200.fixed import run_stage
    from maomi_b200.optics import pupil
    d = golden("stage_reftest")
    base = cfg_from(d)
    raw = [d[f"raw{i}"] for i in range(3)]
    for mode in ("two-photon", "three-photon", "temporal-focusing"):
        cfg = replace(base, scaling=mode)
        u = pupil(cfg, custom_phase=d["custom_phase"])
        out = run_stage(cfg, raw, d["points"], uin=u)
        errs = _stage_errors(out, d, f"{mode}_f64_")
        bad = {k: v for k, v in errs.items() if not v < TOL}
        assert not bad, (mode, errs)


def test_v4_matches_reference():
    from maomi_b200.numerics import v4_interpolate
    from maomi_b200.backends.cuda.interpolation import evaluate_v4
    d = golden("numerics")
    np.testing.assert_allclose(v4_interpolate(d["v4_points"], d["v4_values"], d["v4_queries"]), d["v4_out"],
                               rtol=1e-9, atol=1e-10)
    q = d["v4_queries"].reshape(2, 71, 2)
    np.testing.assert_allclose(v4_interpolate(d["v4_points"], d["v4_values"][:, :3], q),
                               d["v4_out"][:, :3].reshape(2, 71, 3), rtol=1e-9, atol=1e-10)
    lq = np.stack(np.meshgrid(np.arange(64) + .5, np.arange(64) + .5, indexing="ij"), -1)
    np.testing.assert_allclose(v4_interpolate(d["v4l_points"], d["v4l_values"], lq), d["v4l_out"], rtol=1e-9,
                               atol=1e-10)
    from oracle.optics import v4_coefficients
    c = v4_coefficients(d["v4_points"], d["v4_values"])
    np.testing.assert_allclose(evaluate_v4(d["v4_points"], c, d["v4_queries"]), d["v4_out"], rtol=1e-9, atol=1e-10)
    # edge cases of numerics.py:116-120
    one = v4_interpolate([[3, 4]], [[2, 7]], np.zeros((5, 6, 2)))
    np.testing.assert_array_equal(one, np.broadcast_to([2, 7], (5, 6, 2)))
    assert v4_interpolate(d["v4_points"], d["v4_values"], np.empty((0, 2))).shape == (0, 4)


def test_gather_and_resample_plan():
    import torch
    from oracle.optics import resample_matrix
    from maomi_b200.backends.cuda.native import ResamplePlan, gather
    rng = np.random.default_rng(5)
    src = (rng.standard_normal((3, 40, 44)) + 1j * rng.standard_normal((3, 40, 44))).astype(np.complex64)
    edge = rng.uniform(0.5, 1, (16, 16)).astype(np.float32)
    off = np.array([[0, 0], [24, 28], [5, 9]], np.int32)
    out = gather(torch.as_tensor(src, device="cuda"), torch.as_tensor(edge, device="cuda"), off, 16).cpu().numpy()
    for b, (x, y) in enumerate(off):
        np.testing.assert_array_equal(out[b], src[:, x:x + 16, y:y + 16] * edge)
    field = (rng.standard_normal((2, 4, 24, 24)) + 1j * rng.standard_normal((2, 4, 24, 24))).astype(np.complex64)
    axial = rng.uniform(0.5, 1, 4).astype(np.float32)
    for ss, order in ((2, 2), (3, 1), (1, 3)):
        rp = ResamplePlan(24, 24, ss, "cuda")
        got = rp(torch.as_tensor(field, device="cuda"), 1.7, order=order, axial=axial).cpu().numpy()
        m = resample_matrix(24, ss)
        p = np.abs(field.astype(np.complex128)) ** (2 * order)
        ref = np.einsum("xh,bzhw,yw->bxyz", m, p, m) * 1.7 * axial
        assert rel_l2(got, ref) < 1e-6


def test_full_size_translation_invariance():
    """Benchmark geometry, 4,225 sites, zero screens: every site sees the same
    optics, so all PSFs coincide and the v4 mask is flat."""
    from maomi_b200 import synthetic
    from maomi_b200.fixed import field_shapes, run_stage
    from maomi_b200.optics import OpticalConfig
    cfg = synthetic.benchmark_stage_config(OpticalConfig)
    raw = [np.zeros(s, np.float32) for s in field_shapes(cfg)]
    out = run_stage(cfg, raw)
    p = out["psf_3d"]
    assert p.shape == (4225, 40, 40, 46)
    np.testing.assert_array_equal(p, np.broadcast_to(p[0], p.shape))
    # equal site values: the v4 mask is that value times the spline of ones,
    # checked against the FP64 oracle on a sample of pixels
    from oracle.optics import v4_coefficients, v4_evaluate
    pts = out["points_um"] * cfg.vres
    ones = v4_coefficients(pts, np.ones(len(pts)))
    rng = np.random.default_rng(0)
    ij = rng.integers(0, 512, (400, 2))
    ref = v4_evaluate(pts, ones, ij + 0.5) * out["energies"][0]
    np.testing.assert_allclose(out["mask_raw"][ij[:, 0], ij[:, 1]], ref, rtol=1e-9)
    np.testing.assert_allclose(out["energies"], out["energies"][0], rtol=1e-12)  # FP64 atomics order
    for t in ("psfT", "psfB"):
        assert out[t]["weight"] > 0
        np.testing.assert_allclose(out[t]["weights_per_point"], out[t]["weights_per_point"][0], rtol=1e-6)


@pytest.mark.gpu
def test_v4_lattice_parity_solve_matches_dense():
    """The fixed 65x65 site lattice solved as four reflection-parity blocks
    gives the dense FP64 LU's masks (4,225 points -> 512x512, 3 columns)."""
    from maomi_b200 import synthetic
    from maomi_b200.fixed import fixed_locations
    from maomi_b200.numerics import lattice_index, v4_evaluate_grid_device, v4_factor_device, v4_solve_device
    from maomi_b200.optics import OpticalConfig
    cfg = synthetic.benchmark_stage_config(OpticalConfig)
    pts = fixed_locations(cfg) * cfg.vres
    assert lattice_index(pts) is not None
    vals = np.random.default_rng(3).uniform(0.5, 2.0, (len(pts), 3))
    p, c_lat = v4_solve_device(v4_factor_device(pts), vals)
    _, c_den = v4_solve_device(v4_factor_device(pts, structured=False), vals)
    m_lat = v4_evaluate_grid_device(p, c_lat, 512, 512).cpu().numpy()
    m_den = v4_evaluate_grid_device(p, c_den, 512, 512).cpu().numpy()
    assert rel_l2(m_lat, m_den) < 1e-9
    # tabulated Green function on the integer lattice: the same sums, bit for bit
    m_tab = v4_evaluate_grid_device(p, c_lat, 512, 512, points_host=pts).cpu().numpy()
    np.testing.assert_array_equal(m_tab, m_lat)
    assert rel_l2(c_lat.cpu().numpy(), c_den.cpu().numpy()) < 1e-6


@pytest.mark.gpu
def test_pipelined_stages_match_single_runs(small):
    """run_stages (upload of block i+1 and compute overlapping the copies of
    block i) returns, block for block, what run_stage returns."""
    import torch
    from maomi_b200 import synthetic
    from maomi_b200.fixed import run_stage, run_stages
    from oracle import optics as O
    d, cfg, raw = small
    other = synthetic.raw_fields(cfg, O.field_shapes(cfg), sigma=2.0, rms=0.01, seed=99)
    blocks = [raw, [torch.from_numpy(a).pin_memory() for a in other], raw]
    got = list(run_stages(cfg, blocks, d["points"], device="cuda", precision="fp64"))
    assert len(got) == 3
    reused = [dict(r) for r in run_stages(cfg, blocks[:1], d["points"], device="cuda", precision="fp64",
                                          reuse=True)]
    np.testing.assert_array_equal(reused[0]["psf_3d"], got[0]["psf_3d"])
    for res, src in zip(got, (raw, other, raw)):
        ref = run_stage(cfg, src, d["points"], device="cuda", precision="fp64")
        # psf_3d is deterministic; the site sums, energies and profiles are
        # FP64 atomic sums whose order may differ between runs
        np.testing.assert_array_equal(res["psf_3d"], ref["psf_3d"])
        for key in ("psf", "psf_raw", "mask_raw", "energies"):
            np.testing.assert_allclose(res[key], ref[key], rtol=1e-10, err_msg=key)
        for t in ("psfT", "psfB"):
            np.testing.assert_allclose(res[t]["convmask"], ref[t]["convmask"], rtol=1e-10)
            np.testing.assert_allclose(res[t]["weight"], ref[t]["weight"], rtol=1e-10)
        np.testing.assert_allclose(res["negative_resampling_mass_fraction"], ref["negative_resampling_mass_fraction"],
                                   rtol=1e-10, atol=1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny", [(4, 5), (7, 6), (2, 3)])
def test_v4_parity_blocks_small_lattices(nx, ny):
    """Even and odd lattice sizes (with and without a centre row/column),
    shuffled point order: the parity-block solve equals the dense LU."""
    from maomi_b200.numerics import lattice_index, v4_factor_device, v4_solve_device
    rng = np.random.default_rng(nx * 10 + ny)
    pts = np.array([(8.0 * i, 8.0 * j + 4.0) for i in range(nx) for j in range(ny)])[rng.permutation(nx * ny)]
    assert lattice_index(pts) is not None
    vals = rng.normal(size=(len(pts), 3))
    _, a = v4_solve_device(v4_factor_device(pts), vals)
    _, b = v4_solve_device(v4_factor_device(pts, structured=False), vals)
    assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-10


def test_single_site_stage_matches_oracle_fp64(small):
    """One site: the v4 masks degenerate to the site's constant values (the
    reference's single-point branch); PSFs and tails as for any site."""
    from oracle import optics as O
    from maomi_b200.fixed import run_stage
    d, cfg, raw = small
    pt = np.asarray(d["points"])[:1]
    out = run_stage(cfg, raw, pt, precision="fp64")
    u64 = O.pupil(cfg, np.float64)
    ref = O.propagate(cfg, [np.asarray(a, np.float64) for a in raw], pt, u64)
    for key in ("psf_3d", "psf", "mask_raw", "energies"):
        assert rel_l2(out[key], ref[key]) < TOL, key
    assert np.allclose(out["mask_raw"], out["mask_raw"].flat[0])
    for t in ("psfT", "psfB"):
        assert rel_l2(out[t]["convmask"], ref[t]["convmask"]) < TOL


@pytest.mark.gpu
def test_reused_pinned_buffers_hold_for_depth_results(small):
    """run_stages(reuse=True) over 5 blocks of 3 different tissues: every
    result equals run_stage's, and each stays intact while ``depth`` further
    results are yielded; a second generator running side by side never
    writes into the first one's buffers."""
    from maomi_b200 import synthetic
    from maomi_b200.fixed import run_stage, run_stages
    from oracle import optics as O
    d, cfg, raw = small
    tissues = [raw] + [synthetic.raw_fields(cfg, O.field_shapes(cfg), sigma=2.0, rms=0.01, seed=s) for s in (51, 52)]
    expect = [run_stage(cfg, t, d["points"], precision="fp64")["psf_3d"] for t in tissues]
    order = [0, 1, 2, 0, 1]
    depth = 2
    gen_a = run_stages(cfg, [tissues[i] for i in order], d["points"], precision="fp64", reuse=True, depth=depth)
    gen_b = run_stages(cfg, [tissues[i] for i in reversed(order)], d["points"], precision="fp64", reuse=True,
                       depth=depth)
    got_a, got_b = [], []
    for k in range(len(order)):
        got_a.append(next(gen_a))
        got_b.append(next(gen_b))
        for j in range(max(0, k - depth), k + 1):
            np.testing.assert_array_equal(got_a[j]["psf_3d"], expect[order[j]], err_msg=f"a: result {j} at {k}")
            np.testing.assert_array_equal(got_b[j]["psf_3d"], expect[order[::-1][j]], err_msg=f"b: result {j} at {k}")
    for g in (gen_a, gen_b):
        with pytest.raises(StopIteration):
            next(g)


@pytest.mark.gpu
def test_dependency_wait_runs_out_with_timeout_status(small):
    """The persistent launch's bounded dependency wait: one site's first item
    waits for a counter nothing publishes (a short poll limit), the kernel
    sets its error flag, every CTA leaves, and the call reports the timeout.
    The context stays usable: the next run matches a fresh plan's."""
    import torch
    from maomi_b200.backends.cuda.batched import OpticalPlan
    d, cfg, raw = small
    plan = OpticalPlan(cfg, raw)
    _, off = plan.offsets(d["points"])
    with torch.inference_mode():
        with pytest.raises(RuntimeError, match="timed out"):
            plan.run_sites(off, tail_per_site=True, slots=4, schedule="persistent",
                           fault_drill={"hold_site": 3, "spin_limit": 2048})
        torch.cuda.synchronize()
        again = plan.run_sites(off, tail_per_site=True, slots=4, schedule="persistent")["focal"].cpu().numpy()
        fresh = OpticalPlan(cfg, raw).run_sites(off, tail_per_site=True, slots=4)["focal"].cpu().numpy()
    np.testing.assert_array_equal(again, fresh)
