"""The CPU oracle against the reference's own outputs (golden fixtures).

These pin the oracle: FP64 restatement vs the reference's FP64 run to ~1e-10,
FP32 restatement vs the reference's FP32 run to the level set by PyTorch's
float32 vector norm (a global scale of a few 1e-6 in |E|^4)."""

import numpy as np
import pytest

from conftest import cfg_from, golden, rel_l2
from oracle import optics as O
from maomi_b200 import synthetic

STAGE_KEYS = ("psf_3d", "psf", "psf_raw", "mask_raw", "energies")
TAIL_KEYS = ("convmask", "weight", "psfZ", "mask_raw")


def _check(out, d, prefix, tol, keys=STAGE_KEYS, tails=True):
    for k in keys:
        assert rel_l2(out[k], d[f"{prefix}{k}"]) < tol, (prefix, k, rel_l2(out[k], d[f"{prefix}{k}"]))
    if tails:
        for t in ("psfT", "psfB"):
            for k in TAIL_KEYS:
                e = rel_l2(out[t][k], d[f"{prefix}{t}_{k}"])
                assert e < tol, (prefix, t, k, e)


def _small_raw(d, cfg):
    raw = synthetic.raw_fields(cfg, O.field_shapes(cfg), sigma=float(d["raw_sigma"]), rms=float(d["raw_rms"]),
                               seed=int(d["raw_seed"]))
    np.testing.assert_allclose([float(np.sum(a, dtype=np.float64)) for a in raw], d["raw_checksum"], rtol=1e-6,
                               atol=1e-9)
    return raw


@pytest.mark.parametrize("rdt,prefix,tol", [(np.float64, "f64_", 1e-10), (np.float32, "f32_", 5e-5)])
def test_small_stage(rdt, prefix, tol):
    d = golden("stage_small")
    cfg = cfg_from(d)
    raw = _small_raw(d, cfg)
    u = O.pupil(cfg, rdt)
    assert rel_l2(u, d["pupil64" if rdt == np.float64 else "pupil32"]) < (1e-14 if rdt == np.float64 else 1e-6)
    out = O.propagate(cfg, [np.asarray(a, rdt) for a in raw], d["points"], u)
    _check(out, d, prefix, tol)


@pytest.mark.parametrize("mode", ["flat", "two-photon", "three-photon", "temporal-focusing"])
def test_reference_test_geometry(mode):
    """n=112 / n2=72, ss=2, custom pupil phase, both tails (tests/test_fixed.py:147-172)."""
    from dataclasses import replace
    d = golden("stage_reftest")
    cfg = cfg_from(d)
    if mode == "flat":
        raw = [np.zeros(np.shape(d[f"raw{i}"]), np.float32) for i in range(3)]
        prefix = "flat_"
    else:
        cfg = replace(cfg, scaling=mode)
        raw = [d[f"raw{i}"] for i in range(3)]
        prefix = f"{mode}_"
    for rdt, p, tol in ((np.float64, "f64_", 1e-10), (np.float32, "f32_", 5e-5)):
        u = O.pupil(cfg, rdt, custom_phase=d["custom_phase"])
        assert rel_l2(u, d[prefix + ("pupil64" if rdt == np.float64 else "pupil32")]) < 1e-6
        out = O.propagate(cfg, [np.asarray(a, rdt) for a in raw], d["points"], u)
        _check(out, d, prefix + p, tol)


def test_benchmark_geometry_sites():
    """256x256 windows, 60 screens, Zernike pupil: per-site products (FP64)."""
    d = golden("stage_bench_sites")
    cfg = cfg_from(d)
    raw = synthetic.raw_fields(cfg, O.field_shapes(cfg), sigma=float(d["raw_sigma"]), rms=float(d["raw_rms"]),
                               seed=int(d["raw_seed"]))
    np.testing.assert_allclose([float(np.sum(a, dtype=np.float64)) for a in raw], d["raw_checksum"], rtol=1e-6)
    u = O.pupil(cfg, np.float64)
    sites = O.propagate_sites(cfg, [np.asarray(a, np.float64) for a in raw], d["points"], u)
    # The Zernike phase passes through a float32 buffer in both precisions
    # (_optical_math.py:190); its occasional 1-ulp float32 re-roundings bound
    # the FP64 agreement at ~1e-9 here.
    assert rel_l2(sites["psfs"], d["f64_psf_3d"]) < 1e-8
    assert rel_l2(sites["psfs"].sum((1, 2, 3)), d["f64_energies"]) < 1e-8


def test_numerics():
    d = golden("numerics")
    a = d["resize_in"]
    for s in (2, 0.5, 3):
        assert rel_l2(O.resize_xy(a, s), d[f"resize_{s}"]) < 1e-6
        assert rel_l2(O.resize_xy(a.astype(np.float64), s), d[f"resize64_{s}"]) < 1e-14
    for sh in (0.5, 1.0, 0.0):
        np.testing.assert_allclose(O.translate_xy(a.astype(np.float64), sh), d[f"translate_{sh}"], atol=1e-12)
    np.testing.assert_allclose(O.edge_apodization(64, np.float64), d["edge_64"], rtol=1e-14)
    np.testing.assert_allclose(O.edge_apodization(64, np.float32), d["edge_32"], rtol=5e-7)  # 1-2 ulp (powf)
    from types import SimpleNamespace
    cfg = SimpleNamespace(scaling="temporal-focusing", vres=1.0, prop_um=5.0, psf_um=(8.0, 8.0, 10.0),
                          temporal_length_um=10.0)
    for part, size in (("focus", 20), ("top", 7), ("bottom", 5)):
        np.testing.assert_allclose(O.axial_profile(cfg, size, part), d[f"axial_{part}"], rtol=1e-7)
    np.testing.assert_allclose(O.v4_interpolate(d["v4_points"], d["v4_values"], d["v4_queries"]), d["v4_out"],
                               rtol=1e-9, atol=1e-10)
    lq = np.stack(np.meshgrid(np.arange(64) + .5, np.arange(64) + .5, indexing="ij"), -1)
    np.testing.assert_allclose(O.v4_interpolate(d["v4l_points"], d["v4l_values"], lq), d["v4l_out"], rtol=1e-9,
                               atol=1e-10)


def test_zernike_pupil():
    d = golden("numerics")
    cfg = cfg_from(d, "zcfg_")
    assert rel_l2(O.pupil(cfg, np.float64), d["zpupil64"]) < 1e-13
    assert rel_l2(O.pupil(cfg, np.float32), d["zpupil32"]) < 1e-6


def test_resample_matrix_composes_resize_and_translate():
    """native.py:27-48 composes translate_xy and resize_xy into one operator."""
    rng = np.random.default_rng(3)
    for n, ss in ((40, 2), (24, 3), (20, 1)):
        img = rng.standard_normal((n, n))
        mx = O.resample_matrix(n, ss)
        ref = O.resize_xy(O.translate_xy(img, ss / 2 - 0.5), 1 / ss)
        np.testing.assert_allclose(mx @ img @ mx.T, ref, atol=1e-12)
