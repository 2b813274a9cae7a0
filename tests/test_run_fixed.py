"""``run_fixed`` as a drop-in for maomi/fixed.py:193-411, and the collection
mask (maomi/optics.py:384-409).

CPU: the collection-mask oracle against the reference's own outputs.  GPU:
every branch of ``run_fixed`` against the oracle stage (``propagate``, FP64)
and the oracle static scan, at the stage tolerance (1e-5 relative L2).
"""

import numpy as np
import pytest

from conftest import cfg_from, golden, rel_l2

TOL = 1e-5


def test_oracle_collection_mask_pin():
    from oracle import optics as O
    d = golden("collection")
    for i in range(2):
        cfg = cfg_from(d, prefix=f"c{i}_cfg_")
        got = O.collection_mask(d[f"c{i}_vessels"].astype(np.float64), cfg)
        # the reference evaluates in float32
        assert rel_l2(got, d[f"c{i}_colmask"]) < 1e-6


def test_collection_disk_geometry_matches_oracle():
    from oracle import optics as O
    from maomi_b200.optics import _collection_disks
    d = golden("collection")
    for i in range(2):
        cfg = cfg_from(d, prefix=f"c{i}_cfg_")
        shape = d[f"c{i}_vessels"].shape
        for (s0, a), (s1, b) in zip(_collection_disks(cfg, shape), O.collection_disks(cfg, shape)):
            assert s0 == s1 and (a is None) == (b is None)
            if a is not None:
                np.testing.assert_allclose(a, b, rtol=1e-6)


# ------------------------------------------------------------------ GPU
def _oracle_stage(cfg, raw, pts):
    from oracle import optics as O
    return O.propagate(cfg, [np.asarray(a, np.float64) for a in raw], pts, O.pupil(cfg, np.float64))


def _assert_stage(out, ref, tails=True):
    keys = ["psf_3d", "psf", "psf_raw", "mask_raw", "energies"]
    errs = {k: rel_l2(out[k], ref[k]) for k in keys}
    if tails:
        for t in ("psfT", "psfB"):
            for k in ("convmask", "weight", "psfZ", "mask_raw"):
                errs[f"{t}.{k}"] = rel_l2(out[t][k], ref[t][k])
    bad = {k: v for k, v in errs.items() if not v < TOL}
    assert not bad, errs


@pytest.fixture(scope="module")
def vessel_case():
    """Small benchmark-recipe geometry with a vessel occupancy volume; raw
    fields from the reference's vessel-aware generator (no scatter)."""
    d = golden("collection")
    cfg = cfg_from(d, prefix="c1_cfg_")
    raw = [d[f"c1_raw{j}"] for j in range(3)]
    vol = np.random.default_rng(21).uniform(0, 1, tuple(int(v) for v in np.round(
        np.asarray(cfg.volume_um) * cfg.vres))).astype(np.float32)
    return d, cfg, raw, vol


@pytest.mark.gpu
def test_collection_mask_gpu():
    import torch
    from maomi_b200.optics import collection_mask
    d = golden("collection")
    for i in range(2):
        cfg = cfg_from(d, prefix=f"c{i}_cfg_")
        ves = d[f"c{i}_vessels"].astype(np.float32)
        got = collection_mask(ves, cfg)
        assert isinstance(got, np.ndarray) and got.dtype == np.float32
        assert rel_l2(got, d[f"c{i}_colmask"]) < TOL
        dev = collection_mask(torch.as_tensor(ves, device="cuda"), cfg)
        assert dev.is_cuda and rel_l2(dev.cpu().numpy(), d[f"c{i}_colmask"]) < TOL


@pytest.mark.gpu
def test_vessel_fields_match_reference():
    """Scatter-free fields are the vessel occupancies (optics.py:176-197)."""
    from maomi_b200.fields import prepare_fields
    d = golden("collection")
    for i in range(2):
        cfg = cfg_from(d, prefix=f"c{i}_cfg_")
        raw = prepare_fields(cfg, d[f"c{i}_vessels"].astype(np.float32), scatter=False)
        for j in range(3):
            np.testing.assert_allclose(raw[j].cpu().numpy(), d[f"c{i}_raw{j}"], rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
def test_run_fixed_with_vessels_and_image(vessel_case):
    """Supplied raw fields, vessels -> collection mask, the static image."""
    from oracle import scanning as S
    from maomi_b200.fixed import fixed_locations, run_fixed
    d, cfg, raw, vol = vessel_case
    ves = d["c1_vessels"].astype(np.float32)
    out = run_fixed(cfg, vol, vessels=ves, raw_fields=raw, count_per_axis=3, batch_size=4)
    ref = _oracle_stage(cfg, raw, fixed_locations(cfg, 3))
    _assert_stage(out, ref)
    assert rel_l2(out["colmask"], d["c1_colmask"]) < TOL
    img = S.zstack(vol, ref["psf"].astype(np.float32), mask=ref["mask"], collection_mask=d["c1_colmask"])
    assert out["image"].shape == vol.shape and rel_l2(out["image"], img) < TOL
    assert out["settings"]["fields"] == "provided" and out["settings"]["collection_absorption"]
    assert set(out["timing_seconds"]) >= {"plan", "static_scan"}


@pytest.mark.gpu
def test_run_fixed_generates_fields(vessel_case):
    """raw_fields=None generates them on the device; without scatter they are
    the vessel occupancies, so the stage equals the supplied-fields run."""
    from maomi_b200.fixed import run_fixed
    d, cfg, raw, vol = vessel_case
    ves = d["c1_vessels"].astype(np.float32)
    gen = run_fixed(cfg, vol, vessels=ves, scatter=False, count_per_axis=3, batch_size=4)
    sup = run_fixed(cfg, vol, vessels=ves, raw_fields=raw, count_per_axis=3, batch_size=4)
    for k in ("psf_3d", "mask_raw", "image"):
        assert rel_l2(gen[k], sup[k]) < 1e-6, k
    assert gen["settings"]["fields"] == "generated" and gen["settings"]["scatter"] is False
    scat = run_fixed(cfg, vol, vessels=ves, count_per_axis=3, batch_size=4, render_image=False)
    assert "image" not in scat and np.isfinite(scat["psf_3d"]).all()
    assert rel_l2(scat["psf_3d"], gen["psf_3d"]) > 1e-4  # scattering screens were drawn


@pytest.mark.gpu
def test_run_fixed_focal_only_keeps_image(vessel_case):
    """tails=False drops the tail products but not the focal image
    (tests/test_fixed.py:111-116 of the reference)."""
    from maomi_b200.fixed import run_fixed
    d, cfg, raw, vol = vessel_case
    full = run_fixed(cfg, vol, raw_fields=raw, count_per_axis=3, batch_size=4)
    focal = run_fixed(cfg, vol, raw_fields=raw, count_per_axis=3, batch_size=4, tails=False)
    assert not focal["tails_computed"] and "psfT" not in focal
    # equal up to the order of the FP64 site-sum atomics behind the mean PSF
    assert rel_l2(focal["image"], full["image"]) < 1e-12
    assert np.all(full["colmask"] == 1)


@pytest.mark.gpu
def test_run_fixed_multibeam(vessel_case):
    """Dict pupils are incoherent channels on shared fields; the image is the
    weighted sum of the channel images (fixed.py:237-285)."""
    from maomi_b200.fixed import run_fixed
    from maomi_b200.optics import pupil
    d, cfg, raw, vol = vessel_case
    u = pupil(cfg).cpu().numpy()
    beams = {"a": u, "b": (u * np.exp(0.3j * np.linspace(0, 1, u.size).reshape(u.shape))).astype(np.complex64)}
    w = {"a": 0.25, "b": 1.5}
    out = run_fixed(cfg, vol, raw_fields=raw, input_pupil=beams, beam_weights=w, count_per_axis=3, batch_size=4)
    assert set(out["channels"]) == {"a", "b"} and out["unique_optical_paths"] == 18
    one = run_fixed(cfg, vol, raw_fields=raw, input_pupil=beams["b"], count_per_axis=3, batch_size=4)
    np.testing.assert_allclose(out["channels"]["b"]["psf_3d"], one["psf_3d"], rtol=0, atol=0)
    img = w["a"] * out["channels"]["a"]["image"] + w["b"] * out["channels"]["b"]["image"]
    np.testing.assert_allclose(out["image"], img, rtol=1e-6)
    with pytest.raises(ValueError, match="Nonnegative"):
        run_fixed(cfg, vol, raw_fields=raw, input_pupil=beams, beam_weights={"a": -1.0, "b": 1.0})
    with pytest.raises(ValueError, match="Compose"):
        run_fixed(cfg, vol, raw_fields=raw, input_pupil=beams, custom_phase=np.zeros((3, 3)))


@pytest.mark.gpu
def test_run_fixed_argument_errors(vessel_case):
    from maomi_b200.fixed import run_fixed
    d, cfg, raw, vol = vessel_case
    with pytest.raises(ValueError, match="finite volume"):
        run_fixed(cfg, vol[:-1], raw_fields=raw)
    with pytest.raises(ValueError, match="shapes"):
        run_fixed(cfg, vol, raw_fields=raw[:2])
    with pytest.raises(ValueError, match="batch_size"):
        run_fixed(cfg, vol, raw_fields=raw, batch_size=0)
    with pytest.raises(ValueError, match="optical grid"):
        run_fixed(cfg, vol, raw_fields=raw, input_pupil=np.zeros((4, 4), np.complex64))
    with pytest.raises(ValueError, match="matlab_v4"):
        run_fixed(cfg, vol, raw_fields=raw, mask_mode="cubic")
