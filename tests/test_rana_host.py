"""Host side of the local-PSF renderer (no GPU): file formats against files the
reference wrote, the bank contracts, the lateral tile tables of
``mm_local_tiles`` and the operator's weights and kernel transforms."""

import numpy as np
import pytest

from conftest import GOLDEN, golden
from oracle import local_fft as L


def test_full_field_file_written_by_the_reference_loads_and_round_trips(tmp_path):
    from maomi_b200.rana import FullFieldPSF
    d = golden("rana_files")
    f = FullFieldPSF.load(GOLDEN / "ref_full_field_psf.npz")
    np.testing.assert_array_equal(f.kernels, d["field_kernels"])
    np.testing.assert_array_equal(f.x_um, d["x_um"])
    np.testing.assert_array_equal(f.y_um, d["y_um"])
    assert f.voxel_size_um == (0.5, 0.5, 1.0) and f.wavelength_nm == 920.0 and f.operator == "excitation"
    assert f.provenance == {"note": "reference-written", "n": 3}
    f.save(tmp_path / "ours.npz")
    with np.load(GOLDEN / "ref_full_field_psf.npz") as ref, np.load(tmp_path / "ours.npz") as ours:
        assert sorted(ref.files) == sorted(ours.files)
        for k in ref.files:
            np.testing.assert_array_equal(ours[k], ref[k], err_msg=k)
            assert ours[k].dtype == ref[k].dtype, k


def test_depth_bank_file_written_by_the_reference_loads_and_round_trips(tmp_path):
    from maomi_b200.rana import DepthPSFBank
    d = golden("rana_files")
    b = DepthPSFBank.load(GOLDEN / "ref_depth_psf_bank.npz")
    np.testing.assert_array_equal(b.depths_um, [1.0, 9.0])
    for i, f in enumerate(b.fields):
        np.testing.assert_array_equal(f.kernels, d["bank_kernels"][i])
        assert f.provenance == {"depth": i} and f.operator == "detection"
    assert b.operator == "detection" and b.voxel_size_um == (0.5, 0.5, 1.0)
    b.save(tmp_path / "ours.npz")
    with np.load(GOLDEN / "ref_depth_psf_bank.npz") as ref, np.load(tmp_path / "ours.npz") as ours:
        assert sorted(ref.files) == sorted(ours.files)
        for k in ref.files:
            np.testing.assert_array_equal(ours[k], ref[k], err_msg=k)


def test_field_contract_rejections():
    from maomi_b200.rana import FullFieldPSF
    k = np.ones((2, 2, 3, 3, 3))
    ok = dict(x_um=[0, 1], y_um=[0, 1], voxel_size_um=(1, 1, 1), wavelength_nm=920., operator="excitation")
    FullFieldPSF(k, **ok)
    bad = [({"kernels": k * 1j}, ValueError), ({"kernels": -k}, ValueError), ({"kernels": k * np.nan}, ValueError),
           ({"kernels": np.zeros_like(k)}, ValueError), ({"kernels": k[:1]}, ValueError),
           ({"x_um": [1, 0]}, ValueError), ({"x_um": [0]}, ValueError), ({"voxel_size_um": (1, 1)}, ValueError),
           ({"voxel_size_um": (1, 0, 1)}, ValueError), ({"wavelength_nm": -1.}, ValueError),
           ({"operator": "both"}, ValueError), ({"provenance": {"x": float("nan")}}, ValueError)]
    for change, exc in bad:
        args = dict(ok, kernels=k)
        args.update(change)
        with pytest.raises(exc):
            FullFieldPSF(**args)
    f = FullFieldPSF(k, **ok)
    with pytest.raises(ValueError):
        f.kernels[0, 0, 0, 0, 0] = 2.0   # frozen arrays


def test_field_builders():
    from maomi_b200.rana import DepthPSFBank, FullFieldPSF
    from types import SimpleNamespace
    f = FullFieldPSF.from_provider(lambda x, y: np.full((3, 3, 2), 1.0 + x + 10 * y), [0, 1], [0, 2, 3],
                                   voxel_size_um=(1, 1, 1), wavelength_nm=900., operator="detection")
    assert f.kernels.shape == (2, 3, 3, 3, 2) and f.kernels[1, 2, 0, 0, 0] == 1 + 1 + 30
    b = DepthPSFBank.from_provider(lambda x, y, z: np.full((3, 3, 2), 1.0 + z), [0, 1], [0, 1], [2.0, 5.0],
                                   voxel_size_um=(1, 1, 1), wavelength_nm=900.)
    assert b.fields[1].kernels[0, 0, 0, 0, 0] == 6.0 and b.fields[1].provenance["focal_depth_um"] == 5.0
    psf = SimpleNamespace(intensity=np.full((2, 2, 3, 3), 1 / 9), x_um=[0, 1], y_um=[0, 1], pixel_size_um=(1, 1),
                          wavelength_nm=900., provenance={"id": 1})
    g = FullFieldPSF.from_psf_field(psf, operator="excitation", gains=[[1, 2], [3, 4]])
    np.testing.assert_allclose(g.kernels.sum((2, 3)), [[1, 2], [3, 4]])
    assert g.provenance["gain_source"] == "explicit node gains"
    with pytest.raises(TypeError):
        FullFieldPSF.from_psf_field(np.ones((3, 3)), operator="excitation")
    with pytest.raises(ValueError):
        DepthPSFBank([0.0, 1.0], (f,))


def _tiles_reference(w, max_len=18):
    """Plain restatement of the tiling rule: runs of equal active sets, split evenly."""
    active = [tuple(np.flatnonzero(w[:, x])) for x in range(w.shape[1])]
    tiles, a = [], 0
    while a < len(active):
        b = a
        while b < len(active) and active[b] == active[a]:
            b += 1
        n = b - a
        pieces = -(-n // max_len)
        for k in range(pieces):
            s, e = a + n * k // pieces, a + n * (k + 1) // pieces
            if active[a]:
                tiles.append((s, e - s, active[a]))
        a = b
    return tiles


@pytest.mark.parametrize("nodes,n", [(np.linspace(0, 256, 16), 256), (np.linspace(0, 64, 4), 64),
                                     (np.array([0., 1.5, 2.0, 9.0, 40.0]), 40), (np.linspace(0, 12, 7), 12)])
def test_lateral_tiles_partition_the_axis(nodes, n):
    from maomi_b200.rana._fft import lateral_tiles
    from maomi_b200.rana.operator import _axis_weights
    w = _axis_weights(nodes, np.arange(n) + 0.5)
    t = lateral_tiles(w)
    expect = _tiles_reference(w)
    assert len(t) == len(expect)
    for rec, (s, ln, act) in zip(t, expect):
        assert (rec[0], rec[1], rec[2]) == (s, ln, len(act)) and tuple(rec[3:3 + rec[2]]) == act
        assert 1 <= rec[1] <= 18
    covered = np.zeros(n, int)
    for rec in t:
        covered[rec[0]:rec[0] + rec[1]] += 1
    assert (covered == 1).all()


def test_lateral_tiles_reject_dense_weights():
    from maomi_b200 import _lib
    from maomi_b200.rana._fft import lateral_tiles
    with pytest.raises(ValueError, match="more than 4"):
        lateral_tiles(np.ones((5, 10)))
    assert _lib.load().mm_local_tiles(None, 2, 4, 0, None, 0) == _lib.MM_ERR_ARGUMENT


def test_operator_weights_and_kernel_transforms_match_the_oracle():
    from maomi_b200.rana.depth import depth_weights
    from maomi_b200.rana.operator import _axis_weights, _bin_planes, _mirror_depth
    d = golden("local_fft")
    np.testing.assert_allclose(_axis_weights(d["c_nodes"], d["c_pos"]), d["c_weights"], rtol=0, atol=1e-15)
    z = np.linspace(0.5, 9.5, 10)
    np.testing.assert_allclose(depth_weights([0.0, 4.0, 10.0], z), L.depth_weights(np.array([0.0, 4.0, 10.0]), z),
                               rtol=0, atol=1e-15)
    k = np.arange(2 * 9, dtype=float).reshape(2, 9)
    ids = 2 * 4 - np.arange(9)
    ref = np.take(k, np.minimum(ids, 8), axis=-1)
    ref[..., ids >= 9] = 0
    np.testing.assert_array_equal(_mirror_depth(k, 4), ref)
    k4 = np.arange(8, dtype=float).reshape(2, 4)
    ref4 = np.take(k4, np.minimum(2 * 2 - np.arange(4), 3), axis=-1)
    ref4[..., 2 * 2 - np.arange(4) >= 4] = 0
    np.testing.assert_array_equal(_mirror_depth(k4, 2), ref4)
    np.testing.assert_array_equal(_bin_planes(k, 4), np.add.reduceat(k, np.arange(0, 9, 4), axis=-1))


def test_physical_tail_keeps_the_integrated_gain():
    from maomi_b200.rana import RanaOperator
    a = np.array([[1.0, -0.2], [0.5, 0.7]])
    out = RanaOperator.physical_tail(a)
    assert (out >= 0).all() and np.isclose(out.sum(), a.sum())
    b = np.array([1.0, 2.0])
    assert RanaOperator.physical_tail(b) is b
    for bad in (np.array([1j]), np.array([np.nan]), np.array([-1.0, 0.5])):
        with pytest.raises(ValueError):
            RanaOperator.physical_tail(bad)
