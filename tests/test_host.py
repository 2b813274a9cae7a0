"""Host-side logic (no GPU): geometry, tables, validation and the C ABI surface."""

import re
from pathlib import Path

import numpy as np
import pytest

from conftest import REPO, cfg_from, golden, rel_l2
from oracle import optics as O
from maomi_b200 import synthetic
from maomi_b200._propagation import center_slice, edge_window_1d, geometry
from maomi_b200.backends.cuda.batched import transfer_kernels, trapezoid
from maomi_b200.excitation import axial_profile, excitation_order, temporal_profile
from maomi_b200.fixed import field_shapes, fixed_locations
from maomi_b200.numerics import is_identity_table, resample_matrix, resize_table, sparse_rows
from maomi_b200.optics import OpticalConfig, locations


def _configs():
    yield synthetic.small_stage_config(OpticalConfig)
    yield synthetic.benchmark_stage_config(OpticalConfig)
    yield OpticalConfig(volume_um=(16.0, 16.0, 10.0), depth_um=20.0, tail_um=10.0)
    yield OpticalConfig()


@pytest.mark.parametrize("cfg", list(_configs()))
def test_geometry_matches_oracle(cfg):
    shapes = field_shapes(cfg)
    assert shapes == O.field_shapes(cfg)
    raw = [np.zeros((1, 1, s[2])) for s in shapes]
    g, go = geometry(cfg, raw), O.geometry(cfg, [s for s in shapes])
    for k in ("n", "n2", "fl", "d1", "d2", "wvl", "nr", "cut"):
        assert getattr(g, k) == getattr(go, k), k
    for a, b in zip(g.z, go.z):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(g.focal_shape, go.focal_shape)
    assert g.crop == go.crop and g.focal_crop == go.focal_crop


def test_benchmark_geometry_numbers():
    cfg = synthetic.benchmark_stage_config(OpticalConfig)
    shapes = field_shapes(cfg)
    assert shapes == [(768, 768, 10), (768, 768, 46), (768, 768, 4)]
    g = geometry(cfg, [np.zeros(s[2]) for s in shapes])
    assert (g.n, g.n2, g.cut) == (256, 256, 6)
    assert [len(z) - 1 for z in g.z] == [10, 46, 4]
    assert tuple(g.focal_shape) == (40, 40)
    pts = fixed_locations(cfg)
    assert pts.shape == (4225, 2) and len(np.unique(pts, axis=0)) == 4225
    np.testing.assert_array_equal(pts.max(0), [256, 256])


def test_fixed_locations_contract():
    cfg = OpticalConfig(volume_um=(16.0, 24.0, 10.0), vres=2.0)
    p = fixed_locations(cfg, 32)
    assert p.shape == (1024, 2) and len(np.unique(p, axis=0)) == 1024
    np.testing.assert_allclose(p * 4, np.round(p * 4))
    np.testing.assert_array_equal(fixed_locations(cfg, 32), O.fixed_locations(cfg, 32))
    for bad in (1, 3.5, True):
        with pytest.raises(ValueError):
            fixed_locations(cfg, bad)
    with pytest.raises(ValueError):
        fixed_locations(OpticalConfig(volume_um=(4.0, 4.0, 4.0)))
    np.testing.assert_array_equal(locations((16.0, 16.0, 10.0), 1), [[8, 8]])


def test_excitation_tables():
    for mode, order in (("one-photon", 1), ("two-photon", 2), ("three-photon", 3), ("temporal-focusing", 2)):
        cfg = OpticalConfig(scaling=mode)
        assert excitation_order(cfg) == order
        for part, size in (("focus", 11), ("top", 5), ("bottom", 4)):
            np.testing.assert_array_equal(axial_profile(cfg, size, part), O.axial_profile(cfg, size, part))
    with pytest.raises(ValueError):
        excitation_order(OpticalConfig(scaling="four-photon"))
    with pytest.raises(ValueError):
        temporal_profile(0, 1.0, 1.0)
    with pytest.raises(ValueError):
        OpticalConfig(temporal_length_um=-1).parameters()


def test_resize_tables_and_resample_matrix():
    for n, s in ((20, 2), (18, 0.5), (31, 3), (16, 1)):
        idx, w = resize_table(n, s)
        io, wo = O.resize_plan(n, s)
        np.testing.assert_array_equal(idx, io)
        np.testing.assert_allclose(w, wo, rtol=1e-15)
        assert is_identity_table(idx, w) == (s == 1)
    for n, ss in ((40, 2), (72, 2), (25, 3), (40, 1)):
        np.testing.assert_allclose(resample_matrix(n, ss), O.resample_matrix(n, ss), rtol=1e-15)
        ix, wx = sparse_rows(resample_matrix(n, ss))
        dense = np.zeros((ix.shape[0], n))
        for i in range(ix.shape[0]):
            np.add.at(dense[i], ix[i], wx[i])
        np.testing.assert_allclose(dense, resample_matrix(n, ss), rtol=1e-6)


def test_edge_window_matches_reference():
    d = golden("numerics")
    e = edge_window_1d(64)
    np.testing.assert_allclose(e[:, None] * e[None, :], d["edge_64"], rtol=3e-7)


@pytest.mark.parametrize("size", [64, 128, 256])
def test_separable_transfer_function(size):
    """The 1-D FFT-order kernels reproduce the reference's 2-D transfer function
    ifftshift(exp(-i pi (wvl/nr) dz (fx^2+fy^2))) (batched.py:68-82) and carry 1/size."""
    cfg = synthetic.benchmark_stage_config(OpticalConfig)
    g = geometry(cfg, [np.zeros(s[2]) for s in field_shapes(cfg)])
    z = g.z[0]
    q = transfer_kernels(z, size, g.d2, g.wvl, g.nr).astype(np.complex128) * size
    x = np.arange(-size / 2, size / 2)
    lam = float(g.wvl) / float(g.nr)
    for i, dz in enumerate(np.diff(z)):
        f2 = (x / (size * float(g.d2))) ** 2
        ref = np.fft.ifftshift(np.exp(-1j * np.pi * lam * dz * (f2[:, None] + f2[None, :])))
        assert rel_l2(np.outer(q[i], q[i]), ref) < 1e-6


def test_trapezoid():
    np.testing.assert_array_equal(trapezoid(5), [.5, 1, 1, 1, .5])
    np.testing.assert_array_equal(trapezoid(1), [.25])


def test_center_slice():
    assert center_slice(256, 40) == slice(108, 148)
    with pytest.raises(ValueError):
        center_slice(10, 5)


def test_header_symbols_exported():
    """Every entry point declared in include/maomi_b200.h is bound and exported."""
    from maomi_b200 import _lib
    header = (REPO / "include" / "maomi_b200.h").read_text()
    declared = set(re.findall(r"^\s*(?:int|size_t|const char\*|unsigned long long)\s+(mm_\w+)\s*\(", header, re.M))
    assert declared, "no declarations found"
    assert declared <= set(_lib.SIGNATURES), declared - set(_lib.SIGNATURES)
    lib = _lib.load()
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.mm_version() >= 100


def test_descriptor_layouts_match_the_library():
    """The ctypes records bind the C structs byte for byte (sizes agree)."""
    import ctypes
    from maomi_b200 import _lib
    lib = _lib.load()
    for name, cls in (("mm_stage_desc", _lib.StageDesc), ("mm_stage_plan", _lib.StagePlan),
                      ("mm_item_class", _lib.ItemClass), ("mm_pupil_desc", _lib.PupilDesc),
                      ("mm_base_desc", _lib.BaseDesc), ("mm_local_desc", _lib.LocalDesc),
                      ("mm_surrogate_desc", _lib.SurrogateDesc), ("mm_scan_planes", _lib.ScanPlanes),
                      ("mm_scan_desc", _lib.ScanDesc), ("mm_scan_conv", _lib.ScanConv)):
        assert lib.mm_struct_size(name.encode()) == ctypes.sizeof(cls), name
    assert lib.mm_struct_size(b"nothing") == 0


def test_status_mapping():
    from maomi_b200 import _lib
    _lib.check(0)
    with pytest.raises(ValueError):
        _lib.check(_lib.MM_ERR_ARGUMENT, "x")
    with pytest.raises(ValueError):
        _lib.check(_lib.MM_ERR_UNSUPPORTED, "x")
    with pytest.raises(RuntimeError):
        _lib.check(_lib.MM_ERR_CUDA, "x")
    with pytest.raises(RuntimeError):
        _lib.check(_lib.MM_ERR_TIMEOUT, "x")


def test_product_refuses_cpu():
    """No CPU fallback: the product path raises instead of computing on the host."""
    from maomi_b200.backends.cuda.batched import OpticalPlan
    from maomi_b200.fixed import run_fixed
    cfg = synthetic.small_stage_config(OpticalConfig)
    raw = [np.zeros(s, np.float32) for s in field_shapes(cfg)]
    with pytest.raises(ValueError):
        OpticalPlan(cfg, raw, device="cpu")
    with pytest.raises(ValueError, match="requires CUDA"):
        run_fixed(cfg, raw_fields=raw, device="cpu")
    with pytest.raises(ValueError, match="requires CUDA"):
        run_fixed(cfg, device="cpu", render_image=False)
    with pytest.raises(ValueError, match="beam"):
        run_fixed(cfg, input_pupil={}, device="cpu")
    with pytest.raises(ValueError, match="mapping"):
        run_fixed(cfg, beam_weights={"a": 1.0}, device="cpu")


def test_lattice_index_detects_symmetric_lattices():
    from maomi_b200.numerics import lattice_index
    xs, ys = np.arange(5) * 8.0, np.arange(4) * 8.0 + 2.0
    pts = np.array([(x, y) for x in xs for y in ys])
    perm = np.random.default_rng(0).permutation(len(pts))
    nx, ny, idx = lattice_index(pts[perm])
    assert (nx, ny) == (5, 4)
    np.testing.assert_array_equal(pts[perm][idx], pts)
    assert lattice_index(pts[:-1]) is None                       # incomplete
    bent = pts.copy()
    bent[pts[:, 0] == 32.0, 0] = 33.0                            # not symmetric
    assert lattice_index(bent) is None
    assert lattice_index(np.array([[0.0, 0.0], [1.0, 0.0]])) is None  # one row

