"""The sharded stage on one GPU: band-only uploads and a one-rank NCCL group.

A band of sites computed from only the raw rows it reads must equal the same
sites of the whole-block stage; ``run_stage_sharded`` over a one-rank NCCL
group (all-gathers, all-reduces and the device v4 solve) must equal
``run_stage``.  The host combine logic over two ranks is covered on CPU by
tests/test_distributed.py.
"""

import socket

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _case():
    from oracle import optics as O
    from maomi_b200 import synthetic
    from maomi_b200.fixed import fixed_locations
    from maomi_b200.optics import OpticalConfig
    cfg = synthetic.small_stage_config(OpticalConfig)
    raw = synthetic.raw_fields(cfg, O.field_shapes(cfg), sigma=2.0, rms=0.01, seed=5)
    return cfg, raw, fixed_locations(cfg, 5)


def test_band_window_rows():
    from maomi_b200.distributed import band_window
    cfg, raw, pts = _case()
    rows, local = band_window(cfg, pts[5:15], (128, 96, 128))
    x0 = np.round(pts[5:15, 0] * cfg.vres).astype(int)
    assert rows[0] == (x0.min(), x0.max() + 128) and rows[1] == (x0.min(), x0.max() + 96)
    np.testing.assert_allclose(local[:, 1], pts[5:15, 1])
    assert np.round(local[:, 0] * cfg.vres).min() == 0


def test_band_upload_matches_whole_block():
    import torch
    from maomi_b200.distributed import band_stage
    from maomi_b200.fixed import run_stage
    cfg, raw, pts = _case()
    full = run_stage(cfg, raw, pts, slots=8)
    dev = band_stage(cfg, raw, pts[5:15], device="cuda", slots=4)
    assert dev["masks"] is None
    band_rows = dev["plan"].phases[0].shape[1]
    assert band_rows < raw[0].shape[0]  # only the rows the band reads were prepared
    np.testing.assert_array_equal(dev["psf_3d"].cpu().numpy(), full["psf_3d"][5:15])
    assert rel_l2(dev["energies"].cpu().numpy(), full["energies"][5:15]) < 1e-12
    for j, t in enumerate(("psfT", "psfB")):
        assert rel_l2(dev["profiles"][j].cpu().numpy(), full[t]["profiles_per_point"][5:15]) < 1e-12
    torch.cuda.synchronize()


@pytest.fixture
def one_rank_nccl():
    import torch
    import torch.distributed as dist
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    from datetime import timedelta
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60), device_id=torch.device("cuda:0"))
    try:
        yield dist.group.WORLD
    finally:
        dist.destroy_process_group()


def test_sharded_stage_one_rank_matches_run_stage(one_rank_nccl):
    from maomi_b200.distributed import run_stage_sharded
    from maomi_b200.fixed import run_stage
    cfg, raw, pts = _case()
    ref = run_stage(cfg, raw, pts, slots=8)
    got = run_stage_sharded(cfg, raw, pts, group=one_rank_nccl, slots=8)
    lo, hi, psf3d = got["psf_3d_band"]
    assert (lo, hi) == (0, len(pts))
    np.testing.assert_array_equal(psf3d.cpu().numpy(), ref["psf_3d"])
    for k in ("psf", "psf_raw", "mask_raw", "mask", "energies"):
        assert rel_l2(got[k], ref[k]) < 1e-12, k
    for t in ("psfT", "psfB"):
        for k in ("convmask", "weight", "psfZ", "mask_raw", "weights_per_point", "profiles_per_point"):
            assert rel_l2(got[t][k], ref[t][k]) < 1e-12, (t, k)
