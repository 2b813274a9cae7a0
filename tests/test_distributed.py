"""Sharded-stage host logic on two gloo ranks (CPU).

Each rank computes its band of sites with the CPU oracle (standing in for the
GPU propagation of that band), then ``assemble_sharded`` all-gathers the
per-site rows, all-reduces the PSF and tail sums and solves the v4 masks; the
result must equal the single-process oracle stage."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import golden, cfg_from, rel_l2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    import torch
    import torch.distributed as dist
    from conftest import golden, cfg_from
    from oracle import optics as O
    from maomi_b200 import synthetic
    from maomi_b200.distributed import assemble_sharded, shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = golden("stage_small")
        cfg = cfg_from(d)
        raw = synthetic.raw_fields(cfg, O.field_shapes(cfg), sigma=float(d["raw_sigma"]), rms=float(d["raw_rms"]),
                                   seed=int(d["raw_seed"]))
        raw = [np.asarray(a, np.float64) for a in raw]
        pts = d["points"]
        lo, hi = shard(len(pts), rank, world)
        u = O.pupil(cfg, np.float64)
        band = O.propagate_sites(cfg, raw, pts[lo:hi], u)
        t = lambda a: torch.as_tensor(np.asarray(a, np.float64))
        parts = {"energies": t(band["psfs"].sum((1, 2, 3))), "profiles": [t(p) for p in band["profiles"]],
                 "psf_sum": t(band["psfs"].sum(0)), "psf_abs_sum": t(np.abs(band["psfs"]).sum(0)),
                 "tail_sum": [t(c.sum(0)) for c in band["convmasks"]]}
        g = band["geometry"]

        def solve(points, values, shape):
            q = np.stack(np.meshgrid(*[np.arange(k) + 0.5 for k in shape], indexing="ij"), -1)
            return O.v4_interpolate(points, values, q)

        res = assemble_sharded(cfg, parts, len(pts), points_um=pts, z_positions=g.z, cut=g.cut, solve=solve)
        np.savez(f"{out_dir}/rank{rank}.npz", psf=res["psf"], mask_raw=res["mask_raw"], energies=res["energies"],
                 convT=res["psfT"]["convmask"], convB=res["psfB"]["convmask"], psfZT=res["psfT"]["psfZ"],
                 wB=res["psfB"]["weights_per_point"])
    finally:
        dist.destroy_process_group()


def test_sharded_stage_two_gloo_ranks(tmp_path):
    from oracle import optics as O
    from maomi_b200 import synthetic
    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    d = golden("stage_small")
    cfg = cfg_from(d)
    raw = synthetic.raw_fields(cfg, O.field_shapes(cfg), sigma=float(d["raw_sigma"]), rms=float(d["raw_rms"]),
                               seed=int(d["raw_seed"]))
    ref = O.propagate(cfg, [np.asarray(a, np.float64) for a in raw], d["points"], O.pupil(cfg, np.float64))
    for rank in range(2):
        got = np.load(tmp_path / f"rank{rank}.npz")
        assert rel_l2(got["psf"], ref["psf"]) < 1e-12
        assert rel_l2(got["mask_raw"], ref["mask_raw"]) < 1e-12
        assert rel_l2(got["energies"], ref["energies"]) < 1e-12
        assert rel_l2(got["convT"], ref["psfT"]["convmask"]) < 1e-12
        assert rel_l2(got["convB"], ref["psfB"]["convmask"]) < 1e-12
        assert rel_l2(got["psfZT"], ref["psfT"]["psfZ"]) < 1e-12
        assert rel_l2(got["wB"], ref["psfB"]["weights_per_point"]) < 1e-12


def test_shard_bands_cover_sites():
    from maomi_b200.distributed import shard
    for count in (1, 9, 4225):
        for world in (1, 2, 3, 8):
            bands = [shard(count, r, world) for r in range(world)]
            assert bands[0][0] == 0 and bands[-1][1] == count
            assert all(a[1] == b[0] for a, b in zip(bands, bands[1:]))
            assert max(b - a for a, b in bands) - min(b - a for a, b in bands) <= 1
    with pytest.raises(ValueError):
        shard(10, 2, 2)
