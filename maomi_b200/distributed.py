"""One tissue block sharded over several GPUs (one process per GPU).

Sites are independent, so each rank propagates a contiguous band of the
site list; the only exchange is small: per-site energies, tail weights and
profiles are all-gathered, the PSF sums and tail images all-reduced, and the
v4 mask is then solved and evaluated on every rank.  ``psf_3d`` stays
sharded (each rank keeps its band).  The collectives run over the process
group given (NCCL on GPUs; any backend for the host logic).
"""

import numpy as np


def shard(count, rank, world):
    """Contiguous [lo, hi) band of `count` sites for `rank` of `world`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(count, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_sites(local, count, group=None):
    """All-gather per-site rows (band of this rank, any trailing shape) into
    the full (count, ...) array on every rank.  `local` is a torch tensor."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = shard(count, rank, world)
    if local.shape[0] != hi - lo:
        raise ValueError(f"rank {rank} holds {local.shape[0]} sites, its band is {hi - lo}")
    width = -(-count // world)
    pad = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:hi - lo] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    rows = [parts[r][:shard(count, r, world)[1] - shard(count, r, world)[0]] for r in range(world)]
    return torch.cat(rows, 0)


def sum_over_ranks(t, group=None):
    """In-place all-reduce (sum) of a partial sum; returns the tensor."""
    import torch.distributed as dist
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def assemble_sharded(config, parts, count, group=None, *, points_um, z_positions, cut, solve=None):
    """Combine the per-rank partial products of one stage.

    `parts` (torch tensors on this rank): ``energies`` (band,), ``profiles``
    [top (band, planes), bottom], ``psf_sum`` / ``psf_abs_sum`` (X, Y, Z)
    partial site sums, ``tail_sum`` [top (h, w), bottom] partial sums of the
    site tail images.  Returns the host dictionary of maomi.optics.propagate
    except ``psf_3d`` (kept sharded by the caller).  ``solve(points, values,
    shape)`` evaluates the v4 masks (GPU path by default)."""
    import torch
    from .backends.cuda.batched import trapezoid
    from .fixed import _psf_z
    energies = gather_sites(parts["energies"], count, group)
    profiles = [gather_sites(p, count, group) for p in parts["profiles"]]
    s1 = sum_over_ranks(parts["psf_sum"].clone(), group)
    s2 = sum_over_ranks(parts["psf_abs_sum"].clone(), group)
    tails = [sum_over_ranks(t.clone(), group) for t in parts["tail_sum"]]
    weights = [(p * torch.as_tensor(trapezoid(p.shape[1]), dtype=p.dtype, device=p.device)).sum(1) * config.prop_um
               for p in profiles]
    values = torch.stack([energies, weights[0], weights[1]], 1)
    shape = tuple(int(v) for v in np.round(np.array(config.volume_um[:2]) * config.vres))
    pts = np.asarray(points_um, float)
    if solve is None:
        # every rank factors, solves and evaluates the same v4 system on its
        # own GPU (no further collective)
        from .numerics import v4_evaluate_grid_device, v4_factor_device, v4_solve_device
        dev = values.device
        p_dev, coef = v4_solve_device(v4_factor_device(pts * config.vres, device=dev), values)
        masks = v4_evaluate_grid_device(p_dev, coef, *shape, device=dev, points_host=pts * config.vres).cpu().numpy()
    else:
        masks = solve(pts * config.vres, values.cpu().numpy(), shape)
    mask = masks[..., 0]
    mean = float(mask.mean())
    res = {"psf": (s2 / count).cpu().numpy(), "psf_raw": (s1 / count).cpu().numpy(), "points_um": pts,
           "energies": energies.cpu().numpy(), "mask_raw": mask, "mask": mask / mean, "mask_mean": mean}
    for j, name in enumerate(("psfT", "psfB")):
        z = z_positions[0][cut:] if j == 0 else z_positions[2]
        tm = masks[..., j + 1]
        tm_mean = float(tm.mean())
        prof = profiles[j].cpu().numpy()
        res[name] = {"convmask": (tails[j] / count).cpu().numpy(), "weight": float(weights[j].mean()),
                     "psfZ": _psf_z(config, z, prof.sum(0)), "mask_raw": tm,
                     "mask": tm / tm_mean if tm_mean > 0 else tm, "mask_mean": tm_mean,
                     "weights_per_point": weights[j].cpu().numpy(), "profiles_per_point": prof}
    return res


def band_window(config, points_um, sizes):
    """Raw-field rows a band of sites reads: per stage (window size in
    ``sizes``) the rows [x0_min, x0_max + size) of the site windows, and the
    band's points shifted so its first row is row 0.  Only for ss = 1 (the
    phase preparation then reads each raw row alone; the bicubic resize of
    ss > 1 mixes neighbouring rows at the crop edges)."""
    pts = np.asarray(points_um, float).reshape(-1, 2)
    x0 = np.round(pts[:, 0] * config.vres).astype(int)
    lo = int(x0.min())
    rows = [(lo, int(x0.max()) + int(s)) for s in sizes]
    return rows, pts - np.array([lo / config.vres, 0.0])


def band_stage(config, raw_fields, points_um, *, device, precision="compensated", slots=96, band_upload=True):
    """Stage products of one band of sites, uploading only the raw rows the
    band's windows touch (``band_window``); no v4 masks (see
    ``assemble_sharded``).  Returns the ``fixed.stage_device`` dictionary."""
    from ._propagation import geometry
    from .fixed import stage_device
    pts = np.asarray(points_um, float).reshape(-1, 2)
    raw, local = raw_fields, pts
    if band_upload and config.ss == 1:
        g = geometry(config, raw_fields)
        rows, local = band_window(config, pts, (g.n, g.n2, g.n))
        raw = [a[r0:r1] for a, (r0, r1) in zip(raw_fields, rows)]
    dev = stage_device(config, raw, local, device=device, slots=slots, precision=precision, masks=False)
    dev["points_um"] = pts
    return dev


def run_stage_sharded(config, raw_fields, points_um=None, *, group=None, device=None, precision="compensated",
                      slots=96, band_upload=True):
    """The optical stage of one tissue block on every rank of `group`, each
    rank propagating its contiguous band of sites on its own GPU from the raw
    rows that band reads (plus the window halo), then the small exchange of
    ``assemble_sharded`` and the v4 masks on every rank."""
    import torch
    import torch.distributed as dist
    from .fixed import fixed_locations
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    device = device or f"cuda:{torch.cuda.current_device()}"
    pts = fixed_locations(config) if points_um is None else np.asarray(points_um, float)
    lo, hi = shard(len(pts), rank, world)
    dev = band_stage(config, raw_fields, pts[lo:hi], device=device, precision=precision, slots=slots,
                     band_upload=band_upload)
    plan = dev["plan"]
    # stage_device returns the band's mean tail image: scale back to its sum
    tail_sum = [c * (hi - lo) for c in dev["convmask"]]
    parts = {"energies": dev["energies"], "profiles": dev["profiles"], "psf_sum": dev["psf_sum"],
             "psf_abs_sum": dev["psf_abs_sum"], "tail_sum": tail_sum}
    res = assemble_sharded(config, parts, len(pts), group, points_um=pts, z_positions=plan.z_positions, cut=plan.cut)
    res["psf_3d_band"] = (lo, hi, dev["psf_3d"])
    return res
