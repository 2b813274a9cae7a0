"""The optical stage on the fixed 65 x 65 site lattice, end to end on the GPU.

Mirrors maomi/fixed.py: ``fixed_locations`` (:15-33), ``field_shapes``
(:36-56), ``assemble`` (:119-190, the ``matlab_v4`` mode) and ``run_fixed``
(:193-411).  ``run_stage`` is the fused device path behind them: phase
preparation, the persistent propagation of every site, both tails reduced on
the device, focal PSF finalisation with FP64 site sums, and the FP64 v4 mask
assembly (Green matrix, dense solve and grid evaluation on the GPU).  Only
the final products are copied to the host.
"""

import time

import numpy as np

from . import _lib
from ._optical_math import gaussian_beam_size
from .numerics import v4_evaluate_grid_device, v4_factor_device, v4_interpolate, v4_solve_device


def fixed_locations(config, count_per_axis=65):
    """Uniform physical XY locations snapped to the supersampled lattice."""
    if isinstance(count_per_axis, bool) or not isinstance(count_per_axis, int) or count_per_axis < 2:
        raise ValueError("count_per_axis must be an integer >= 2")
    ticks = np.asarray(config.volume_um[:2], float) * config.vres * config.ss
    if (not np.all(np.isfinite(ticks)) or np.any(ticks < count_per_axis - 1)
            or not np.allclose(ticks, np.round(ticks))):
        raise ValueError(
            f"Fixed {count_per_axis}x{count_per_axis} requires an integer optical lattice "
            f"with at least {count_per_axis} positions per axis; choose count_per_axis explicitly")
    axes = [np.round(np.linspace(0, int(round(t)), count_per_axis)) / (config.vres * config.ss) for t in ticks]
    points = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 2)
    if len(np.unique(points, axis=0)) != count_per_axis ** 2:
        raise ValueError("Grid contains duplicate locations")
    return points


def field_shapes(config):
    """Shapes of the raw A/B/C occupancy fields the stage expects."""
    v, p = config.parameters()
    r = config.vres
    n = int(round((v.vasc_sz[0] - v.vol_sz[0]) * r))
    n2 = int(round(min(max(gaussian_beam_size(p, config.psf_um[2] / 2, 3)) * r * 2, n))) if config.propcrop else n
    za = int(round((config.depth_um + config.volume_um[2] / 2 - config.psf_um[2] / 2) * r))
    zb = int(round(config.psf_um[2] * r))
    pc = int(round(config.prop_um * r))
    nc = int(round(config.tail_um * r))
    if min(za, zb, pc, nc) <= 0:
        raise ValueError("Optical A/B/C propagation extents must be positive")
    xy = np.round(np.asarray(config.volume_um[:2]) * r).astype(int)
    return [(int(xy[0] + n), int(xy[1] + n), int(np.ceil(za / pc))),
            (int(xy[0] + n2), int(xy[1] + n2), zb),
            (int(xy[0] + n), int(xy[1] + n), int(np.ceil(nc / pc)))]


_SIDE_STREAMS = {}
#: per device, an event after the most recent persistent propagation launch
_LAST_PROPAGATION = {}
RESERVE_SMS = 0   # SMs the persistent kernel leaves to the overlapped v4 factorisation
# Sites in flight in the persistent schedule: 96 (94 after balancing 4,225
# sites into 45 waves) measured 3 % faster than 64 and than 128 on the
# benchmark stage; their 256^2 fields (48 MB) stay in L2.
SLOTS = 96


def _side_stream(device):
    """A high-priority stream per device for work that overlaps the propagation."""
    import torch
    key = str(torch.device(device))
    if key not in _SIDE_STREAMS:
        _SIDE_STREAMS[key] = torch.cuda.Stream(device=device, priority=-1)
    return _SIDE_STREAMS[key]


def _psf_z(config, z, profile):
    """Tail axial profile resampled to the voxel pitch and normalised to unit mean."""
    actual = z - z[0]
    axial = np.arange(round(actual[-1] * 1e6 * config.vres) + 1) / config.vres
    interp = np.interp(axial, actual * 1e6, profile)
    return interp / interp.mean() if interp.mean() > 0 else interp


def assemble(config, out, shape, *, mask_mode="matlab_v4", z_positions=None, cut=None, device="cuda"):
    """Masks and averaged PSFs from per-site outputs (fixed.py:119-190).

    Only ``matlab_v4`` is provided (the cubic mode is diagnostic-only in the
    reference); the v4 system is solved and evaluated on the GPU."""
    if mask_mode != "matlab_v4":
        raise ValueError("mask_mode must be matlab_v4 (cubic aggregation is not provided)")
    points = out["points_um"]
    psfs = out["psfs"]
    energies = psfs.sum((1, 2, 3), dtype=np.float64)
    values = [energies]
    tails = bool(out["tails_computed"])
    if tails:
        values.extend(out[k]["weight"] for k in ("top", "bottom"))
    values = np.stack(values, axis=1)
    q = np.stack(np.meshgrid(*[np.arange(k) + 0.5 for k in shape], indexing="ij"), -1)
    masks = v4_interpolate(points * config.vres, values, q, device=device)
    mask = masks[..., 0]
    mean = float(mask.mean())
    if not np.isfinite(mean) or mean <= 0:
        raise ValueError("Nonpositive or invalid mean excitation energy")
    weights = np.full(len(points), 1 / len(points))
    result = {
        "psf": (weights @ np.abs(psfs).reshape(len(points), -1)).reshape(psfs.shape[1:]),
        "psf_raw": (weights @ psfs.reshape(len(points), -1)).reshape(psfs.shape[1:]),
        "psf_3d": psfs, "points_um": points, "energies": energies,
        "mask_raw": mask, "mask": mask / mean, "mask_mean": mean, "mask_mode": mask_mode,
        "geometry_cache_hit": False, "tails_computed": tails, "unique_optical_paths": len(points),
        "negative_resampling_mass_fraction": float(
            -np.minimum(psfs, 0).sum(dtype=np.float64) / max(np.abs(psfs).sum(dtype=np.float64), 1e-30)),
    }
    if tails:
        for j, (native, name) in enumerate([("top", "psfT"), ("bottom", "psfB")]):
            data = out[native]
            z = z_positions[0][cut:] if j == 0 else z_positions[2]
            tm = masks[..., j + 1]
            tm_mean = float(tm.mean())
            result[name] = {
                "convmask": data["convmask"].mean(0),
                "weight": float(data["weight"].mean()),
                "psfZ": _psf_z(config, z, data["profile"].sum(0, dtype=np.float64)),
                "mask_raw": tm, "mask": tm / tm_mean if tm_mean > 0 else tm, "mask_mean": tm_mean,
                "weights_per_point": data["weight"], "profiles_per_point": data["profile"],
            }
    return result


def stage_device(config, raw_fields, points_um=None, *, uin=None, device="cuda", tails=True, count_per_axis=65,
                 slots=SLOTS, schedule=None, plan=None, check=True, events=None, precision="compensated",
                 reserve_sms=RESERVE_SMS, masks=True):
    """Fused optical stage leaving every product on the device.

    Phase preparation (inside ``OpticalPlan``), the persistent propagation of
    every site with both tails reduced on the fly, focal PSF finalisation with
    FP64 site sums and the FP64 v4 mask assembly.  Returns a dict of device
    tensors (``psf_3d``, ``energies``, ``psf_sum``, ``psf_abs_sum``, ``masks``,
    tail ``profiles``/``weights``/``convmask``) plus the plan.  ``events``
    (a pair of CUDA events) brackets the propagation launch.  The v4 system
    depends on the site positions only; it is factored on a high-priority side
    stream that waits only for the previous stage's propagation launch, so it
    runs beside that stage's reductions and this stage's preparation; the
    propagation launch waits for it (unless ``reserve_sms`` SMs are left to
    it), because factorisation kernels running beside the persistent launch
    hold SMs it would otherwise use.  ``masks=False`` skips the v4 masks
    (``masks`` is then None): a sharded stage solves them once over every
    rank's sites."""
    import torch
    from .backends.cuda.batched import OpticalPlan, trapezoid
    _lib.require_cuda(device)
    points = fixed_locations(config, count_per_axis) if points_um is None else np.asarray(points_um, float)
    if np.any(points < 0) or np.any(points > np.asarray(config.volume_um[:2])):
        raise ValueError("Outside FOV")
    dev = device if plan is None else plan.device
    with torch.inference_mode():
        main = torch.cuda.current_stream(dev)
        factor = None
        if masks and len(points) > 1:
            # the factorisation depends on the host-side site positions only:
            # it waits for the last persistent launch queued on this device
            # (not for the reductions behind it), so it runs beside them
            side = _side_stream(dev)
            last = _LAST_PROPAGATION.get(str(torch.device(dev)))
            if last is not None:
                side.wait_event(last)
            with torch.cuda.stream(side):
                factor = v4_factor_device(points * config.vres, device=dev)
        if plan is None:
            plan = OpticalPlan(config, raw_fields, uin=uin, device=device, precision=precision)
        pts, off = plan.offsets(points)
        P = len(pts)
        if factor is not None and not reserve_sms:
            # the factorisation's kernels take whole SMs from the persistent
            # launch if they overlap it: let them finish first (they overlap
            # the previous stage's reductions and this stage's preparation)
            main.wait_stream(side)
        res = plan.run_sites(off, tail_per_site=False, slots=slots, schedule=schedule, check=check, events=events,
                             reserve_sms=reserve_sms if factor is not None else 0)
        done = torch.cuda.Event()
        done.record(main)
        _LAST_PROPAGATION[str(torch.device(dev))] = done
        psf, energies, s1, s2 = plan.finalize_focal(res["focal"], psf=True, sums=True)
        prof, wts = [], []
        for j in range(2):
            pj = res["profiles"][j] * plan.tail_axial[j]
            prof.append(pj)
            wts.append((pj * plan.tail_trapezoid[j]).sum(1) * config.prop_um)
        values = torch.stack([energies, wts[0], wts[1]] if tails else [energies], 1)
        shape = tuple(int(v) for v in np.round(np.array(config.volume_um[:2]) * config.vres))
        if not masks:
            masks = None
        elif P > 1:
            main.wait_stream(side)
            for t in factor.tensors():
                t.record_stream(main)
            p_dev, coef = v4_solve_device(factor, values)
            masks = v4_evaluate_grid_device(p_dev, coef, *shape, device=dev, points_host=pts * config.vres)
        else:
            masks = values[0].reshape(1, 1, -1).expand(shape[0], shape[1], -1).contiguous()
        convs = []
        if tails:
            rt = plan.tail_resample
            X, Y = rt.shape
            scratch = torch.empty(plan.n2 * plan.n2, dtype=torch.float64, device=dev)
            for j in range(2):
                conv = torch.empty((X, Y), dtype=torch.float64, device=dev)
                imgs = res["images"][j]
                _lib.call("mm_tail_finalize", _lib.ptr(imgs), imgs.shape[0], plan.n2, plan.n2, _lib.ptr(rt.mx),
                          _lib.ptr(rt.my), X, Y, float(config.ss ** 4) / P, _lib.ptr(conv), _lib.ptr(scratch),
                          _lib.stream_of(dev))
                convs.append(conv)
    return dict(plan=plan, points_um=pts, psf_3d=psf, energies=energies, psf_sum=s1, psf_abs_sum=s2, masks=masks,
                profiles=prof, weights=wts, convmask=convs, tails=bool(tails))


def stage_copy_async(dev, *, return_psf_3d=True, out=None, stream=None):
    """Enqueue the device -> host copies of one ``stage_device`` result on
    ``stream`` (ordered after the current stream's work); returns the pending
    copy for ``stage_result``.  Destinations are pinned host buffers (``out``
    entries where given), so the copies overlap later device work."""
    import torch
    plan, P = dev["plan"], len(dev["points_um"])
    main = torch.cuda.current_stream(plan.device)
    stream = main if stream is None else stream
    if stream is not main:
        stream.wait_stream(main)

    with torch.inference_mode(), torch.cuda.stream(stream):
        def host(t, key):
            dst = out[key] if out is not None and key in out else torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            dst.copy_(t, non_blocking=True)
            if stream is not main:
                t.record_stream(stream)
            return dst

        neg = -torch.clamp(dev["psf_3d"], max=0).sum(dtype=torch.float64) / torch.clamp(dev["psf_abs_sum"].sum(),
                                                                                          min=1e-30)
        h = {"masks": host(dev["masks"], "masks"), "psf": host(dev["psf_abs_sum"] / P, "psf"),
             "psf_raw": host(dev["psf_sum"] / P, "psf_raw"), "energies": host(dev["energies"], "energies"),
             "psf_3d": host(dev["psf_3d"], "psf_3d") if return_psf_3d else None,
             "profiles": [host(p, f"profile{j}") for j, p in enumerate(dev["profiles"])],
             "weights": [host(w, f"weight{j}") for j, w in enumerate(dev["weights"])],
             "convmask": [host(c, f"convmask{j}") for j, c in enumerate(dev["convmask"])],
             "neg": host(neg.reshape(1), "neg")}
        done = torch.cuda.Event()
        done.record(stream)
    return {"dev": dev, "host": h, "event": done}


def stage_result(config, pending):
    """Host result dictionary (the keys of maomi.optics.propagate / assemble)
    of a ``stage_copy_async`` once its copies have completed."""
    pending["event"].synchronize()
    dev, h = pending["dev"], pending["host"]
    plan, P = dev["plan"], len(dev["points_um"])
    masks_h = h["masks"].numpy()
    mask = masks_h[..., 0]
    mean = float(mask.mean())
    if not np.isfinite(mean) or mean <= 0:
        raise ValueError("Nonpositive or invalid mean excitation energy")
    result = {
        "psf": h["psf"].numpy(), "psf_raw": h["psf_raw"].numpy(),
        "psf_3d": h["psf_3d"].numpy() if h["psf_3d"] is not None else None,
        "points_um": dev["points_um"], "energies": h["energies"].numpy(),
        "mask_raw": mask, "mask": mask / mean, "mask_mean": mean, "mask_mode": "matlab_v4",
        "tails_computed": dev["tails"], "unique_optical_paths": P,
        "negative_resampling_mass_fraction": float(h["neg"][0]),
    }
    if dev["tails"]:
        for j, name in enumerate(("psfT", "psfB")):
            z = plan.z_positions[0][plan.cut:] if j == 0 else plan.z_positions[2]
            tm = masks_h[..., j + 1]
            tm_mean = float(tm.mean())
            prof_j, wts_j = h["profiles"][j].numpy(), h["weights"][j].numpy()
            result[name] = {
                "convmask": h["convmask"][j].numpy(), "weight": float(wts_j.mean()),
                "psfZ": _psf_z(config, z, prof_j.sum(0)),
                "mask_raw": tm, "mask": tm / tm_mean if tm_mean > 0 else tm, "mask_mean": tm_mean,
                "weights_per_point": wts_j, "profiles_per_point": prof_j,
            }
    return result


def stage_to_host(config, dev, *, return_psf_3d=True, out=None):
    """Host result dictionary (the keys of maomi.optics.propagate / assemble)
    from ``stage_device`` output.  ``out`` may hold pinned host buffers."""
    return stage_result(config, stage_copy_async(dev, return_psf_3d=return_psf_3d, out=out))


#: pinned host buffer sets not held by a running ``run_stages`` call, keyed
#: by the shapes of the products they hold
_PINNED_FREE = {}


def _pinned_set(dev, return_psf_3d):
    """Pinned host buffers for every product of one stage (shapes of ``dev``)."""
    import torch
    items = {"masks": dev["masks"], "psf": dev["psf_abs_sum"], "psf_raw": dev["psf_sum"], "energies": dev["energies"]}
    if return_psf_3d:
        items["psf_3d"] = dev["psf_3d"]
    for j in range(len(dev["profiles"])):
        items[f"profile{j}"], items[f"weight{j}"] = dev["profiles"][j], dev["weights"][j]
    for j in range(len(dev["convmask"])):
        items[f"convmask{j}"] = dev["convmask"][j]
    out = {k: torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for k, t in items.items()}
    out["neg"] = torch.empty(1, dtype=torch.float64, pin_memory=True)
    return out


def run_stages(config, blocks, points_um=None, *, device="cuda", depth=2, return_psf_3d=True, reuse=False,
               **kwargs):
    """Stage results of a sequence of tissue blocks (each three raw A/B/C
    fields: NumPy arrays, pinned host tensors or device tensors), pipelined:
    while block i's products are copied to the host on a copy stream, block
    i+1 is uploaded and computed.  Yields the host dictionaries in order.

    ``reuse=True`` copies into ``2 * depth`` pinned buffer sets that this call
    takes from a pool kept between calls (no page-locked allocation per
    block).  Block k's products land in set k mod 2*depth, which the copy of
    block k + 2*depth overwrites; that copy is enqueued only after result
    k + depth has been yielded, so a yielded result's arrays stay valid until
    ``depth`` further results have been yielded.  Calls running side by side
    hold disjoint sets.  When a call ends its sets return to the pool, and
    the arrays of its last results stay valid until another ``reuse=True``
    call starts."""
    import collections
    import torch
    copy = torch.cuda.Stream(device=device)
    up = torch.cuda.Stream(device=device)
    main = torch.cuda.current_stream(device)
    pending = collections.deque()
    held = {}
    count = 0
    try:
        for raw in blocks:
            # uploads run on their own stream, so block i+1's fields cross PCIe
            # while block i still computes; the compute stream waits for them
            with torch.cuda.stream(up):
                fields = [a.to(device, non_blocking=True) if isinstance(a, torch.Tensor) else _lib.upload(a, device)
                          for a in raw]
            main.wait_stream(up)
            for f in fields:
                f.record_stream(main)
            dev = stage_device(config, fields, points_um, device=device, **kwargs)
            out = None
            if reuse:
                key = (str(device), tuple((k, tuple(v.shape)) for k, v in dev.items() if hasattr(v, "shape")),
                       len(dev["profiles"]), bool(return_psf_3d))
                sets = held.setdefault(key, [])
                if len(sets) < 2 * depth:
                    free = _PINNED_FREE.setdefault(key, [])
                    sets.append(free.pop() if free else _pinned_set(dev, return_psf_3d))
                out = sets[count % (2 * depth)]
            pending.append(stage_copy_async(dev, return_psf_3d=return_psf_3d, out=out, stream=copy))
            count += 1
            if len(pending) >= depth:
                yield stage_result(config, pending.popleft())
        while pending:
            yield stage_result(config, pending.popleft())
    finally:
        # copies still in flight (a generator closed early) finish before
        # their buffers can be handed to another call
        copy.synchronize()
        for key, sets in held.items():
            _PINNED_FREE.setdefault(key, []).extend(sets)


def run_stage(config, raw_fields, points_um=None, *, uin=None, device="cuda", tails=True, count_per_axis=65,
              slots=SLOTS, schedule=None, return_psf_3d=True, plan=None, check=True, precision="compensated"):
    """The whole optical stage on the GPU, returning the host result dictionary
    of maomi.optics.propagate (optics.py:341-381) / fixed.assemble."""
    dev = stage_device(config, raw_fields, points_um, uin=uin, device=device, tails=tails,
                       count_per_axis=count_per_axis, slots=slots, schedule=schedule, plan=plan, check=check,
                       precision=precision)
    return stage_to_host(config, dev, return_psf_3d=return_psf_3d)




def _multibeam(config, volume, input_pupil, beam_weights, opts):
    """Incoherent channels (fixed.py:237-285): one stage per named pupil on
    shared raw fields; detected intensities add with nonnegative weights."""
    from .fields import prepare_fields
    if opts["custom_phase"] is not None:
        raise ValueError("Compose channel pupil phases explicitly")
    if not input_pupil:
        raise ValueError("At least one beam required")
    weights = {k: 1.0 for k in input_pupil} if beam_weights is None else dict(beam_weights)
    if (set(weights) != set(input_pupil) or not all(np.isfinite(w) and w >= 0 for w in weights.values())
            or sum(weights.values()) <= 0):
        raise ValueError("Nonnegative detected-intensity weight per beam required")
    start = time.perf_counter()
    _lib.require_cuda(opts["device"])
    raw = (prepare_fields(config, opts["vessels"], scatter=opts["scatter"], device=opts["device"])
           if opts["raw_fields"] is None else opts["raw_fields"])
    keep = ("vessels", "tails", "batch_size", "count_per_axis", "mask_mode", "device", "render_image")
    channels = {name: run_fixed(config, volume, raw_fields=raw, input_pupil=field, **{k: opts[k] for k in keep})
                for name, field in input_pupil.items()}
    points = fixed_locations(config, opts["count_per_axis"])
    out = {"channels": channels, "beam_weights": weights, "points_um": points,
           "unique_optical_paths": len(points) * len(channels), "unique_optical_positions": len(points),
           "total_seconds": time.perf_counter() - start,
           "settings": {"combination": "incoherent detected-intensity sum", "scaling": config.scaling,
                        "paths_per_position": len(channels), "count_per_axis": opts["count_per_axis"],
                        "mask_mode": opts["mask_mode"]}}
    if opts["render_image"]:
        out["image"] = sum(weights[k] * v["image"] for k, v in channels.items())
    return out


def run_fixed(config, volume=None, *, vessels=None, raw_fields=None, scatter=True, custom_phase=None,
              phase_units="radians", phase_aperture="objective", input_pupil=None, beam_weights=None, tails=True,
              batch_size=32, count_per_axis=65, mask_mode="matlab_v4", device="cuda", rana=False,
              render_image=True):
    """MATLAB v4 masks and arithmetic PSF averaging on the fixed site lattice
    (maomi/fixed.py:193-411), every stage on the GPU.

    Raw fields are generated on the device when not supplied
    (``maomi_b200.fields.prepare_fields``; its noise is a device draw from
    ``config.seed``, not the reference's CPU stream), the collection mask is
    built from ``vessels``, a mapping of pupils runs incoherent channels, and
    ``render_image`` convolves the masked volume with the mean PSF
    (``maomi_b200.scanning.zstack``).  ``batch_size`` is the number of sites in
    flight.  The RANA attach branch belongs to the reference's RANA add-on
    package and is not provided (``rana`` must be False or None)."""
    from .fields import prepare_fields
    from .optics import collection_mask, pupil
    from .scanning import zstack
    if rana is not False and rana is not None:
        raise ValueError("the RANA add-on attach path is not part of maomi_b200.run_fixed; render with "
                         "maomi_b200.rana.RanaOperator over the returned psf_3d")
    if mask_mode != "matlab_v4":
        raise ValueError("run_fixed requires matlab_v4; use maomi.enhanced.CubicFullFieldRenderer "
                         "with a complete custom FullFieldPSF for cubic imaging")
    if isinstance(input_pupil, dict):
        return _multibeam(config, volume, input_pupil, beam_weights,
                          dict(vessels=vessels, raw_fields=raw_fields, scatter=scatter, custom_phase=custom_phase,
                               tails=tails, batch_size=batch_size, count_per_axis=count_per_axis,
                               mask_mode=mask_mode, device=device, render_image=render_image))
    if beam_weights is not None:
        raise ValueError("beam_weights requires a mapping of pupils")
    if not str(device).startswith("cuda"):
        raise ValueError("Fixed fast pipeline requires CUDA; use maomi.optics for CPU reference calculations")
    _lib.require_cuda(device)
    import torch
    if isinstance(batch_size, bool) or not isinstance(batch_size, int) or batch_size < 1:
        raise ValueError("batch_size must be a positive integer")
    if phase_units not in ("radians", "waves") or phase_aperture not in ("objective", "excitation"):
        raise ValueError("Invalid pupil phase units/aperture")
    if input_pupil is not None and custom_phase is not None:
        raise ValueError("Supply either input_pupil or custom_phase; compose the field explicitly")
    expected = tuple(int(v) for v in np.round(np.asarray(config.volume_um) * config.vres).astype(int))
    if render_image:
        vol = volume if isinstance(volume, torch.Tensor) else np.asarray(volume, np.float32)
        if tuple(vol.shape) != expected or not bool(np.isfinite(np.asarray(vol.cpu() if isinstance(
                vol, torch.Tensor) else vol)).all()):
            raise ValueError(f"Expected finite volume of shape {expected}")
    started = time.perf_counter()
    timings = {}
    supplied = raw_fields is not None
    t = time.perf_counter()
    raw = prepare_fields(config, vessels, scatter=scatter, device=device) if raw_fields is None else raw_fields
    shapes = field_shapes(config)
    if len(raw) != 3 or any(tuple(np.shape(a)) != tuple(s) for a, s in zip(raw, shapes)):
        raise ValueError(f"Raw A/B/C fields must have shapes {shapes}")
    for a in raw:
        if (a.is_complex() if isinstance(a, torch.Tensor) else np.iscomplexobj(a)) or not bool(
                (torch.isfinite(a).all() if isinstance(a, torch.Tensor) else np.isfinite(np.asarray(a)).all())):
            raise ValueError("Raw refractive-index fields must be finite and real")
    col = (collection_mask(vessels, config, device=device) if vessels is not None
           else np.ones(expected[:2], np.float32))
    timings["fields_and_collection"] = time.perf_counter() - t
    t = time.perf_counter()
    u = (pupil(config, custom_phase=custom_phase, phase_units=phase_units, phase_aperture=phase_aperture,
               device=device) if input_pupil is None
         else torch.as_tensor(input_pupil, dtype=torch.complex64).to(device))
    v, _ = config.parameters()
    n = int(round((v.vasc_sz[0] - config.volume_um[0]) * config.vres * config.ss))
    if tuple(u.shape) != (n, n) or not bool(torch.isfinite(u).all()) or not bool((u.abs() > 0).any()):
        raise ValueError("Input pupil must be a finite nonzero complex field on the optical grid")
    from .backends.cuda.batched import OpticalPlan
    plan = OpticalPlan(config, raw, uin=u, device=device)
    torch.cuda.synchronize(device)
    timings["plan"] = time.perf_counter() - t
    t = time.perf_counter()
    result = run_stage(config, raw, fixed_locations(config, count_per_axis), device=device, tails=tails,
                       slots=batch_size, plan=plan)
    result["colmask"] = col
    timings["propagation_and_aggregation"] = time.perf_counter() - t
    t = time.perf_counter()
    if render_image:
        result["image"] = zstack(volume, result["psf"].astype(np.float32), mask=result["mask"].astype(np.float32),
                                 collection_mask=col, device=device).cpu().numpy()
    timings["static_scan"] = time.perf_counter() - t
    result["timing_seconds"] = timings
    result["total_seconds"] = time.perf_counter() - started
    result["settings"] = {"seed": config.seed, "scaling": config.scaling,
                          "fields": "provided" if supplied else "generated",
                          "scatter": None if supplied else bool(scatter), "phase_units": phase_units,
                          "phase_aperture": phase_aperture,
                          "input_pupil": "provided" if input_pupil is not None else "gaussian",
                          "collection_absorption": vessels is not None, "tail_background_added_to_image": False,
                          "count_per_axis": count_per_axis, "adaptive": False, "low_order_subtraction": False,
                          "mask_mode": mask_mode, "psf_average": "arithmetic mean of absolute per-point PSFs"}
    return result
