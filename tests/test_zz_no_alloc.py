"""The allocation-free propagation entry point against the workspace one.

mm_propagate_sites_noalloc serves callers that cannot allocate device memory
(hosts that keep the whole device heap in their own pool, or code that must
not call cudaMalloc while it runs): it takes its workspace from a fixed array
inside the library.  Both entry points are called through the C ABI on the
same plan; the no-alloc one is called twice in a row (the array keeps the
previous call's contents) and must reproduce the workspace call each time.
This file is collected last so a failure here leaves every other test run.
"""

import numpy as np
import pytest

from conftest import cfg_from, golden, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-6  # same kernel and data: only FP64 atomic order differs (profiles)


def _plan_struct(plan, off, outs):
    """The mm_stage_plan for `plan` writing into `outs` (per-site tails)."""
    from maomi_b200 import _lib
    sp = _lib.StagePlan()
    for s, (size, vol, kern) in enumerate(zip((plan.n, plan.n2, plan.n), plan.phases, plan.kernels)):
        d = sp.stage[s]
        d.size, d.steps = size, kern.shape[0]
        d.screens, d.vol_h, d.vol_w = vol.data_ptr(), vol.shape[1], vol.shape[2]
        d.edge1d, d.kernels = plan.edges[size].data_ptr(), kern.data_ptr()
    sp.base = plan.base.data_ptr()
    sp.n, sp.n2, sp.order, sp.cut = plan.n, plan.n2, plan.order, plan.cut
    sp.focal_x0, sp.focal_y0 = plan.fc[0].start, plan.fc[1].start
    sp.focal_h, sp.focal_w = plan.focal_shape
    sp.tail_weight[0], sp.tail_weight[1] = plan.tail_weight[0].data_ptr(), plan.tail_weight[1].data_ptr()
    sp.focal = outs["focal"].data_ptr()
    sp.tail_image[0], sp.tail_image[1] = outs["img0"].data_ptr(), outs["img1"].data_ptr()
    sp.tail_per_site = 1
    sp.tail_profile[0], sp.tail_profile[1] = outs["prof0"].data_ptr(), outs["prof1"].data_ptr()
    sp.offsets, sp.nsites = off.data_ptr(), off.shape[0]
    sp.precision = _lib.PRECISIONS[plan.precision]
    return sp


def _outputs(plan, P):
    import torch
    zb = plan.kernels[1].shape[0]
    planes = [len(plan.axial["top"]), len(plan.axial["bottom"])]
    f = dict(focal=torch.full((P, zb) + plan.focal_shape, np.nan, dtype=torch.float32, device="cuda"))
    for j in range(2):
        f[f"img{j}"] = torch.full((P, plan.n2, plan.n2), np.nan, dtype=torch.float32, device="cuda")
        f[f"prof{j}"] = torch.full((P, planes[j]), np.nan, dtype=torch.float64, device="cuda")
    return f


@pytest.mark.parametrize("schedule", [0, 1])
def test_noalloc_matches_workspace_entry_point(schedule):
    import torch
    from oracle import optics as O
    from maomi_b200 import _lib, synthetic
    from maomi_b200.backends.cuda.batched import OpticalPlan
    d = golden("stage_small")
    cfg = cfg_from(d)
    raw = synthetic.raw_fields(cfg, O.field_shapes(cfg), sigma=float(d["raw_sigma"]), rms=float(d["raw_rms"]),
                               seed=int(d["raw_seed"]))
    plan = OpticalPlan(cfg, raw)
    _, off_np = plan.offsets(d["points"])
    off = torch.as_tensor(off_np, device="cuda")
    P, slots = off.shape[0], 4
    lib = _lib.load()
    stream = _lib.stream_of("cuda")
    ref = _outputs(plan, P)
    sp = _plan_struct(plan, off, ref)
    nbytes = lib.mm_propagate_workspace_size(sp, slots, schedule)
    work = torch.empty(nbytes + 256, dtype=torch.uint8, device="cuda")
    base = (work.data_ptr() + 255) // 256 * 256
    _lib.check(lib.mm_propagate_sites(sp, schedule, slots, _lib.c_void_p(base), nbytes, 1, stream))
    torch.cuda.synchronize()
    for call in range(2):
        got = _outputs(plan, P)
        _lib.check(lib.mm_propagate_sites_noalloc(_plan_struct(plan, off, got), schedule, slots, 1, stream))
        torch.cuda.synchronize()
        for key in ref:
            a, b = got[key].cpu().numpy(), ref[key].cpu().numpy()
            assert np.isfinite(a).all(), (call, key)
            assert rel_l2(a, b) <= TOL, (call, key, rel_l2(a, b))


def _small_plan(count_per_axis):
    import torch
    from oracle import optics as O
    from maomi_b200 import synthetic
    from maomi_b200.backends.cuda.batched import OpticalPlan
    from maomi_b200.fixed import fixed_locations
    d = golden("stage_small")
    cfg = cfg_from(d)
    raw = synthetic.raw_fields(cfg, O.field_shapes(cfg), sigma=float(d["raw_sigma"]), rms=float(d["raw_rms"]),
                               seed=int(d["raw_seed"]))
    plan = OpticalPlan(cfg, raw)
    _, off_np = plan.offsets(fixed_locations(cfg, count_per_axis))
    return plan, torch.as_tensor(off_np, device="cuda")


def test_noalloc_sizes_requests_as_they_run():
    """A request is sized after the same clamping the workspace entry point
    applies (at most one slot per site, waves balanced): 4,096 slots asked
    for the 9-site plan run as 9 and fit; 144 sites in flight at 128 x 128
    (256 KiB each, 36 MiB) do not fit the 32 MiB array and are rejected."""
    from maomi_b200 import _lib
    lib = _lib.load()
    stream = _lib.stream_of("cuda")
    plan, off = _small_plan(3)
    outs = _outputs(plan, off.shape[0])
    _lib.check(lib.mm_propagate_sites_noalloc(_plan_struct(plan, off, outs), 0, 4096, 1, stream))
    assert np.isfinite(outs["focal"].cpu().numpy()).all()
    plan, off = _small_plan(12)
    outs = _outputs(plan, off.shape[0])
    for slots in (144, 4096):
        rc = lib.mm_propagate_sites_noalloc(_plan_struct(plan, off, outs), 0, slots, 1, stream)
        assert rc == _lib.MM_ERR_ARGUMENT
        assert "static array" in _lib.last_error()
    # 72 slots balance to 72 (two waves of 72): 18 MiB, accepted
    _lib.check(lib.mm_propagate_sites_noalloc(_plan_struct(plan, off, outs), 0, 72, 1, stream))
