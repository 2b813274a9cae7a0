"""``OpticalPlan``: persistent device geometry and the fused CUDA propagation.

Drop-in for maomi/backends/cuda/batched.py:18-250: the same constructor,
``evaluate`` / ``evaluate_graph`` / ``prepare_graph`` / ``cached`` methods and
attributes (``n``, ``n2``, ``z_positions``, ``cut``, ``paths_evaluated``).
What changes is underneath: every site runs through ``mm_propagate_sites``
(one persistent launch fed by a device work queue, or segment launches per
batch), screens are applied at each site's offset inside the propagation
kernel, the transfer functions' phases are formed in FP64, and saved planes
are reduced on the fly instead of being copied out.
"""

import copy

import numpy as np

from ... import _lib
from ..._propagation import edge_window_1d, geometry
from ...excitation import axial_profile, excitation_order
from ...numerics import is_identity_table, resample_matrix, resize_table, sparse_rows
from ...optics import pupil


FFT_SIZES = (64, 128, 256, 512)


def transfer_kernels(z, size, d2, wvl, nr, *, circulant=None):
    """Per-step 1-D transfer functions in FFT order with 1/size folded in:
    exp(-1j*pi*(wvl/nr)*dz*(k/(size*d2))^2)/size, phases formed in FP64.

    For windows without a radix-2 kernel (``circulant``, default: size not in
    64..512 powers of two) the kernels are the equivalent circular-convolution
    taps IDFT(Q), also formed in FP64."""
    if circulant is None:
        circulant = size not in FFT_SIZES
    lam = float(wvl) / float(nr)
    ks = np.fft.fftfreq(size) * size  # signed integer frequencies in FFT order
    f2 = (ks / (size * float(d2))) ** 2
    out = np.empty((len(z) - 1, size), np.complex64)
    for i, dz in enumerate(np.diff(np.asarray(z, float))):
        q = np.exp(1j * np.mod(-np.pi * lam * dz * f2, 2 * np.pi))
        out[i] = (np.fft.ifft(q) if circulant else q / size).astype(np.complex64)
    return out


def trapezoid(planes):
    w = np.ones(planes)
    w[0] *= 0.5
    w[-1] *= 0.5
    return w


class ResampleTables:
    """Sparse and dense forms of the ss-resample operator of one plane size."""

    def __init__(self, h, w, ss, device):
        import torch
        mx, my = resample_matrix(h, ss), resample_matrix(w, ss)
        (ix, wx), (iy, wy) = sparse_rows(mx), sparse_rows(my)
        self.shape = (mx.shape[0], my.shape[0])
        #: ss = 1: the resample is the identity (one unit tap per output)
        self.identity = bool(mx.shape == (h, h) and my.shape == (w, w) and np.array_equal(mx, np.eye(h))
                             and np.array_equal(my, np.eye(w)))
        self.ix = _lib.upload(ix, device)
        self.wx = _lib.upload(wx, device)
        self.iy = _lib.upload(iy, device)
        self.wy = _lib.upload(wy, device)
        self.mx = _lib.upload(mx, device, torch.float32)
        self.my = _lib.upload(my, device, torch.float32)


def _tables(config, g, raw_fields, device):
    """Device tables that depend on the configuration only: edge windows,
    transfer kernels, axial weights and the resample operators."""
    import torch
    counts = tuple(int(np.shape(a)[-1]) for a in raw_fields)
    r, ss = config.vres, config.ss
    n, n2 = g.n, g.n2
    a, b, c = counts
    t = {"edges": {k: _lib.upload(edge_window_1d(k), device) for k in {n, n2}}}
    t["axial"] = {key_: np.asarray(axial_profile(config, size, key_), np.float32)
                  for key_, size in [("focus", b), ("top", a + 1 - g.cut), ("bottom", c + 1)]}
    t["kernels"] = [_lib.upload(transfer_kernels(z, size, g.d2, g.wvl, g.nr), device)
                    for size, z in zip((n, n2, n), g.z)]
    axial = [t["axial"][k] for k in ("top", "bottom")]
    t["tail_weight"] = [_lib.upload((trapezoid(len(x)) * x).astype(np.float32), device) for x in axial]
    t["tail_axial"] = [_lib.upload(x.astype(np.float64) * ss ** 2, device) for x in axial]
    t["tail_trapezoid"] = [_lib.upload(trapezoid(len(x)), device) for x in axial]
    t["axial_focus"] = _lib.upload(t["axial"]["focus"], device)
    fshape = g.focal_shape
    t["focal_shape"] = (int(fshape[0]), int(fshape[1]))
    t["focal_resample"] = ResampleTables(*t["focal_shape"], ss, device)
    t["tail_resample"] = ResampleTables(n2, n2, ss, device)
    t["scale"] = float(ss ** 4 * (r * (1e6 * g.wvl) ** 1.5) / (np.pi * g.nr))
    return t


class OpticalPlan:
    """Persistent device state of the optical stage for one configuration."""

    def __init__(self, config, raw_fields, *, uin=None, device="cuda", native=True, precision="compensated"):
        import torch
        _lib.require_cuda(device)
        if precision not in _lib.PRECISIONS:
            raise ValueError("precision must be one of " + ", ".join(_lib.PRECISIONS))
        #: arithmetic of the radix-2 line transforms: "compensated" (FP32
        #: butterflies, DFT rotation constants as hi + lo float pairs),
        #: "compensated-full" (the twiddle tables too),
        #: "fp64" (FP64 butterflies, twiddles and filter), "mixed" (forward
        #: FP32, inverse FP64) or "fp32"; fields are stored complex64 in every mode
        self.precision = precision
        self.config = copy.deepcopy(config)
        self.device = device
        self.native = native
        self.order = excitation_order(config)
        r, ss = config.vres, config.ss
        g = geometry(config, raw_fields)
        self.geometry = g
        self.n, self.n2 = g.n, g.n2
        self.c, self.fc = g.crop, g.focal_crop
        self.wvl, self.nr = g.wvl, g.nr
        if raw_fields is None or len(raw_fields) != 3:
            raise ValueError("Three raw A/B/C fields are required")
        u = pupil(config, device=device) if uin is None else torch.as_tensor(uin, device=device)
        if u.dtype != torch.complex64:
            raise ValueError("This native backend requires complex64; use reference optics for other precision.")
        if tuple(u.shape) != (self.n, self.n):
            raise ValueError(f"Input pupil must be {self.n}x{self.n}, got {tuple(u.shape)}")
        stream = _lib.stream_of(device)
        t = _tables(config, g, raw_fields, device)
        self.edges = t["edges"]
        # ---- base field: pupil -> tissue top, scaled Fresnel step (FP64 chirps)
        z1 = float(np.float32(g.fl - (config.depth_um + config.volume_um[2] / 2) * 1e-6))
        self.base = torch.empty((self.n, self.n), dtype=torch.complex64, device=device)
        work = torch.empty_like(self.base)
        scratch = torch.empty(1024, dtype=torch.float64, device=device)
        desc = _lib.BaseDesc(n=self.n, d1=float(g.d1), d2=float(g.d2), dz=z1,
                             lambda_medium=float(g.wvl) / float(g.nr), edge1d=self.edges[self.n].data_ptr())
        _lib.check(_lib.load().mm_base_field(desc, _lib.ptr(u.contiguous()), _lib.ptr(self.base), _lib.ptr(work),
                                              _lib.ptr(scratch), stream), "base field")
        # ---- phase screens (Z, H, W) complex64
        scale = config.n_diff * 2 * np.pi / (config.wavelength_um * r)
        self.phases = [self._screens(a, ss, scale) for a in raw_fields]
        self.z_positions = g.z
        self.cut = g.cut
        self.axial = t["axial"]
        self.kernels = t["kernels"]
        self.tail_weight = t["tail_weight"]
        self.tail_axial = t["tail_axial"]
        self.tail_trapezoid = t["tail_trapezoid"]
        self.axial_focus = t["axial_focus"]
        self.focal_shape = t["focal_shape"]
        self.focal_resample = t["focal_resample"]
        self.tail_resample = t["tail_resample"]
        self.scale = t["scale"]
        self.cache = {}
        self.paths_evaluated = 0
        self.graphs = {}

    # ------------------------------------------------------------------ setup
    def _screens(self, raw, ss, scale):
        import torch
        a = torch.as_tensor(np.ascontiguousarray(raw, np.float32) if not isinstance(raw, torch.Tensor) else raw,
                            dtype=torch.float32, device=self.device).contiguous()
        H, W, Z = a.shape
        ix, wx = resize_table(H, ss)
        iy, wy = resize_table(W, ss)
        Ho, Wo = ix.shape[0], iy.shape[0]
        out = torch.empty((Z, Ho, Wo), dtype=torch.complex64, device=self.device)
        stream = _lib.stream_of(self.device)
        if is_identity_table(ix, wx) and is_identity_table(iy, wy):
            _lib.call("mm_phase_prepare", _lib.ptr(a), H, W, Z, None, None, Ho, 1, None, None, Wo, 1,
                      float(np.float32(scale)), _lib.ptr(out), None, stream)
            return out
        t = [_lib.upload(x, self.device) for x in
             (ix.astype(np.int32), wx.astype(np.float32), iy.astype(np.int32), wy.astype(np.float32))]
        tmp = torch.empty((Ho, W, Z), dtype=torch.float32, device=self.device)
        _lib.call("mm_phase_prepare", _lib.ptr(a), H, W, Z, _lib.ptr(t[0]), _lib.ptr(t[1]), Ho, ix.shape[1],
                  _lib.ptr(t[2]), _lib.ptr(t[3]), Wo, iy.shape[1], float(np.float32(scale)), _lib.ptr(out),
                  _lib.ptr(tmp), stream)
        return out

    def offsets(self, points_um):
        pts = np.asarray(points_um, float).reshape(-1, 2)
        scaled = pts * self.config.vres * self.config.ss
        if np.any(pts < 0) or np.any(pts > np.asarray(self.config.volume_um[:2])):
            raise ValueError("Outside FOV")
        if not np.allclose(scaled, np.round(scaled)):
            raise ValueError("Points must lie on supersampled grid")
        return pts, np.round(scaled).astype(np.int32)

    def schedule_for(self, schedule=None):
        if schedule is None:
            schedule = "persistent" if self.n == self.n2 else "batched"
        if schedule not in ("persistent", "batched"):
            raise ValueError("schedule must be persistent or batched")
        return _lib.MM_SCHEDULE_PERSISTENT if schedule == "persistent" else _lib.MM_SCHEDULE_BATCHED

    # ------------------------------------------------------------ propagation
    def run_sites(self, offsets, *, tail_per_site, slots, schedule=None, check=True, events=None, reserve_sms=0,
                  fault_drill=None):
        """Propagate every site; returns device buffers (focal, tail images, profiles).

        ``fault_drill`` (tests only): ``{"hold_site": s + 1, "spin_limit": polls}``
        makes site s's first item wait for a counter that is never published,
        so the persistent launch's bounded wait runs out and the call raises
        the timeout error."""
        import torch
        dev = self.device
        P = len(offsets)
        if isinstance(offsets, torch.Tensor) and offsets.is_cuda:  # already on the device (graph capture)
            if offsets.dtype != torch.int32 or tuple(offsets.shape) != (P, 2) or not offsets.is_contiguous():
                raise ValueError("device offsets must be a contiguous (P, 2) int32 tensor")
            off = offsets
        else:
            off = _lib.upload(np.asarray(offsets, np.int32), dev)
        zb = self.kernels[1].shape[0]
        fh, fw = self.focal_shape
        focal = torch.empty((P, zb, fh, fw), dtype=torch.float32, device=dev)
        planes = [len(self.axial["top"]), len(self.axial["bottom"])]
        sched = self.schedule_for(schedule)
        slots = max(1, min(int(slots), P))
        nimg = P if tail_per_site else slots
        if tail_per_site:
            imgs = [torch.empty((nimg, self.n2, self.n2), dtype=torch.float32, device=dev) for _ in range(2)]
        else:
            imgs = [torch.zeros((nimg, self.n2, self.n2), dtype=torch.float32, device=dev) for _ in range(2)]
        prof = [torch.empty((P, k), dtype=torch.float64, device=dev) for k in planes]
        plan = _lib.StagePlan()
        for s, (size, vol, kern) in enumerate(zip((self.n, self.n2, self.n), self.phases, self.kernels)):
            d = plan.stage[s]
            d.size, d.steps = size, kern.shape[0]
            d.screens = vol.data_ptr()
            d.vol_h, d.vol_w = vol.shape[1], vol.shape[2]
            d.edge1d = self.edges[size].data_ptr()
            d.kernels = kern.data_ptr()
        plan.base = self.base.data_ptr()
        plan.n, plan.n2, plan.order, plan.cut = self.n, self.n2, self.order, self.cut
        plan.focal_x0, plan.focal_y0 = self.fc[0].start, self.fc[1].start
        plan.focal_h, plan.focal_w = fh, fw
        plan.tail_weight[0], plan.tail_weight[1] = self.tail_weight[0].data_ptr(), self.tail_weight[1].data_ptr()
        plan.focal = focal.data_ptr()
        plan.tail_image[0], plan.tail_image[1] = imgs[0].data_ptr(), imgs[1].data_ptr()
        plan.tail_per_site = int(bool(tail_per_site))
        plan.tail_profile[0], plan.tail_profile[1] = prof[0].data_ptr(), prof[1].data_ptr()
        plan.offsets = off.data_ptr()
        plan.nsites = P
        plan.precision = _lib.PRECISIONS[self.precision]
        plan.reserve_sms = int(reserve_sms)
        if fault_drill:
            plan.hold_site = int(fault_drill.get("hold_site", 0))
            plan.spin_limit = int(fault_drill.get("spin_limit", 0))
        lib = _lib.load()
        wbytes = lib.mm_propagate_workspace_size(plan, slots, sched)
        work = torch.empty(wbytes + 256, dtype=torch.uint8, device=dev)
        base = (work.data_ptr() + 255) // 256 * 256
        if events is not None:
            events[0].record()
        rc = lib.mm_propagate_sites(plan, sched, slots, _lib.c_void_p(base), wbytes, int(check), _lib.stream_of(dev))
        if events is not None:
            events[1].record()
        _lib.check(rc, "propagation")
        self.paths_evaluated += P
        return dict(focal=focal, images=imgs, profiles=prof, offsets=off, workspace=work, plan=plan, schedule=sched,
                    slots=slots, workspace_base=base)

    def finalize_focal(self, focal, *, psf=True, sums=False):
        """(P,Z,h,w) focal powers -> psf (P,X,Y,Z), energies (P) and site sums."""
        import torch
        dev = self.device
        P, Z, H, W = focal.shape
        X, Y = self.focal_resample.shape
        out = torch.empty((P, X, Y, Z), dtype=torch.float32, device=dev) if psf else None
        energies = torch.empty(P, dtype=torch.float64, device=dev)
        s1 = torch.empty((X, Y, Z), dtype=torch.float64, device=dev) if sums else None
        s2 = torch.empty((X, Y, Z), dtype=torch.float64, device=dev) if sums else None
        rt = self.focal_resample
        tabs = (None, None, None, None) if rt.identity else (rt.ix, rt.wx, rt.iy, rt.wy)
        _lib.call("mm_focal_finalize", _lib.ptr(focal), _lib.ptr(tabs[0]), _lib.ptr(tabs[1]), rt.ix.shape[1],
                  _lib.ptr(tabs[2]), _lib.ptr(tabs[3]), rt.iy.shape[1], _lib.ptr(self.axial_focus),
                  float(np.float32(self.scale)), P, Z, H, W, X, Y, _lib.ptr(out), _lib.ptr(energies),
                  _lib.ptr(s1), _lib.ptr(s2), _lib.stream_of(dev))
        return out, energies, s1, s2

    def tail_profiles(self, prof, j):
        """Per-site tail profiles ss^2*axial*sum|E|^(2*order) (float64)."""
        axial = self.axial["top" if j == 0 else "bottom"].astype(np.float64)
        return prof * (self.config.ss ** 2 * axial)

    def tail_weights(self, profiles):
        return (profiles * trapezoid(profiles.shape[1])).sum(1) * self.config.prop_um

    # ------------------------------------------------------------- public API
    def evaluate(self, points_um, *, batch_size=16, tails=False, schedule=None):
        """Per-site PSFs (and tails) in the schema of batched.py:228-235.

        ``batch_size`` is the number of sites in flight."""
        import torch
        pts, off = self.offsets(points_um)
        with torch.inference_mode():
            res = self.run_sites(off, tail_per_site=bool(tails), slots=max(batch_size, 1), schedule=schedule)
            psf, _, _, _ = self.finalize_focal(res["focal"])
            out = {"psfs": psf.cpu().numpy(), "points_um": pts, "tails_computed": bool(tails)}
            if tails:
                rt = self.tail_resample
                X, Y = rt.shape
                for j, name in enumerate(("top", "bottom")):
                    imgs = res["images"][j]
                    conv = torch.empty((len(pts), X, Y), dtype=torch.float32, device=self.device)
                    _lib.call("mm_resample_images", _lib.ptr(imgs), imgs.shape[0], self.n2, self.n2,
                              _lib.ptr(rt.ix), _lib.ptr(rt.wx), rt.ix.shape[1], _lib.ptr(rt.iy), _lib.ptr(rt.wy),
                              rt.iy.shape[1], X, Y, float(self.config.ss ** 4), _lib.ptr(conv),
                              _lib.stream_of(self.device))
                    profile = self.tail_profiles(res["profiles"][j].cpu().numpy(), j)
                    out[name] = {"convmask": conv.cpu().numpy(),
                                 "weight": self.tail_weights(profile).astype(np.float32),
                                 "profile": profile.astype(np.float32)}
        return out

    def prepare_graph(self, batch_size=32):
        """Capture the focal path of one fixed batch of ``batch_size`` sites
        (queue reset, persistent propagation, focal finalize) in a CUDA graph
        over a device offset buffer; evaluate_graph replays it with only the
        offsets changed (batched.py:103-120)."""
        import torch
        if not self.native:
            raise ValueError("Graph requires native gather without CPU indexing")
        batch_size = int(batch_size)
        if batch_size < 1:
            raise ValueError("batch_size must be >= 1")
        if self.graphs.get(batch_size) is not None:
            return
        dev = self.device
        buf = torch.zeros((batch_size, 2), dtype=torch.int32, device=dev)  # window (0, 0) is always valid
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side), torch.inference_mode():
            for _ in range(3):  # settles allocations and kernel attributes before capture
                self.finalize_focal(self.run_sites(buf, tail_per_site=False, slots=batch_size)["focal"])
        torch.cuda.current_stream(dev).wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph), torch.inference_mode():
            run = self.run_sites(buf, tail_per_site=False, slots=batch_size, check=False)
            psf, _, _, _ = self.finalize_focal(run["focal"])
        self.paths_evaluated -= 4 * batch_size  # warm-up and capture evaluated no caller's sites
        host = torch.zeros((batch_size, 2), dtype=torch.int32, pin_memory=True)
        self.graphs[batch_size] = dict(graph=graph, offsets=buf, host=host, psf=psf, run=run)

    def evaluate_graph(self, points_um, *, batch_size=32):
        """Focal-only evaluation by graph replay, ``batch_size`` sites per
        replay with the last batch padded by window (0, 0) sites
        (batched.py:121-146 schema)."""
        import torch
        self.prepare_graph(batch_size)
        g = self.graphs[int(batch_size)]
        pts, off = self.offsets(points_um)
        off = np.asarray(off, np.int32).reshape(-1, 2)
        run = g["run"]
        collected = []
        with torch.inference_mode():
            for s0 in range(0, len(pts), batch_size):
                part = off[s0:s0 + batch_size]
                g["host"].zero_()
                g["host"][:len(part)] = torch.from_numpy(part)
                g["offsets"].copy_(g["host"], non_blocking=True)
                g["graph"].replay()
                _lib.check(_lib.load().mm_propagate_status(run["plan"], run["schedule"], run["slots"],
                                                           _lib.c_void_p(run["workspace_base"]),
                                                           _lib.stream_of(self.device)), "propagation")
                collected.append(g["psf"][:len(part)].cpu().numpy().copy())
                self.paths_evaluated += len(part)
        X, Y = self.focal_resample.shape
        psfs = np.concatenate(collected) if collected else np.zeros((0, X, Y, self.kernels[1].shape[0]), np.float32)
        return {"psfs": psfs, "points_um": pts, "tails_computed": False,
                "graph_padding_slots": int(np.ceil(len(pts) / batch_size)) * batch_size - len(pts)}

    def cached(self, points_um, *, batch_size=16):
        pts, off = self.offsets(points_um)
        keys = [tuple(int(v) for v in o) for o in off]
        missing = list(dict.fromkeys(k for k in keys if k not in self.cache))
        if missing:
            pos = np.array(missing) / (self.config.vres * self.config.ss)
            out = self.evaluate(pos, batch_size=batch_size)
            self.cache.update(zip(missing, out["psfs"]))
        return np.stack([self.cache[k] for k in keys])
