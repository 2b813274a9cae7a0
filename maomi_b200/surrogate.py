"""Learned surrogate for the per-site scattered focal PSF.

A Fourier neural operator (lifting, 4 spectral layers of width 32 with 12 x 12
retained modes and a pointwise 1x1 branch, linear projection) maps a site's
64 x 64 window of pooled refractive-index screens to its focal PSF on 64 x 64
pixels x 9 planes (unit sum).  Training and inference run on the library's
BF16 tcgen05 GEMMs (FP32 accumulation) and CUDA-core kernels for the
spectral mixing, activations, loss and Adam; PyTorch only provides device
memory, streams and indexing.

The plain propagator is both the teacher and the gatekeeper: ``training_set``
builds (inputs, PSF) pairs with it, and ``SurrogateStage.run`` re-propagates a
seeded fraction of the sites with it and replaces the whole surrogate output
by the plain result when the sample's relative L2 error exceeds the
tolerance.  The reference has no learned component; this module has no
reference counterpart.
"""

import ctypes
import math
import time
from dataclasses import replace

import numpy as np

from . import _lib

GRID = 64
NPIX = GRID * GRID
WIDTH = 32
NMODES = 288
NROWS = 576
OUT = 16
PLANES = 9
LAYERS = 4
GROUPS = 16
PARAM_NAMES = ["Wl", "bl"] + [f"{k}{l}" for l in range(LAYERS) for k in ("W", "b", "Rr", "Ri")] + ["Wp", "bp"]
PARAM_SHAPES = {"Wl": (WIDTH, WIDTH), "bl": (WIDTH,), "Wp": (OUT, WIDTH), "bp": (OUT,),
                **{f"W{l}": (WIDTH, WIDTH) for l in range(LAYERS)}, **{f"b{l}": (WIDTH,) for l in range(LAYERS)},
                **{f"Rr{l}": (NMODES, WIDTH, WIDTH) for l in range(LAYERS)},
                **{f"Ri{l}": (NMODES, WIDTH, WIDTH) for l in range(LAYERS)}}


SurrogateDesc = _lib.SurrogateDesc


def screen_groups(total):
    """Boundaries of the 16 consecutive screen groups (sizes differ by at most one)."""
    sizes = [len(a) for a in np.array_split(np.arange(total), GROUPS)]
    return np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)


def plane_index(planes):
    """The 9 focal planes (of ``planes``) the surrogate predicts, evenly spread."""
    return np.round(np.linspace(2, planes - 3, PLANES)).astype(int)


def surrogate_config(config):
    """``config`` with the focal crop widened to the surrogate's 64 x 64 pixels
    and one-photon scaling: the surrogate predicts the scattered focal
    intensity |E|^2 (the excitation order is applied to it afterwards)."""
    lateral = GRID / (config.vres * config.ss)
    return replace(config, psf_um=(lateral, lateral, config.psf_um[2]), scaling="one-photon")


def _layout():
    off = (ctypes.c_longlong * 21)()
    _lib.check(_lib.load().mm_surrogate_layout(off, 21), "surrogate layout")
    return list(off)


class PSFSurrogate:
    """Network parameters, optimiser state and per-batch device buffers."""

    def __init__(self, *, device="cuda", seed=0, input_scale=1.0):
        import torch
        _lib.require_cuda(device)
        self.device = device
        self.input_scale = float(input_scale)
        self.offsets = _layout()
        n = self.offsets[-1]
        dev = device
        self.params = torch.zeros(n, dtype=torch.float32, device=dev)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_count = 0
        self.base = torch.zeros((NPIX, OUT), dtype=torch.float32, device=dev)
        bf = torch.bfloat16
        self.F = torch.empty((NROWS, NPIX), dtype=bf, device=dev)
        self.G = torch.empty((NPIX, NROWS), dtype=bf, device=dev)
        self.FT = torch.empty((NPIX, NROWS), dtype=bf, device=dev)
        self.GT = torch.empty((NROWS, NPIX), dtype=bf, device=dev)
        _lib.check(_lib.load().mm_surrogate_constants(self.F.data_ptr(), self.G.data_ptr(), self.FT.data_ptr(),
                                                       self.GT.data_ptr(), _lib.stream_of(dev)), "constants")
        self.wb = [torch.empty((WIDTH, WIDTH), dtype=bf, device=dev) for _ in range(LAYERS)]
        self.wtb = [torch.empty((WIDTH, WIDTH), dtype=bf, device=dev) for _ in range(LAYERS)]
        self.wlb = torch.empty((WIDTH, WIDTH), dtype=bf, device=dev)
        self.wpb = torch.empty((OUT, WIDTH), dtype=bf, device=dev)
        self.wptb = torch.empty((WIDTH, OUT), dtype=bf, device=dev)
        self.mixb = [torch.empty((NROWS // 2 * 64, 64), dtype=bf, device=dev) for _ in range(LAYERS)]
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.loss_buf = torch.zeros(1, dtype=torch.float64, device=dev)
        self._bufs = {}
        self.initialise(seed)

    # ------------------------------------------------------------ parameters
    def view(self, name, t=None):
        i = PARAM_NAMES.index(name)
        t = self.params if t is None else t
        return t[self.offsets[i]:self.offsets[i + 1]].view(PARAM_SHAPES[name])

    def initialise(self, seed):
        """Seeded initial weights: normal(0, 1/sqrt(fan_in)) pointwise weights,
        uniform spectral weights of scale 4/1024, small projection, zero biases."""
        import torch
        g = torch.Generator(device=self.device).manual_seed(int(seed))
        self.params.zero_()
        wl = self.view("Wl")
        wl[:, :18] = torch.randn((WIDTH, 18), generator=g, device=self.device) / math.sqrt(18)
        for l in range(LAYERS):
            self.view(f"W{l}").copy_(torch.randn((WIDTH, WIDTH), generator=g, device=self.device) / math.sqrt(WIDTH))
            for k in ("Rr", "Ri"):
                u = torch.rand(PARAM_SHAPES[f"{k}{l}"], generator=g, device=self.device)
                self.view(f"{k}{l}").copy_((2 * u - 1) * (4.0 / 1024))
        wp = self.view("Wp")
        wp[:PLANES] = torch.randn((PLANES, WIDTH), generator=g, device=self.device) * (0.01 / math.sqrt(WIDTH))
        self.m.zero_()
        self.v.zero_()
        self.step_count = 0

    def numpy_params(self):
        """Parameters as a dict of float64 arrays (names of the network definition)."""
        host = self.params.detach().cpu().numpy().astype(np.float64)
        out = {}
        for i, name in enumerate(PARAM_NAMES):
            out[name] = host[self.offsets[i]:self.offsets[i + 1]].reshape(PARAM_SHAPES[name])
        out["base"] = self.base.detach().cpu().numpy().astype(np.float64)
        return out

    def numpy_grads(self):
        host = self.grads.detach().cpu().numpy().astype(np.float64)
        return {name: host[self.offsets[i]:self.offsets[i + 1]].reshape(PARAM_SHAPES[name])
                for i, name in enumerate(PARAM_NAMES)}

    # --------------------------------------------------------------- buffers
    def _buffers(self, S):
        import torch
        if S in self._bufs:
            return self._bufs[S]
        dev, bf, f32 = self.device, torch.bfloat16, torch.float32
        b = dict(
            hp=[torch.empty((S * NPIX, WIDTH), dtype=bf, device=dev) for _ in range(LAYERS + 1)],
            hc=[torch.empty((S * WIDTH, NPIX), dtype=bf, device=dev) for _ in range(LAYERS + 1)],
            z=[torch.empty((S, NPIX, WIDTH), dtype=f32, device=dev) for _ in range(LAYERS - 1)],
            v=[torch.empty((S, NROWS, WIDTH), dtype=f32, device=dev) for _ in range(LAYERS)],
            voc=torch.empty((S * WIDTH, NROWS), dtype=bf, device=dev),
            vb=torch.empty((NROWS // 2, S, 64), dtype=bf, device=dev),
            y=torch.empty((S, NPIX, OUT), dtype=f32, device=dev),
            dyp=torch.empty((S * NPIX, OUT), dtype=bf, device=dev),
            dyc=torch.empty((S * OUT, NPIX), dtype=bf, device=dev),
            dzp=[torch.empty((S * NPIX, WIDTH), dtype=bf, device=dev) for _ in range(2)],
            dzc=[torch.empty((S * WIDTH, NPIX), dtype=bf, device=dev) for _ in range(2)],
            dvo=torch.empty((S, NROWS, WIDTH), dtype=f32, device=dev),
            dvc=torch.empty((S * WIDTH, NROWS), dtype=bf, device=dev),
        )
        self._bufs[S] = b
        return b

    def _desc(self, S, xp, xc, train=True):
        b = self._buffers(S)
        d = SurrogateDesc()
        d.sites = S
        d.F, d.G, d.FT, d.GT = self.F.data_ptr(), self.G.data_ptr(), self.FT.data_ptr(), self.GT.data_ptr()
        d.params, d.grads = self.params.data_ptr(), self.grads.data_ptr()
        for l in range(LAYERS):
            d.wb[l], d.wtb[l], d.v[l] = self.wb[l].data_ptr(), self.wtb[l].data_ptr(), b["v"][l].data_ptr()
            d.z[l] = b["z"][l].data_ptr() if (train and l < LAYERS - 1) else None
        d.wlb, d.wpb, d.wptb = self.wlb.data_ptr(), self.wpb.data_ptr(), self.wptb.data_ptr()
        d.base = self.base.data_ptr()
        d.xp, d.xc = xp.data_ptr(), xc.data_ptr()
        for l in range(LAYERS + 1):
            d.hp[l], d.hc[l] = b["hp"][l].data_ptr(), b["hc"][l].data_ptr()
        d.voc, d.y = b["voc"].data_ptr(), b["y"].data_ptr()
        d.dyp, d.dyc = b["dyp"].data_ptr(), b["dyc"].data_ptr()
        for k in range(2):
            d.dzp[k], d.dzc[k] = b["dzp"][k].data_ptr(), b["dzc"][k].data_ptr()
        d.dvo, d.dvc = b["dvo"].data_ptr(), b["dvc"].data_ptr()
        d.err = self.err.data_ptr()
        d.vb = b["vb"].data_ptr()
        for l in range(LAYERS):
            d.mixb[l] = self.mixb[l].data_ptr()
        return d, b

    @staticmethod
    def _check_inputs(xp, xc):
        import torch
        if xp.dtype != torch.bfloat16 or xc.dtype != torch.bfloat16:
            raise ValueError("surrogate inputs must be BF16")
        S = xp.shape[0] // NPIX
        if xp.shape != (S * NPIX, WIDTH) or xc.shape != (S * WIDTH, NPIX) or not (xp.is_contiguous()
                                                                                and xc.is_contiguous()):
            raise ValueError(f"inputs must be contiguous (S*4096, 32) and (S*32, 4096), got {tuple(xp.shape)}, "
                             f"{tuple(xc.shape)}")
        return S

    # ------------------------------------------------------------ execution
    def forward(self, xp, xc, *, check=False, train=True):
        """Prediction (S, 4096, 16) FP32 for S sites of pixel- and channel-major
        inputs.  ``train=False`` skips the stores only the backward pass reads."""
        S = self._check_inputs(xp, xc)
        d, b = self._desc(S, xp, xc, train)
        self._d = d
        _lib.check(_lib.load().mm_surrogate_forward(d, int(check), _lib.stream_of(self.device)),
                   "surrogate forward")
        return b["y"]

    def backward(self, xp, xc, target, *, check=False):
        """Loss of the last forward on (xp, xc) and all gradients into ``self.grads``."""
        S = self._check_inputs(xp, xc)
        d, _ = self._desc(S, xp, xc)
        _lib.check(_lib.load().mm_surrogate_backward(d, target.data_ptr(), self.loss_buf.data_ptr(),
                                                      int(check), _lib.stream_of(self.device)), "surrogate backward")
        return self.loss_buf

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        _lib.check(_lib.load().mm_surrogate_adam(self.params.data_ptr(), self.grads.data_ptr(), self.m.data_ptr(),
                                                  self.v.data_ptr(), self.params.numel(), float(lr), float(beta1),
                                                  float(beta2), float(eps), self.step_count,
                                                  _lib.stream_of(self.device)), "surrogate Adam")

    def fit(self, data, *, epochs=20, batch=64, lr=2e-3, lr_final=1e-4, seed=0, log=None):
        """Adam over ``data`` (``training_set`` output) with a cosine learning-rate
        decay; returns the per-epoch mean training loss."""
        import torch
        xp_all = data["xp"].view(-1, NPIX, WIDTH)
        xc_all = data["xc"].view(-1, WIDTH, NPIX)
        t_all = data["t"]
        n = t_all.shape[0]
        if self.step_count == 0:
            self.base.copy_(data["base"])
        g = torch.Generator(device=self.device).manual_seed(int(seed))
        steps = epochs * (n // batch)
        history = []
        k = 0
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g, device=self.device)
            acc = torch.zeros((), dtype=torch.float64, device=self.device)
            for i in range(n // batch):
                idx = perm[i * batch:(i + 1) * batch]
                xp = xp_all[idx].reshape(-1, WIDTH)
                xc = xc_all[idx].reshape(-1, NPIX)
                self.forward(xp, xc)
                acc += self.backward(xp, xc, t_all[idx])[0]
                rate = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * k / max(1, steps)))
                self.adam(rate)
                k += 1
            history.append(float(acc) / max(1, n // batch))
            if log:
                log(f"epoch {ep}: loss {history[-1]:.5f}")
        return history

    def predict(self, xp, xc, *, batch=8192):
        """PSF planes (S, 9, 64, 64) FP32 (negatives clipped) for S sites."""
        import torch
        S = self._check_inputs(xp, xc)
        out = torch.empty((S, PLANES, GRID, GRID), dtype=torch.float32, device=self.device)
        xp3, xc3 = xp.view(S, NPIX, WIDTH), xc.view(S, WIDTH, NPIX)
        for s0 in range(0, S, batch):
            s1 = min(S, s0 + batch)
            xpb, xcb = xp3[s0:s1].reshape(-1, WIDTH), xc3[s0:s1].reshape(-1, NPIX)
            d, _ = self._desc(s1 - s0, xpb, xcb, train=False)
            _lib.check(_lib.load().mm_surrogate_predict(d, out[s0:s1].data_ptr(), 0, _lib.stream_of(self.device)),
                       "surrogate predict")
        return out


# ---------------------------------------------------------------- data
def _device_raw(raw_fields, device):
    import torch
    return [a if isinstance(a, torch.Tensor) and str(a.device).startswith("cuda") else
            torch.as_tensor(np.ascontiguousarray(a, np.float32), device=device) for a in raw_fields]


def site_inputs(raw_fields, offsets, *, scale=1.0, device="cuda", check=True):
    """BF16 inputs (P*4096, 32) and (P*32, 4096) of the sites at window
    ``offsets`` (P, 2) of the raw A/B/C fields: screens in 16 groups, pooled
    4 x 4, times ``scale``, plus two coordinate channels."""
    import torch
    raw = [a.contiguous() for a in _device_raw(raw_fields, device)]
    h, w = raw[0].shape[:2]
    zpart = (ctypes.c_int * 3)(*[int(a.shape[2]) for a in raw])
    groups = (ctypes.c_int * 17)(*screen_groups(sum(zpart)).tolist())
    ptrs = (ctypes.c_void_p * 3)(*[a.data_ptr() for a in raw])
    off = torch.as_tensor(np.ascontiguousarray(offsets, np.int32), device=device)
    P = off.shape[0]
    pooled = torch.empty((GROUPS, h // 4, w // 4), dtype=torch.float32, device=device)
    xp = torch.empty((P * NPIX, WIDTH), dtype=torch.bfloat16, device=device)
    xc = torch.empty((P * WIDTH, NPIX), dtype=torch.bfloat16, device=device)
    err = torch.zeros(1, dtype=torch.int32, device=device)
    _lib.check(_lib.load().mm_surrogate_inputs(ptrs, zpart, h, w, groups, float(scale), pooled.data_ptr(),
                                                off.data_ptr(), P, xp.data_ptr(), xc.data_ptr(), err.data_ptr(),
                                                int(check), _lib.stream_of(device)), "surrogate inputs")
    return xp, xc, pooled


def input_scale(raw_fields, *, device="cuda"):
    """1 / RMS of the pooled screen groups of a volume (the input normalisation)."""
    import torch
    _, _, pooled = site_inputs(raw_fields, np.zeros((0, 2), np.int32), device=device, check=True)
    return float(1.0 / torch.sqrt((pooled.double() ** 2).mean()).clamp_min(1e-30))


def plain_targets(config, raw_fields, points_um, *, device="cuda", plan=None, precision="compensated"):
    """Plain-propagator PSFs of the sites as training targets: (P, 4096, 16)
    FP32 (9 planes, unit sum per site) plus the plan used."""
    import torch
    from .backends.cuda.batched import OpticalPlan
    if plan is None:
        plan = OpticalPlan(surrogate_config(config), raw_fields, device=device, precision=precision)
    pts, off = plan.offsets(points_um)
    res = plan.run_sites(off, tail_per_site=False, slots=64, check=True)
    psf, _, _, _ = plan.finalize_focal(res["focal"])          # (P, 64, 64, Z)
    idx = torch.as_tensor(plane_index(psf.shape[-1]), device=device)
    sel = psf.index_select(3, idx)                              # (P, 64, 64, 9)
    sel = sel / sel.sum((1, 2, 3), keepdim=True).clamp_min(1e-30)
    t = torch.zeros((sel.shape[0], NPIX, OUT), dtype=torch.float32, device=device)
    t[..., :PLANES] = sel.reshape(sel.shape[0], NPIX, PLANES)
    return t, plan, off


def targets_to_planes(t):
    """(P, 4096, 16) targets -> (P, 9, 64, 64) planes."""
    return t[..., :PLANES].permute(0, 2, 1).reshape(t.shape[0], PLANES, GRID, GRID)


def training_set(config, n_sites, *, seeds, device="cuda", sigma=3.0, rms=0.015, scale=None, log=None):
    """(inputs, plain PSF) pairs of ``n_sites`` sites drawn from tissue blocks
    with the given raw-field seeds (every lattice site of each block)."""
    import torch
    from . import synthetic
    from .fixed import field_shapes, fixed_locations
    xs, xcs, ts = [], [], []
    have = 0
    for seed in seeds:
        if have >= n_sites:
            break
        raw = synthetic.raw_fields(config, field_shapes(config), sigma=sigma, rms=rms, seed=int(seed))
        raw_dev = _device_raw(raw, device)
        if scale is None:
            scale = input_scale(raw_dev, device=device)
        pts = fixed_locations(config)[:n_sites - have]
        t, _, off = plain_targets(config, raw_dev, pts, device=device)
        xp, xc, _ = site_inputs(raw_dev, off, scale=scale, device=device)
        xs.append(xp.view(-1, NPIX, WIDTH))
        xcs.append(xc.view(-1, WIDTH, NPIX))
        ts.append(t)
        have += len(pts)
        if log:
            log(f"block seed {seed}: {len(pts)} sites")
    t = torch.cat(ts)
    return {"xp": torch.cat(xs).reshape(-1, WIDTH), "xc": torch.cat(xcs).reshape(-1, NPIX), "t": t,
            "base": t.mean(0), "scale": scale}


def rel_l2_per_site(a, b):
    """Relative L2 error of a against b per site (leading axis), FP64."""
    a = a.reshape(a.shape[0], -1).double()
    b = b.reshape(b.shape[0], -1).double()
    return (a - b).norm(dim=1) / b.norm(dim=1).clamp_min(1e-300)


class SurrogateStage:
    """Surrogate PSFs for every site, gated by the plain propagator on a seeded
    fraction of the sites (whole output replaced by the plain result when the
    sample's relative L2 error exceeds ``tolerance``).

    The gate runs first, on its sites only (their inputs, their predictions
    and their plain PSFs); the surrogate runs on every site only after the
    gate passes.  A failed gate keeps the gate sites' plain PSFs and
    propagates the remaining sites.  Each site's prediction and plain PSF
    depend on that site alone, so both orders give the same output."""

    def __init__(self, model, *, gate_fraction=0.05, tolerance=0.01, seed=0):
        self.model = model
        self.gate_fraction = float(gate_fraction)
        self.tolerance = float(tolerance)
        self.seed = int(seed)

    def gate_sites(self, count):
        k = max(1, int(math.ceil(self.gate_fraction * count)))
        return np.sort(np.random.default_rng(self.seed).choice(count, k, replace=False))

    def run(self, config, raw_fields, points_um, *, plan=None):
        import torch
        dev = self.model.device
        t0 = time.perf_counter()
        raw_dev = _device_raw(raw_fields, dev)
        if plan is None:
            from .backends.cuda.batched import OpticalPlan
            plan = OpticalPlan(surrogate_config(config), raw_dev, device=dev)
        pts, off = plan.offsets(points_um)
        gate = self.gate_sites(len(pts))
        xg, xcg, _ = site_inputs(raw_dev, off[gate], scale=self.model.input_scale, device=dev)
        predicted = self.model.predict(xg, xcg)
        t_gate, _, _ = plain_targets(config, raw_dev, pts[gate], device=dev, plan=plan)
        ref = targets_to_planes(t_gate)
        per_site = rel_l2_per_site(predicted, ref)
        sample = float(rel_l2_per_site(predicted.reshape(1, -1), ref.reshape(1, -1))[0])
        passed = sample <= self.tolerance
        if passed:
            xp, xc, _ = site_inputs(raw_dev, off, scale=self.model.input_scale, device=dev)
            psfs = self.model.predict(xp, xc)
            source = "surrogate"
        else:
            psfs = torch.empty((len(pts), PLANES, GRID, GRID), dtype=torch.float32, device=dev)
            psfs[torch.as_tensor(gate, device=dev)] = ref
            rest = np.setdiff1d(np.arange(len(pts)), gate)
            if len(rest):
                t_rest, _, _ = plain_targets(config, raw_dev, pts[rest], device=dev, plan=plan)
                psfs[torch.as_tensor(rest, device=dev)] = targets_to_planes(t_rest)
            source = "plain"
        torch.cuda.synchronize(dev)
        return {"psfs": psfs, "source": source, "seconds": time.perf_counter() - t0,
                "gate": {"sites": gate, "rel_l2": sample, "max_site_rel_l2": float(per_site.max()),
                         "median_site_rel_l2": float(per_site.median()), "tolerance": self.tolerance,
                         "passed": passed}}
