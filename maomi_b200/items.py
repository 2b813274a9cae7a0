"""Uneven propagation workloads: many independent sites of mixed window size
and depth through per-site phase screens, one persistent launch per window
size (all of them captured in one CUDA graph), schedule chosen by an
autotuner.

An item is the split-step loop of maomi/numerics.py:189-206 with constant
pitch: ``u <- IDFT2(Q * DFT2(u * exp(1j*phase_k)))`` for k = 0..steps-1, where
``Q`` is the angular-spectrum transfer function of one slice (its phase formed
in FP64).  The reference has no batching across items; it would call
``fresnel`` once per item.
"""

import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .backends.cuda.batched import transfer_kernels

SIZES = (64, 128, 256, 512)


@dataclass
class ItemClass:
    """All items of one window size, laid out for the device queue."""
    n: int
    steps: np.ndarray                 # (k,) int, sorted by depth (deepest first)
    order: np.ndarray                 # (k,) original item indices
    phase: object                     # device float32, flat (sum steps*n*n)
    offsets: object                   # device int64 (k,)
    field_in: object                  # device complex64 (n, n)
    kernel: object                    # device complex64 (n,)
    out: object = None                # device complex64 (k, n, n)
    slots: int = 32
    shape: int = 0
    tables: dict = field(default_factory=dict)
    workspace: object = None


def schedule(steps, slots, nblocks):
    """Wave tables of the queue: items run in waves of `slots`; a wave's
    queue holds (levels x slots x blocks) work items, levels = deepest item
    + 1; each slot's counter starts a wave at the blocks all earlier items in
    that slot completed."""
    steps = np.asarray(steps, np.int64)
    k = len(steps)
    waves = max(1, -(-k // slots))
    padded = np.full(waves * slots, -1, np.int64)
    padded[:k] = steps
    grid = padded.reshape(waves, slots)
    levels = grid.max(1) + 1
    wave_items = np.concatenate([[0], np.cumsum(levels * slots * nblocks)])
    done = np.where(grid >= 0, (grid + 1) * nblocks, 0)
    slot_base = np.vstack([np.zeros((1, slots), np.int64), np.cumsum(done, 0)[:-1]])
    return dict(waves=waves, wave_items=wave_items.astype(np.int64), wave_levels=levels.astype(np.int32),
                slot_base=slot_base.reshape(-1).astype(np.int32), total=int(wave_items[-1]))


class ItemQueue:
    """Device-side uneven workload with one queue per window size."""

    def __init__(self, classes, *, device="cuda", precision="compensated"):
        _lib.require_cuda(device)
        if precision not in _lib.PRECISIONS:
            raise ValueError("precision must be one of " + ", ".join(_lib.PRECISIONS))
        self.device, self.precision = device, precision
        self.classes = [c for c in classes if len(c.steps)]
        self.graph = None
        self.tuning = {}
        for c in self.classes:
            self._prepare(c, c.slots, c.shape)

    # ----------------------------------------------------------------- setup
    def _prepare(self, c, slots, shape):
        import torch
        if c.n == 512:
            shape = 0
        c.slots, c.shape = int(max(1, min(slots, len(c.steps)))), int(shape)
        nblocks = _lib.load().mm_items_blocks(c.n, c.shape)
        t = schedule(c.steps, c.slots, nblocks)
        dev = self.device
        c.tables = dict(t, wave_items_d=torch.as_tensor(t["wave_items"], device=dev),
                        wave_levels_d=torch.as_tensor(t["wave_levels"], device=dev),
                        slot_base_d=torch.as_tensor(t["slot_base"], device=dev),
                        steps_d=torch.as_tensor(c.steps.astype(np.int32), device=dev))
        if c.out is None:
            c.out = torch.empty((len(c.steps), c.n, c.n), dtype=torch.complex64, device=dev)
        desc = self._desc(c)
        nbytes = _lib.load().mm_propagate_items_workspace_size(desc)
        c.workspace = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)

    def _desc(self, c):
        d = _lib.ItemClass()
        t = c.tables
        d.n, d.nitems, d.slots, d.waves, d.total_items = c.n, len(c.steps), c.slots, t["waves"], t["total"]
        d.steps, d.phase_offset, d.phase = t["steps_d"].data_ptr(), c.offsets.data_ptr(), c.phase.data_ptr()
        d.field_in, d.field_out, d.kernel = c.field_in.data_ptr(), c.out.data_ptr(), c.kernel.data_ptr()
        d.edge1d = None
        d.wave_items, d.wave_levels, d.slot_base = (t["wave_items_d"].data_ptr(), t["wave_levels_d"].data_ptr(),
                                                    t["slot_base_d"].data_ptr())
        d.precision, d.shape = _lib.PRECISIONS[self.precision], c.shape
        return d

    def _launch(self, c, check):
        base = (c.workspace.data_ptr() + 255) // 256 * 256
        desc = self._desc(c)
        _lib.check(_lib.load().mm_propagate_items(desc, _lib.c_void_p(base), c.workspace.numel() - 256, int(check),
                                                 _lib.stream_of(self.device)), f"items n={c.n}")

    # ------------------------------------------------------------ execution
    def run(self, *, check=True):
        """All classes on concurrent streams (eager)."""
        import torch
        main = torch.cuda.current_stream(self.device)
        streams = [torch.cuda.Stream(self.device) for _ in self.classes]
        for s, c in zip(streams, self.classes):
            s.wait_stream(main)
            with torch.cuda.stream(s):
                self._launch(c, check)
        for s in streams:
            main.wait_stream(s)

    def capture(self):
        """One CUDA graph holding every class's persistent launch."""
        import torch
        self.run(check=True)  # warm up: kernel attributes, lazy module loading
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        streams = [torch.cuda.Stream(self.device) for _ in self.classes]
        with torch.cuda.graph(g):
            cur = torch.cuda.current_stream(self.device)
            for s, c in zip(streams, self.classes):
                s.wait_stream(cur)
                with torch.cuda.stream(s):
                    self._launch(c, False)
            for s in streams:
                cur.wait_stream(s)
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    # ------------------------------------------------------------ autotuner
    def autotune(self, *, slots=(16, 32, 64), shapes=(0, 1), sample=96, repeats=2):
        """Pick (CTA shape = radix split per thread, sites in flight) per window
        size by timing each candidate on the class's deepest `sample` items."""
        import torch
        for c in self.classes:
            full = (c.steps, c.offsets, c.out)
            k = min(sample, len(c.steps))
            c.steps, c.offsets = full[0][:k], full[1][:k]
            c.out = full[2][:k]
            best = None
            for shape in (shapes if c.n != 512 else (0,)):
                for sl in slots:
                    self._prepare(c, sl, shape)
                    self._launch(c, True)
                    torch.cuda.synchronize(self.device)
                    t0 = time.perf_counter()
                    for _ in range(repeats):
                        self._launch(c, False)
                    torch.cuda.synchronize(self.device)
                    dt = (time.perf_counter() - t0) / repeats
                    if best is None or dt < best[0]:
                        best = (dt, shape, c.slots)
            c.steps, c.offsets, c.out = full
            self.tuning[c.n] = {"shape": best[1], "slots": best[2], "sample_ms": best[0] * 1e3}
            self._prepare(c, best[2], best[1])
        self.graph = None
        return self.tuning

    def outputs(self):
        """Final fields in the original item order (host complex64 list)."""
        res = {}
        for c in self.classes:
            host = c.out.cpu().numpy()
            for k, i in enumerate(c.order):
                res[int(i)] = host[k]
        return [res[i] for i in sorted(res)]


def gaussian_field(n, waist_px):
    y, x = np.meshgrid(np.arange(n) - n / 2, np.arange(n) - n / 2, indexing="ij")
    u = np.exp(-(x ** 2 + y ** 2) / waist_px ** 2)
    return (u / np.linalg.norm(u)).astype(np.complex64)


def uneven_workload(count=6000, *, seed=17, device="cuda", wavelength_um=0.92, n_medium=1.35, pitch_um=0.5,
                    dz_um=1.0, sizes=SIZES, probs=(0.4, 0.3, 0.2, 0.1), depth=(16, 120), precision="compensated",
                    slots=32):
    """Seeded mixed workload: window sizes drawn from `sizes` with `probs`,
    depths uniform in `depth` (inclusive), per-item refractive-index screens
    (Gaussian-correlated noise, sigma U(1,4) voxels, RMS dn U(0.005,0.02))
    generated on the device; phase per slice = 2*pi*dn*dz/lambda."""
    import torch
    rng = np.random.default_rng(seed)
    n_of = rng.choice(sizes, p=probs, size=count)
    steps = rng.integers(depth[0], depth[1] + 1, size=count)
    sig = rng.uniform(1.0, 4.0, count)
    rms = rng.uniform(0.005, 0.02, count)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    k0 = 2 * np.pi * dz_um / wavelength_um
    classes = []
    for n in sizes:
        idx = np.flatnonzero(n_of == n)
        if not len(idx):
            continue
        idx = idx[np.argsort(-steps[idx], kind="stable")]
        st = steps[idx]
        total = int((st.astype(np.int64) * n * n).sum())
        phase = torch.empty(total, dtype=torch.float32, device=device)
        offs = np.concatenate([[0], np.cumsum(st.astype(np.int64) * n * n)[:-1]])
        f = torch.fft.fftfreq(n, device=device, dtype=torch.float64)
        f2 = f[:, None] ** 2 + f[None, :] ** 2
        for k, i in enumerate(idx):
            noise = torch.randn((int(st[k]), n, n), generator=gen, device=device, dtype=torch.float32)
            filt = torch.exp(-2 * (np.pi * sig[i]) ** 2 * f2).to(torch.complex64)
            g = torch.fft.ifft2(torch.fft.fft2(noise) * filt).real
            g = g / g.pow(2).mean().sqrt()
            phase[offs[k]:offs[k] + int(st[k]) * n * n] = (g * float(rms[i] * k0)).reshape(-1)
        z = np.arange(2) * dz_um * 1e-6
        kern = transfer_kernels(z, n, pitch_um * 1e-6, np.float32(wavelength_um * 1e-6), np.float32(n_medium))[0]
        classes.append(ItemClass(n=n, steps=st, order=idx, phase=phase,
                                 offsets=torch.as_tensor(offs, device=device),
                                 field_in=torch.as_tensor(gaussian_field(n, n / 8), device=device),
                                 kernel=torch.as_tensor(kern, device=device), slots=slots))
    meta = dict(sizes=n_of, steps=steps, sigma=sig, rms=rms, wavelength_um=wavelength_um, n_medium=n_medium,
                pitch_um=pitch_um, dz_um=dz_um)
    return ItemQueue(classes, device=device, precision=precision), meta
