"""Generate golden fixtures by running the REFERENCE implementation (MaoMi 0.8.0b1).

Run in a container where the reference source tree is mounted read-only:

    python tests/golden/make_golden.py <path to the MaoMi source tree>

It imports the reference package from that path (no bytecode is written),
runs its CPU optical stage (``maomi.optics.propagate``, ``v4_interpolate``,
``resize_xy``, ``translate_xy``, ``pupil``), its scattering-field generator
(``prepare_fields``, ``masked_3DGP_test``) and its local
PSF operator (``maomi.rana.RanaOperator``) on seeded inputs, and stores inputs
(where small) and outputs as ``*.npz`` next to this script.  Large inputs are
regenerated from their seeds by ``maomi_b200.synthetic`` and stored only as a
checksum.  The fixtures are what the tests use on machines without the
reference tree.
"""

import sys
from dataclasses import asdict
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(HERE))
from lattice import (LATTICE_FULL_SITES, LATTICE_RAW_SEED, SKETCH_DIM, SKETCH_SEED,  # noqa: E402
                     lattice_points, mask_pixels, psf_sketch)


def _import_reference(path):
    sys.dont_write_bytecode = True
    sys.path.insert(0, str(path))
    sys.path.insert(0, str(REPO))
    import torch  # noqa: F401  (the reference needs it)
    import maomi  # noqa: F401
    return torch


def _cfg_dict(cfg):
    d = asdict(cfg)
    return {k: np.asarray(v) for k, v in d.items()}


def _flat_result(prefix, out):
    flat = {}
    for k in ("psf_3d", "psf_raw", "psf", "mask_raw", "mask", "energies"):
        flat[f"{prefix}{k}"] = np.asarray(out[k])
    flat[f"{prefix}mask_mean"] = np.asarray(out["mask_mean"])
    for t in ("psfT", "psfB"):
        for k in ("convmask", "weight", "psfZ", "mask_raw", "mask_mean"):
            flat[f"{prefix}{t}_{k}"] = np.asarray(out[t][k])
    return flat


def run_stage(torch, cfg, raw, points, *, custom_phase=None, fp64_too=True):
    """Reference CPU stage in FP32 and (optionally) FP64; returns flat dict."""
    from maomi.optics import propagate, pupil
    res = {}
    u32 = pupil(cfg, custom_phase=custom_phase, device="cpu") if custom_phase is not None else pupil(cfg)
    res["pupil32"] = u32.numpy()
    out = propagate(cfg, raw, points, uin=u32, device="cpu")
    res.update(_flat_result("f32_", out))
    if fp64_too:
        old = torch.get_default_dtype()
        torch.set_default_dtype(torch.float64)
        try:
            u64 = pupil(cfg, custom_phase=custom_phase, device="cpu") if custom_phase is not None else pupil(cfg)
            res["pupil64"] = u64.numpy()
            raw64 = [np.asarray(a, np.float64) for a in raw]
            out = propagate(cfg, raw64, points, uin=u64.to(torch.complex128), device="cpu")
            res.update(_flat_result("f64_", out))
        finally:
            torch.set_default_dtype(old)
    return res


def make_stage_small(torch):
    from maomi.optics import OpticalConfig
    from maomi.fixed import field_shapes, fixed_locations
    from maomi_b200 import synthetic
    cfg = synthetic.small_stage_config(OpticalConfig)
    shapes = field_shapes(cfg)
    raw = synthetic.raw_fields(cfg, shapes, sigma=2.0, rms=0.01, seed=1)
    pts = fixed_locations(cfg, 3)
    res = run_stage(torch, cfg, raw, pts)
    res.update(points=pts, raw_seed=np.asarray(1), raw_sigma=np.asarray(2.0), raw_rms=np.asarray(0.01),
               raw_checksum=np.asarray([float(np.sum(a, dtype=np.float64)) for a in raw]))
    res.update({"cfg_" + k: v for k, v in _cfg_dict(cfg).items()})
    return res


def make_stage_reftest(torch):
    """The reference's own GPU-vs-CPU test geometry (n=112, n2=72, ss=2)."""
    from dataclasses import replace
    from maomi.optics import OpticalConfig, prepare_fields, locations
    cfg = OpticalConfig(volume_um=(16.0, 16.0, 10.0), depth_um=20.0, tail_um=10.0)
    pts = locations(cfg.volume_um, 3)
    phase = np.zeros((17, 17), np.float32)
    phase[5:11, 5:11] = 0.2
    res = {}
    raw0 = [a.numpy() for a in prepare_fields(cfg, scatter=False)]
    out = run_stage(torch, cfg, raw0, pts, custom_phase=phase)
    res.update({"flat_" + k: v for k, v in out.items()})
    raw1 = [a.numpy() for a in prepare_fields(cfg, scatter=True)]
    for i, a in enumerate(raw1):
        res[f"raw{i}"] = a
    for mode in ("two-photon", "three-photon", "temporal-focusing"):
        c = replace(cfg, scaling=mode)
        out = run_stage(torch, c, raw1, pts, custom_phase=phase)
        res.update({f"{mode}_" + k: v for k, v in out.items()})
    res.update(points=pts, custom_phase=phase)
    res.update({"cfg_" + k: v for k, v in _cfg_dict(cfg).items()})
    return res


def make_stage_bench_sites(torch):
    """Benchmark geometry (n=256, 60 screens, Zernike pupil) on three sites."""
    from maomi.optics import OpticalConfig, pupil
    from maomi.optics import propagate
    from maomi.fixed import field_shapes
    from maomi_b200 import synthetic
    cfg = synthetic.benchmark_stage_config(OpticalConfig)
    shapes = field_shapes(cfg)
    raw = synthetic.raw_fields(cfg, shapes, sigma=3.0, rms=0.015, seed=7)
    pts = np.array([[0.0, 0.0], [128.0, 128.0], [252.0, 4.0]])
    res = {}
    u32 = pupil(cfg)
    res["pupil32"] = u32.numpy()
    out = propagate(cfg, raw, pts, uin=u32, device="cpu")
    res.update(_flat_result("f32_", out))
    old = torch.get_default_dtype()
    torch.set_default_dtype(torch.float64)
    try:
        u64 = pupil(cfg)
        res["pupil64"] = u64.numpy()
        out = propagate(cfg, [np.asarray(a, np.float64) for a in raw], pts,
                        uin=u64.to(torch.complex128), device="cpu")
        res.update(_flat_result("f64_", out))
    finally:
        torch.set_default_dtype(old)
    # Three sites make a degenerate v4 mask and the pupils are pinned in the
    # numerics fixture: keep only the per-site products.
    for k in list(res):
        if k.startswith("pupil") or "mask" in k or k.endswith(("psf_raw", "_psf")):
            del res[k]
    res.update(points=pts, raw_seed=np.asarray(7), raw_sigma=np.asarray(3.0), raw_rms=np.asarray(0.015),
               raw_checksum=np.asarray([float(np.sum(a, dtype=np.float64)) for a in raw]))
    res.update({"cfg_" + k: v for k, v in _cfg_dict(cfg).items()})
    return res


def _lattice_result(prefix, out, full_psf):
    ij = mask_pixels(np.shape(out["mask_raw"]))
    flat = {f"{prefix}energies": np.asarray(out["energies"]),
            f"{prefix}psf_sketch": psf_sketch(out["psf_3d"]),
            f"{prefix}psf_site_norm": np.linalg.norm(np.asarray(out["psf_3d"], np.float64).reshape(
                len(out["energies"]), -1), axis=1),
            f"{prefix}psf": np.asarray(out["psf"], np.float32),
            f"{prefix}psf_raw": np.asarray(out["psf_raw"], np.float32),
            f"{prefix}mask_raw_px": out["mask_raw"][ij[:, 0], ij[:, 1]],
            f"{prefix}mask_px": out["mask"][ij[:, 0], ij[:, 1]],
            f"{prefix}mask_mean": np.asarray(out["mask_mean"]),
            f"{prefix}negative_resampling_mass_fraction": np.asarray(out["negative_resampling_mass_fraction"])}
    if full_psf:
        flat[f"{prefix}psf_3d_sites"] = np.asarray(out["psf_3d"][LATTICE_FULL_SITES], np.float32)
    for t in ("psfT", "psfB"):
        tail = out[t]
        flat[f"{prefix}{t}_convmask"] = np.asarray(tail["convmask"], np.float32)
        flat[f"{prefix}{t}_weight"] = np.asarray(tail["weight"])
        flat[f"{prefix}{t}_psfZ"] = np.asarray(tail["psfZ"])
        flat[f"{prefix}{t}_mask_raw_px"] = tail["mask_raw"][ij[:, 0], ij[:, 1]]
        flat[f"{prefix}{t}_mask_px"] = tail["mask"][ij[:, 0], ij[:, 1]]
        flat[f"{prefix}{t}_mask_mean"] = np.asarray(tail["mask_mean"])
    return flat


def make_stage_bench_lattice(torch):
    """Benchmark geometry (n=256, 60 screens, Zernike pupil, scattering
    screens sigma=3 vox / RMS 0.015) on a 7 x 7 sub-lattice of the 65 x 65
    site lattice: every product of ``maomi.optics.propagate`` in FP64 and
    FP32.  psf_3d is stored in full for six sites and as a per-site sketch for
    all 49; the 512 x 512 masks at 4,096 seeded pixels plus their means
    (FP64 values rounded to float32 where marked)."""
    from maomi.optics import OpticalConfig, pupil, propagate
    from maomi.fixed import field_shapes, fixed_locations
    from maomi_b200 import synthetic
    cfg = synthetic.benchmark_stage_config(OpticalConfig)
    raw = synthetic.raw_fields(cfg, field_shapes(cfg), sigma=3.0, rms=0.015, seed=LATTICE_RAW_SEED)
    pts = lattice_points(fixed_locations, cfg)
    res = {}
    out = propagate(cfg, raw, pts, uin=pupil(cfg), device="cpu")
    res.update(_lattice_result("f32_", out, full_psf=False))
    old = torch.get_default_dtype()
    torch.set_default_dtype(torch.float64)
    try:
        u64 = pupil(cfg)
        out = propagate(cfg, [np.asarray(a, np.float64) for a in raw], pts, uin=u64.to(torch.complex128),
                        device="cpu")
        res.update(_lattice_result("f64_", out, full_psf=True))
    finally:
        torch.set_default_dtype(old)
    res.update(points=pts, full_sites=LATTICE_FULL_SITES, mask_pixels=mask_pixels(out["mask_raw"].shape),
               sketch_dim=np.asarray(SKETCH_DIM), sketch_seed=np.asarray(SKETCH_SEED),
               raw_seed=np.asarray(LATTICE_RAW_SEED), raw_sigma=np.asarray(3.0), raw_rms=np.asarray(0.015),
               raw_checksum=np.asarray([float(np.sum(a, dtype=np.float64)) for a in raw]))
    res.update({"cfg_" + k: v for k, v in _cfg_dict(cfg).items()})
    return res


def make_numerics(torch):
    from maomi.numerics import resize_xy, translate_xy, v4_interpolate
    from maomi._propagation import edge_apodization
    from maomi.excitation import axial_profile
    from maomi.optics import OpticalConfig
    rng = np.random.default_rng(12)
    res = {}
    a = rng.standard_normal((20, 18, 3)).astype(np.float32)
    res["resize_in"] = a
    for s in (2, 0.5, 3):
        res[f"resize_{s}"] = resize_xy(torch.as_tensor(a), s).numpy()
        res[f"resize64_{s}"] = resize_xy(torch.as_tensor(a.astype(np.float64)), s).numpy()
    for sh in (0.5, 1.0, 0.0):
        res[f"translate_{sh}"] = translate_xy(torch.as_tensor(a.astype(np.float64)), sh).numpy()
    res["edge_64"] = edge_apodization(64, "cpu", torch.float64).numpy()
    res["edge_32"] = edge_apodization(64, "cpu", torch.float32).numpy()
    # Zernike-aberrated pupils (modes 4-11) on a 96-point grid, both precisions
    from maomi.optics import pupil
    from maomi_b200 import synthetic
    from dataclasses import replace
    zc = OpticalConfig(volume_um=(16.0, 16.0, 10.0), depth_um=12.0, vres=1.0, ss=1)
    zc = replace(zc, zernike_weights=synthetic.zernike_weights(zc, 3))
    res["zpupil32"] = pupil(zc).numpy()
    old = torch.get_default_dtype()
    torch.set_default_dtype(torch.float64)
    try:
        res["zpupil64"] = pupil(zc).numpy()
    finally:
        torch.set_default_dtype(old)
    res.update({"zcfg_" + k: v for k, v in _cfg_dict(zc).items()})
    cfg = OpticalConfig(scaling="temporal-focusing")
    for part, size in (("focus", 20), ("top", 7), ("bottom", 5)):
        res[f"axial_{part}"] = axial_profile(cfg, size, part)
    # v4: the reference test's data (tests/test_interpolation.py:21-25)
    rng = np.random.default_rng(471)
    pts = rng.uniform(-20, 20, (37, 2))
    q = np.concatenate((pts, rng.uniform(-25, 25, (105, 2))))
    vals = rng.uniform(.2, 2, (37, 4))
    res.update(v4_points=pts, v4_queries=q, v4_values=vals,
               v4_out=v4_interpolate(pts, vals, q, chunk=19, backend="cpu"))
    # a lattice case shaped like mask assembly (9x9 sites -> 64x64 pixels)
    lat = np.stack(np.meshgrid(np.arange(9) * 8.0, np.arange(9) * 8.0, indexing="ij"), -1).reshape(-1, 2)
    lv = rng.uniform(.5, 2, (81, 3))
    lq = np.stack(np.meshgrid(np.arange(64) + .5, np.arange(64) + .5, indexing="ij"), -1)
    res.update(v4l_points=lat, v4l_values=lv, v4l_out=v4_interpolate(lat, lv, lq, backend="cpu"))
    return res


def make_local_fft(torch):
    from maomi.rana import FullFieldPSF, DepthPSFBank, RanaOperator
    from maomi.rana._fft import LocalFFTPlan
    from maomi.rana.operator import _axis_weights
    rng = np.random.default_rng(631)
    res = {}
    # (a) small native-style field, reference test fixture shapes
    vol = rng.uniform(0, 1, (12, 14, 9))
    k = rng.uniform(.1, 1, (2, 2, 3, 4, 3))
    res.update(a_volume=vol, a_kernels=k)
    for name, op in (("excitation", "excitation"), ("detection", "detection")):
        f = FullFieldPSF(k, [0, 12], [0, 14], (1., 1., 1.), 920., op)
        R = RanaOperator(f, device="cpu")
        res[f"a_{name}_static"] = R.static(vol)
        res[f"a_{name}_slab1"] = R.scan_slab(vol[..., :3], scan_avg=1)
        res[f"a_{name}_slab2"] = R.scan_slab(vol[..., :3], scan_avg=2)
        Rn = RanaOperator(f, native=True, device="cpu")
        res[f"a_{name}_native_static"] = Rn.static(vol)
    # (b) mid-size: 48x40x10 volume, 4x3 nodes, 7x6x5 kernels, 2-depth bank, even/odd sizes
    vol = rng.uniform(0, 2, (48, 40, 10))
    kern = rng.uniform(.05, 1, (2, 4, 3, 7, 6, 5))
    xs, ys = np.linspace(0, 48, 4), np.linspace(0, 40, 3)
    res.update(b_volume=vol, b_kernels=kern, b_x=xs, b_y=ys, b_depths=np.array([0.0, 10.0]))
    for op in ("excitation", "detection"):
        fields = tuple(FullFieldPSF(kern[d], xs, ys, (1., 1., 1.), 920., op) for d in range(2))
        bank = DepthPSFBank(np.array([0.0, 10.0]), fields)
        R = RanaOperator(bank, device="cpu")
        res[f"b_{op}_static"] = R.static(vol)
        res[f"b_{op}_slab"] = R.scan_slab(vol[..., 2:7], z_start=2, scan_avg=1)
    # (c) the weights helper
    nodes = np.array([0.0, 3.0, 10.0, 12.0])
    pos = np.linspace(-1, 13, 29)
    res.update(c_nodes=nodes, c_pos=pos, c_weights=_axis_weights(nodes, pos))
    return res


def make_fields(torch):
    """The scattering-field generator: masked_3DGP_test on odd and even grids
    (the noise is re-drawn by the tests from the recorded seed: real parts,
    then imaginary parts) and prepare_fields with a vessel occupancy volume."""
    from maomi import _optical_math as legacy
    from maomi.optics import OpticalConfig, prepare_fields
    res = {}
    for tag, shape, ls, p_scale in (("odd", (15, 22, 7), [[2.0, 3.0, 0.8], [5.0, 1.5, 2.5]], 3.0),
                                    ("even", (24, 16, 6), [[1.2, 1.2, 0.4]], 1.0)):
        seed = 1234 + len(tag)
        torch.manual_seed(seed)
        l = torch.tensor(ls, dtype=torch.float32)
        w = torch.tensor([0.7, 0.3][:len(ls)], dtype=torch.float32)
        out = legacy.masked_3DGP_test(shape, l, p_scale, l_weights=w, device="cpu")
        res.update({f"{tag}_shape": np.array(shape), f"{tag}_ls": np.array(ls, np.float32), f"{tag}_w": w.numpy(),
                    f"{tag}_p": np.float64(p_scale), f"{tag}_seed": np.int64(seed), f"{tag}_out": out.numpy()})
    cfg = OpticalConfig(volume_um=(16.0, 16.0, 10.0), depth_um=20.0, tail_um=10.0)
    rng = np.random.default_rng(5)
    vessels = (rng.random((72, 72, 45)) < 0.05).astype(np.float32)
    raw = [a.numpy() for a in prepare_fields(cfg, vessels, scatter=True)]
    res.update({f"vessel_raw{i}": a for i, a in enumerate(raw)})
    res["vessels_seed"] = np.int64(5)
    res.update({"cfg_" + k: v for k, v in _cfg_dict(cfg).items()})
    return res


def make_rana_files(torch):
    """Files written by the reference's own FullFieldPSF.save / DepthPSFBank.save
    (maomi/rana/fields.py:96-110, depth.py:50-69) for the format round trips.
    Writes ref_full_field_psf.npz and ref_depth_psf_bank.npz next to this
    script; returns the inputs that built them."""
    from maomi.rana import DepthPSFBank, FullFieldPSF
    rng = np.random.default_rng(808)
    k = rng.uniform(0.1, 1.0, (2, 3, 5, 4, 3))
    x, y = np.array([0.0, 7.5]), np.array([-2.0, 1.0, 6.0])
    f = FullFieldPSF(k, x, y, (0.5, 0.5, 1.0), 920.0, "excitation", {"note": "reference-written", "n": 3})
    f.save(HERE / "ref_full_field_psf.npz")
    ks = rng.uniform(0.1, 1.0, (2, 2, 3, 5, 4, 3))
    fields = tuple(FullFieldPSF(ks[i], x, y, (0.5, 0.5, 1.0), 920.0, "detection", {"depth": i}) for i in range(2))
    DepthPSFBank(np.array([1.0, 9.0]), fields).save(HERE / "ref_depth_psf_bank.npz")
    return {"field_kernels": k, "bank_kernels": ks, "x_um": x, "y_um": y}


def make_scanning(torch):
    """The reference's static and per-frame scan operators on seeded inputs:
    ``zstack`` (maomi/scanning.py:8-53, both modes, with and without masks, FP64
    and FP32), ``single_scan`` with ``psf_fft`` (maomi/movie.py:37-66, grouped
    and ungrouped) and ``blurred_background`` (movie.py:69-102, spatial and
    frequency kernels)."""
    from maomi.movie import blurred_background, psf_fft, single_scan
    from maomi.scanning import zstack
    rng = np.random.default_rng(909)
    out = {}
    # odd/even kernel sizes, kernels wider than half the volume, ragged Z
    cases = [((23, 30, 17), (6, 5, 7)), ((32, 32, 12), (9, 10, 4)), ((40, 36, 9), (33, 33, 9))]
    for i, (vs, ks) in enumerate(cases):
        v = rng.uniform(0, 1, vs)
        p = rng.uniform(0, 1, ks)
        m1 = rng.uniform(0.5, 1.5, vs[:2])
        m2 = rng.uniform(0.2, 1.0, vs[:2])
        out[f"z{i}_volume"], out[f"z{i}_psf"], out[f"z{i}_mask"], out[f"z{i}_colmask"] = v, p, m1, m2
        out[f"z{i}_convn64"] = zstack(v, p, mask=m1, collection_mask=m2).numpy()
        out[f"z{i}_convn32"] = zstack(v.astype(np.float32), p.astype(np.float32), mask=m1,
                                      collection_mask=m2).numpy()
        out[f"z{i}_plain64"] = zstack(v, p).numpy()
        out[f"z{i}_legacy64"] = zstack(v, p, mode="legacy_circular").numpy()
    # single_scan: slab depth == PSF depth, grouped planes
    for i, (vs, ks) in enumerate([((30, 26, 8), (7, 6, 8)), ((48, 40, 9), (12, 11, 9))]):
        v = rng.uniform(0, 1, vs).astype(np.float32)
        p = rng.uniform(0, 1, ks).astype(np.float32)
        out[f"s{i}_volume"], out[f"s{i}_psf"] = v, p
        for g in (1, 2, 3):
            out[f"s{i}_g{g}"] = single_scan(v, p, scan_avg=g)
            out[f"s{i}_g{g}_freq"] = single_scan(v, p, scan_avg=g, frequency_psf=psf_fft(v.shape, p, g))
    # blurred_background: frame volume, planes above / below a slab, tail kernel
    v = rng.uniform(0, 1, (36, 28, 14)).astype(np.float32)
    extra = rng.uniform(0, 1, v.shape).astype(np.float32)
    kern = rng.uniform(0, 1, (16, 16)).astype(np.float32)
    kern /= kern.sum()
    mask = rng.uniform(0.5, 1.5, v.shape[:2]).astype(np.float32)
    zs = rng.uniform(0.5, 2.0, 9)
    out.update(b_volume=v, b_extra=extra, b_kernel=kern, b_mask=mask, b_zscale=zs)
    for name, idx in (("top", np.arange(5)), ("bottom", np.arange(9, 14))):
        kw = dict(power_ratio=0.37, mask=mask, zscale=zs[:len(idx)], extra_volumes=[extra])
        out[f"b_{name}_spatial"] = blurred_background(v, idx, kern, **kw)
        spec = psf_fft(v.shape, kern)
        out[f"b_{name}_freq"] = blurred_background(v, idx, spec, frequency=True, **kw)
        out[f"b_{name}_freq_shape"] = np.asarray(spec.shape)
    return out


def make_collection(torch):
    """The reference's collection mask (maomi/optics.py:384-409) and its
    vessel-aware scattering fields (optics.py:120-197, zero scatter) for seeded
    vessel occupancies on two geometries: the reference's own test geometry
    and the small benchmark-recipe geometry."""
    from maomi.optics import OpticalConfig, collection_mask, prepare_fields
    sys.path.insert(0, str(REPO))
    from maomi_b200 import synthetic
    out = {}
    cfgs = [OpticalConfig(volume_um=(16.0, 16.0, 10.0), depth_um=20.0, tail_um=10.0),
            synthetic.small_stage_config(OpticalConfig)]
    rng = np.random.default_rng(1234)
    for i, cfg in enumerate(cfgs):
        r = cfg.vres
        shapes = [tuple(a.shape) for a in prepare_fields(cfg, scatter=False)]
        za = int(round((cfg.depth_um + cfg.volume_um[2] / 2 - cfg.psf_um[2] / 2) * r))
        zb = int(round(cfg.psf_um[2] * r))
        nc = int(round(cfg.tail_um * r))
        vshape = (shapes[0][0], shapes[0][1], za + zb + nc + 3)
        ves = (rng.uniform(0, 1, vshape) > 0.85).astype(np.uint8)
        out[f"c{i}_vessels"] = ves
        out[f"c{i}_colmask"] = collection_mask(ves.astype(np.float32), cfg)
        for j, a in enumerate(prepare_fields(cfg, ves.astype(np.float32), scatter=False)):
            out[f"c{i}_raw{j}"] = a.numpy()
        out.update({f"c{i}_cfg_" + k: v for k, v in _cfg_dict(cfg).items()})
    return out


def make_cubic(torch):
    """The reference's global cubic-RBF renderers on seeded fields:
    ``CubicFullFieldRenderer`` (maomi/rana/fields.py:113-276) for 2-D and 3-D
    shapes, both operators, even and odd kernels, a non-affine knot and a
    16 x 16-node field; ``DepthFullFieldRenderer`` (maomi/rana/depth.py:72-104)
    with uniform and varying XY fields."""
    from maomi.rana.depth import DepthFullFieldRenderer, DepthPSFBank
    from maomi.rana.fields import CubicFullFieldRenderer, FullFieldPSF
    out = {}
    rng = np.random.default_rng(47)
    case = 0
    for shape in [(5, 4), (4, 3, 3)]:
        for kshape in [(3,) * len(shape), (4, 2) + ((2,) if len(shape) == 3 else ())]:
            for op in ("detection", "excitation"):
                r = np.random.default_rng(18)
                base, dx, dy = r.uniform(.2, 1, kshape), r.uniform(0, .5, kshape), r.uniform(0, .4, kshape)
                x, y = np.linspace(0, shape[0], 3), np.linspace(0, shape[1], 3)
                k = np.array([[base + xx / shape[0] * dx + yy / shape[1] * dy for yy in y] for xx in x])
                a = rng.uniform(0, 2, shape)
                f = FullFieldPSF(k, x, y, (1.,) * len(shape), 920., op)
                out.update({f"k{case}_kernels": k, f"k{case}_x": x, f"k{case}_y": y, f"k{case}_density": a,
                            f"k{case}_op": np.asarray(op),
                            f"k{case}_image": CubicFullFieldRenderer(f, shape, voxel_size_um=(1,) * len(shape))(a)})
                case += 1
    # non-affine knot, and a 16 x 16-node varying field with an origin offset
    k = out["k0_kernels"].copy()
    k[1, 1] *= 1.15
    a = np.random.default_rng(12).uniform(0, 1, (5, 4))
    f = FullFieldPSF(k, out["k0_x"], out["k0_y"], (1, 1), 920, "detection")
    out.update({f"k{case}_kernels": k, f"k{case}_x": out["k0_x"], f"k{case}_y": out["k0_y"], f"k{case}_density": a,
                f"k{case}_op": np.asarray("detection"),
                f"k{case}_image": CubicFullFieldRenderer(f, (5, 4), voxel_size_um=(1, 1))(a)})
    case += 1
    r = np.random.default_rng(33)
    x, y = np.linspace(0, 48, 16) + 2.0, np.linspace(0, 40, 16) - 1.0
    base = r.uniform(.5, 1, (7, 7, 3))
    k = np.array([[base * (1 + .2 * np.sin(xx / 9) * np.cos(yy / 7)) + .05 * r.uniform(0, 1, base.shape)
                   for yy in y] for xx in x])
    for op in ("detection", "excitation"):
        a = r.uniform(0, 1, (48, 40, 6))
        f = FullFieldPSF(k, x, y, (1., 1., 1.), 920., op)
        img = CubicFullFieldRenderer(f, a.shape, voxel_size_um=(1, 1, 1), origin_um=(2.0, -1.0))(a)
        out.update({f"k{case}_kernels": k, f"k{case}_x": x, f"k{case}_y": y, f"k{case}_density": a,
                    f"k{case}_op": np.asarray(op), f"k{case}_origin": np.array([2.0, -1.0]), f"k{case}_image": img})
        case += 1
    out["cases"] = np.asarray(case)
    # depth banks: uniform XY (exact constant basis) and varying XY
    depths = np.array([0.0, 3.0, 8.0])
    for name, vary in (("uniform", False), ("varying", True)):
        for op in ("detection", "excitation"):
            r = np.random.default_rng(71)
            x, y = np.array([0.0, 12.0, 24.0]), np.array([0.0, 10.0, 20.0])
            kern = []
            for d in depths:
                b = r.uniform(.3, 1, (5, 5, 3)) * (1 + d / 10)
                kern.append(np.array([[b * ((1 + .1 * xx / 24 + .05 * yy / 20) if vary else 1) for yy in y]
                                      for xx in x]))
            bank = DepthPSFBank(depths, tuple(FullFieldPSF(kk, x, y, (1., 1., 1.), 920., op) for kk in kern))
            a = r.uniform(0, 1, (24, 20, 8))
            img = DepthFullFieldRenderer(bank, a.shape, voxel_size_um=(1., 1., 1.))(a)
            out.update({f"d_{name}_{op}_kernels": np.stack(kern), f"d_{name}_{op}_density": a,
                        f"d_{name}_{op}_image": img})
    out.update(d_depths=depths, d_x=np.array([0.0, 12.0, 24.0]), d_y=np.array([0.0, 10.0, 20.0]))
    return out


MAKERS = (("numerics", make_numerics), ("local_fft", make_local_fft), ("stage_small", make_stage_small),
          ("stage_reftest", make_stage_reftest), ("stage_bench_sites", make_stage_bench_sites),
          ("fields", make_fields), ("stage_bench_lattice", make_stage_bench_lattice), ("rana_files", make_rana_files),
          ("scanning", make_scanning), ("collection", make_collection),
          ("cubic", make_cubic))


def main(ref_path, only=None):
    torch = _import_reference(ref_path)
    torch.set_num_threads(8)
    for name, fn in MAKERS:
        if only and name not in only:
            continue
        out = fn(torch)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(name, sum(np.asarray(v).nbytes for v in out.values()) // 1024, "KiB raw")


if __name__ == "__main__":
    # make_golden.py <reference source tree> [fixture names...]
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <path to the MaoMi source tree> [fixture names...]")
    main(sys.argv[1], sys.argv[2:] or None)
