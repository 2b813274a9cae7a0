"""Layout of the ``stage_bench_lattice`` fixture and its comparison.

The fixture holds the reference's ``maomi.optics.propagate`` products
(optics.py:341-381) at the benchmark geometry for 49 sites: a 7 x 7
sub-lattice of the 65 x 65 site lattice, raw fields from the same seed as the
benchmark's tissue block, so the 49 sites are also sites of the benchmark run.
Used by ``make_golden.py`` (writing), the tests and the benchmark's parity
report (reading).  NumPy only.
"""

import numpy as np

#: raw-field seed of the fixture: the benchmark's tissue block on rank 0
LATTICE_RAW_SEED = 7
#: lattice indices kept on each axis: every tenth from 2 to 62 (symmetric
#: about the centre, so the mask solve takes the reflection-parity path)
LATTICE_INDEX = np.arange(2, 63, 10)
#: sites whose full psf_3d is stored (corners, centre, an off-axis site)
LATTICE_FULL_SITES = np.array([0, 6, 24, 31, 42, 48])
#: width and seed of the per-site random sketch of psf_3d (all 49 sites)
SKETCH_DIM = 32
SKETCH_SEED = 2024
#: seeded mask pixels stored per 512 x 512 mask
MASK_SAMPLES = 4096
MASK_SEED = 77


def lattice_site_index(count_per_axis=65):
    """Row-major indices of the 49 sites within the full lattice's point list."""
    i = LATTICE_INDEX
    return (i[:, None] * count_per_axis + i[None, :]).reshape(-1)


def lattice_points(fixed_locations, cfg):
    """The 7 x 7 sub-lattice of the 65 x 65 site lattice (um)."""
    return fixed_locations(cfg, 65)[lattice_site_index()]


def psf_sketch(psf_3d):
    """Per-site projections of psf_3d on SKETCH_DIM seeded Gaussian vectors:
    the relative L2 of two sketches estimates that of the full arrays."""
    flat = np.asarray(psf_3d, np.float64).reshape(len(psf_3d), -1)
    r = np.random.default_rng(SKETCH_SEED).standard_normal((flat.shape[1], SKETCH_DIM))
    return flat @ r


def mask_pixels(shape):
    """Seeded (row, column) pixel indices at which the masks are stored."""
    rng = np.random.default_rng(MASK_SEED)
    return np.stack([rng.integers(0, shape[0], MASK_SAMPLES), rng.integers(0, shape[1], MASK_SAMPLES)], 1)


def rel_l2(actual, expected):
    a = np.asarray(actual, np.float64)
    b = np.asarray(expected, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def site_errors(psf_3d, d, prefix="f64_"):
    """Per-site products of the 49 sites (psf_3d, energies) against the fixture."""
    psf_3d = np.asarray(psf_3d)
    e = {"psf_3d[sketch]": rel_l2(psf_sketch(psf_3d), d[f"{prefix}psf_sketch"]),
         "energies": rel_l2(psf_3d.sum((1, 2, 3), dtype=np.float64), d[f"{prefix}energies"])}
    norms = np.linalg.norm(psf_3d.astype(np.float64).reshape(len(psf_3d), -1), axis=1)
    e["psf_3d[site norms]"] = rel_l2(norms, d[f"{prefix}psf_site_norm"])
    if f"{prefix}psf_3d_sites" in d:
        e["psf_3d[sites]"] = rel_l2(psf_3d[d["full_sites"]], d[f"{prefix}psf_3d_sites"])
    return e


def stage_errors(out, d, prefix="f64_"):
    """Relative L2 of every propagate() product of a 49-site stage result."""
    ij = d["mask_pixels"]
    px = (ij[:, 0], ij[:, 1])
    e = site_errors(out["psf_3d"], d, prefix)
    e["energies"] = rel_l2(out["energies"], d[f"{prefix}energies"])
    for k in ("psf", "psf_raw", "mask_mean"):
        e[k] = rel_l2(out[k], d[f"{prefix}{k}"])
    e["mask_raw"] = rel_l2(out["mask_raw"][px], d[f"{prefix}mask_raw_px"])
    e["mask"] = rel_l2(out["mask"][px], d[f"{prefix}mask_px"])
    for t in ("psfT", "psfB"):
        for k in ("convmask", "weight", "psfZ", "mask_mean"):
            e[f"{t}.{k}"] = rel_l2(out[t][k], d[f"{prefix}{t}_{k}"])
        e[f"{t}.mask_raw"] = rel_l2(out[t]["mask_raw"][px], d[f"{prefix}{t}_mask_raw_px"])
        e[f"{t}.mask"] = rel_l2(out[t]["mask"][px], d[f"{prefix}{t}_mask_px"])
    return e
