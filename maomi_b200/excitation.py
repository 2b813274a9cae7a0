"""Photon order and the temporal-focusing axial envelope (host-side tables).

Mirrors maomi/excitation.py:5-49: the same scaling names, the same legacy
offset convention of NAOMi's applyTemporalFocusing, float32 tables.
"""

import numpy as np

ORDERS = {"one-photon": 1, "two-photon": 2, "three-photon": 3, "temporal-focusing": 2}


def excitation_order(config):
    """Photon order of ``config.scaling`` (excitation.py:8-11)."""
    try:
        return ORDERS[config.scaling]
    except KeyError:
        raise ValueError(f"Unknown excitation scaling: {config.scaling}") from None


def temporal_profile(size, length_um, dz_um, *, legacy_offset=0.0):
    """Lorentzian-like axial envelope 1/sqrt(1+(i/z_R)^2) (excitation.py:14-29).

    ``legacy_offset`` is multiplied by ``dz_um`` as NAOMi's source does."""
    if (int(size) != size or size < 1
            or not np.isfinite([length_um, dz_um, legacy_offset]).all()
            or min(length_um, dz_um) <= 0):
        raise ValueError("Positive finite axial length and sampling required")
    z_r = length_um / (dz_um * 2.0 * np.sqrt(3.0))
    planes = np.ceil(size / 2) - np.arange(1, size + 1) + legacy_offset * dz_um
    return 1.0 / np.sqrt(1.0 + (planes / z_r) ** 2)


def axial_profile(config, size, part="focus"):
    """Per-plane excitation weight for the focus or a tail (excitation.py:32-49)."""
    if config.scaling != "temporal-focusing":
        return np.ones(size, np.float32)
    if part == "focus":
        dz_um, offset = 1.0 / config.vres, 0.0
    else:
        slab = config.prop_um * config.vres
        depth = config.psf_um[2] * config.vres
        dz_um = slab / config.vres
        if part == "top":
            offset = (depth * config.vres + 2 * slab) / (slab * slab)
        else:
            offset = -depth * config.vres / (slab * slab)
    return temporal_profile(size, config.temporal_length_um, dz_um, legacy_offset=offset).astype(np.float32)
