"""ctypes binding of ``libmaomi_b200.so`` (the C ABI in ``include/maomi_b200.h``).

The library is built in-tree (``python -m maomi_b200.build``).  There is no
fallback: if the library or a CUDA device is missing every entry point raises.
"""

import ctypes
from ctypes import POINTER, Structure, c_double, c_float, c_int, c_size_t, c_void_p, c_char_p
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libmaomi_b200.so"

MM_OK, MM_ERR_ARGUMENT, MM_ERR_CUDA, MM_ERR_TIMEOUT, MM_ERR_NONFINITE, MM_ERR_UNSUPPORTED = 0, -1, -2, -3, -4, -5
MM_SCHEDULE_PERSISTENT, MM_SCHEDULE_BATCHED = 0, 1
MM_PRECISION_FP32, MM_PRECISION_FP64, MM_PRECISION_MIXED = 0, 1, 2
MM_PRECISION_COMPENSATED, MM_PRECISION_COMPENSATED_FULL = 3, 4
PRECISIONS = {"fp32": MM_PRECISION_FP32, "fp64": MM_PRECISION_FP64, "mixed": MM_PRECISION_MIXED,
              "compensated": MM_PRECISION_COMPENSATED, "compensated-full": MM_PRECISION_COMPENSATED_FULL}

c_int_p = POINTER(c_int)
c_float_p = POINTER(c_float)
c_double_p = POINTER(c_double)


class StageDesc(Structure):
    _fields_ = [("size", c_int), ("steps", c_int), ("screens", c_void_p), ("vol_h", c_int), ("vol_w", c_int),
                ("edge1d", c_void_p), ("kernels", c_void_p)]


class StagePlan(Structure):
    _fields_ = [("stage", StageDesc * 3), ("base", c_void_p), ("n", c_int), ("n2", c_int), ("order", c_int),
                ("cut", c_int), ("focal_x0", c_int), ("focal_y0", c_int), ("focal_h", c_int), ("focal_w", c_int),
                ("tail_weight", c_void_p * 2), ("focal", c_void_p), ("tail_image", c_void_p * 2),
                ("tail_per_site", c_int), ("tail_profile", c_void_p * 2), ("offsets", c_void_p), ("nsites", c_int),
                ("precision", c_int), ("reserve_sms", c_int), ("hold_site", c_int),
                ("spin_limit", ctypes.c_longlong)]


class ItemClass(Structure):
    _fields_ = [("n", c_int), ("nitems", c_int), ("slots", c_int), ("waves", c_int), ("total_items", ctypes.c_longlong),
                ("steps", c_void_p), ("phase_offset", c_void_p), ("phase", c_void_p), ("field_in", c_void_p),
                ("field_out", c_void_p), ("kernel", c_void_p), ("edge1d", c_void_p), ("wave_items", c_void_p),
                ("wave_levels", c_void_p), ("slot_base", c_void_p), ("precision", c_int), ("shape", c_int)]


class PupilDesc(Structure):
    _fields_ = [("n", c_int), ("pitch", c_double), ("beam_radius", c_double), ("aperture", c_double),
                ("k", c_double), ("focal_length", c_double), ("nmodes", c_int), ("mode_coef", c_double_p),
                ("mode_m", c_int_p), ("mode_cos", c_int_p), ("mode_nterms", c_int_p), ("term_coef", c_double_p),
                ("term_pow", c_int_p), ("custom_phase", c_void_p), ("custom_h", c_int), ("custom_w", c_int),
                ("custom_radius", c_double), ("custom_scale", c_double)]


class BaseDesc(Structure):
    _fields_ = [("n", c_int), ("d1", c_double), ("d2", c_double), ("dz", c_double), ("lambda_medium", c_double),
                ("edge1d", c_void_p)]


class LocalDesc(Structure):
    _fields_ = [("sx", c_int), ("sy", c_int), ("sz", c_int), ("kx", c_int), ("ky", c_int), ("kz", c_int),
                ("nodes_x", c_int), ("nodes_y", c_int), ("kernels", c_void_p), ("wx", c_void_p), ("wy", c_void_p),
                ("detection", c_int), ("correlate", c_int), ("plane", c_int), ("nfields", c_int),
                ("tiles_x", c_void_p), ("ntiles_x", c_int), ("tiles_y", c_void_p), ("ntiles_y", c_int)]


class ScanPlanes(Structure):
    _fields_ = [("data", c_void_p), ("s0", ctypes.c_longlong), ("s1", ctypes.c_longlong), ("s2", ctypes.c_longlong),
                ("nx", c_int), ("ny", c_int), ("nz", c_int), ("group", c_int), ("mask0", c_void_p),
                ("mask1", c_void_p), ("data2", c_void_p)]


class ScanDesc(Structure):
    _fields_ = [("fp64", c_int), ("fx", c_int), ("fy", c_int), ("kx", c_int), ("ky", c_int), ("kplanes", c_int)]


class ScanConv(Structure):
    _fields_ = [("src", ScanPlanes), ("wrap", c_int), ("wrap_x0", c_int), ("wrap_y0", c_int), ("ext_x", c_int),
                ("ext_y", c_int), ("zrule", c_int), ("zoff", c_int), ("out_planes", c_int), ("crop_x", c_int),
                ("crop_y", c_int), ("out_x", c_int), ("out_y", c_int), ("out", c_void_p), ("o0", ctypes.c_longlong),
                ("o1", ctypes.c_longlong), ("o2", ctypes.c_longlong), ("accumulate", c_int), ("alpha", c_double),
                ("src_spectra", c_void_p), ("out_spectra", c_void_p), ("out_weight", c_void_p)]


MM_SCAN_CONV_Z, MM_SCAN_CORR_Z, MM_SCAN_SUM_Z, MM_SCAN_EACH_Z = 0, 1, 2, 3


class SurrogateDesc(ctypes.Structure):
    _fields_ = [("sites", c_int), ("F", c_void_p), ("G", c_void_p), ("FT", c_void_p),
                ("GT", c_void_p), ("params", c_void_p), ("grads", c_void_p),
                ("wb", c_void_p * 4), ("wtb", c_void_p * 4), ("wlb", c_void_p),
                ("wpb", c_void_p), ("wptb", c_void_p), ("base", c_void_p),
                ("xp", c_void_p), ("xc", c_void_p), ("hp", c_void_p * 5),
                ("hc", c_void_p * 5), ("z", c_void_p * 4), ("v", c_void_p * 4),
                ("voc", c_void_p), ("y", c_void_p), ("dyp", c_void_p), ("dyc", c_void_p),
                ("dzp", c_void_p * 2), ("dzc", c_void_p * 2), ("dvo", c_void_p),
                ("dvc", c_void_p), ("err", c_void_p), ("vb", c_void_p), ("mixb", c_void_p * 4)]


# name -> (restype, argtypes)
SIGNATURES = {
    "mm_version": (c_int, []),
    "mm_last_error": (c_char_p, []),
    "mm_device_supported": (c_int, []),
    "mm_launch_count": (ctypes.c_ulonglong, []),
    "mm_struct_size": (ctypes.c_size_t, [c_char_p]),
    "mm_gemm_bf16_tn": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_void_p]),
    "mm_surrogate_layout": (c_int, [c_void_p, c_int]),
    "mm_surrogate_constants": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mm_surrogate_forward": (c_int, [POINTER(SurrogateDesc), c_int, c_void_p]),
    "mm_surrogate_backward": (c_int, [POINTER(SurrogateDesc), c_void_p, c_void_p, c_int, c_void_p]),
    "mm_surrogate_adam": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_longlong, c_float, c_float, c_float,
                                  c_float, c_int, c_void_p]),
    "mm_surrogate_inputs": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_float, c_void_p, c_void_p, c_int,
                                    c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "mm_surrogate_planes": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "mm_surrogate_predict": (c_int, [POINTER(SurrogateDesc), c_void_p, c_int, c_void_p]),
    "mm_gather_screens": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p]),
    "mm_resample_power": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                  c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_float, c_void_p]),
    "mm_green_apply": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p]),
    "mm_green_matrix": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "mm_green_apply_grid": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_void_p]),
    "mm_green_blocks": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p]),
    "mm_lu_solve_batched": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p]),
    "mm_green_apply_grid_table": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_int,
                                          c_int, c_int, c_void_p, c_size_t, c_void_p]),
    "mm_v4_parity": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "mm_phase_prepare": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p,
                                 c_int, c_int, c_float, c_void_p, c_void_p, c_void_p]),
    "mm_pupil": (c_int, [POINTER(PupilDesc), c_void_p, c_void_p, c_void_p]),
    "mm_base_field": (c_int, [POINTER(BaseDesc), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mm_propagate_workspace_size": (c_size_t, [POINTER(StagePlan), c_int, c_int]),
    "mm_propagate_sites": (c_int, [POINTER(StagePlan), c_int, c_int, c_void_p, c_size_t, c_int, c_void_p]),
    "mm_propagate_status": (c_int, [POINTER(StagePlan), c_int, c_int, c_void_p, c_void_p]),
    "mm_propagate_sites_noalloc": (c_int, [POINTER(StagePlan), c_int, c_int, c_int, c_void_p]),
    "mm_items_blocks": (c_int, [c_int, c_int]),
    "mm_propagate_items_workspace_size": (c_size_t, [POINTER(ItemClass)]),
    "mm_propagate_items": (c_int, [POINTER(ItemClass), c_void_p, c_size_t, c_int, c_void_p]),
    "mm_focal_finalize": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_void_p, c_float,
                                  c_int, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                  c_void_p]),
    "mm_tail_finalize": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_int, c_int, c_double, c_void_p,
                                 c_void_p, c_void_p]),
    "mm_resample_images": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int,
                                   c_int, c_int, c_float, c_void_p, c_void_p]),
    "mm_gp_spectrum": (c_int, [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                               c_void_p, c_void_p, c_void_p, c_void_p]),
    "mm_gp_finish": (c_int, [c_void_p, c_int, c_int, c_int, c_float, c_float, c_float, c_void_p, c_void_p]),
    "mm_vessel_combine": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_float, c_void_p, c_int,
                                  c_int, c_int, c_void_p]),
    "mm_local_tiles": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_int]),
    "mm_local_render_workspace_size": (c_size_t, [POINTER(LocalDesc)]),
    "mm_local_render": (c_int, [POINTER(LocalDesc), c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "mm_scan_spectrum_bytes": (c_size_t, [POINTER(ScanDesc)]),
    "mm_scan_workspace_size": (c_size_t, [POINTER(ScanDesc), c_int]),
    "mm_scan_kernel_spectrum": (c_int, [POINTER(ScanDesc), POINTER(ScanPlanes), c_void_p, c_void_p, c_size_t,
                                        c_void_p]),
    "mm_scan_convolve": (c_int, [POINTER(ScanDesc), POINTER(ScanConv), c_void_p, c_void_p, c_size_t, c_void_p]),
    "mm_scan_forward": (c_int, [POINTER(ScanDesc), POINTER(ScanConv), c_void_p, c_void_p]),
    "mm_scan_inverse": (c_int, [POINTER(ScanDesc), POINTER(ScanConv), c_void_p, c_void_p]),
    "mm_scan_background": (c_int, [c_int, POINTER(c_void_p), c_int, ctypes.c_longlong, ctypes.c_longlong,
                                   ctypes.c_longlong, c_int, c_int, c_int, c_void_p, c_void_p, c_int, c_double,
                                   c_void_p, c_void_p, c_void_p]),
}

_lib = None


def load():
    """Load the library once (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH.name} is not built; run `python -m maomi_b200.build`")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def exported_symbols():
    """Names declared in the header that the binding expects."""
    return list(SIGNATURES)


def last_error():
    msg = load().mm_last_error()
    return msg.decode() if msg else ""


def check(rc, what=""):
    """Map a C status to the reference's exception types."""
    if rc == MM_OK:
        return
    msg = last_error() or what
    if rc in (MM_ERR_ARGUMENT, MM_ERR_NONFINITE, MM_ERR_UNSUPPORTED):
        raise ValueError(msg)
    raise RuntimeError(msg)


def call(name, *args):
    check(getattr(load(), name)(*args), name)


def require_cuda(device):
    """Product entry points run on CUDA only (no CPU fallback)."""
    import torch
    if not str(device).startswith("cuda"):
        raise ValueError("Use reference optics for CPU")
    if not torch.cuda.is_available():
        raise RuntimeError("CUDA-enabled PyTorch and an NVIDIA GPU are required")
    load()


def ptr(t):
    """Device (or host) address of a tensor / None."""
    if t is None:
        return None
    return c_void_p(t.data_ptr())


def upload(values, device, dtype=None):
    """Host array -> device tensor through pinned memory on the current
    stream, without blocking the host (no pipeline drain)."""
    import torch
    t = torch.as_tensor(np.ascontiguousarray(values))
    if dtype is not None:
        t = t.to(dtype)
    return t.pin_memory().to(device, non_blocking=True)


def stream_of(device=None):
    import torch
    return c_void_p(torch.cuda.current_stream(device).cuda_stream)


def host_array(values, ctype):
    a = np.ascontiguousarray(values)
    return (ctype * max(1, len(a)))(*a.tolist())
