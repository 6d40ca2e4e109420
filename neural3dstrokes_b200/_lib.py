"""ctypes binding of the in-tree CUDA library ``lib/libn3ds.so`` (C ABI: include/n3ds.h).

There is no CPU fallback: importing an operator without the built library raises.
Build it with ``python -m neural3dstrokes_b200.build``.
"""
import ctypes
import os
import threading

import torch

# N3DS_LIB selects another build of the same library (e.g. a tuning variant)
LIB_PATH = os.environ.get("N3DS_LIB") or os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib",
                                                      "libn3ds.so")

N3DS_OK = 0
N3DS_GRAD_EXACT = 0
N3DS_GRAD_COMPAT = 1

c_float_p = ctypes.c_void_p
c_size_t = ctypes.c_size_t
c_i64 = ctypes.c_int64
c_i32 = ctypes.c_int32
c_u32 = ctypes.c_uint32


class Batch(ctypes.Structure):
    _fields_ = [("n_scenes", c_i32), ("n_rays", ctypes.POINTER(c_i64)),
                ("n_strokes", ctypes.POINTER(c_i32)), ("n_samples", c_i32)]


class Rays(ctypes.Structure):
    _fields_ = [("x", ctypes.c_void_p), ("radius", ctypes.c_void_p), ("tdist", ctypes.c_void_p),
                ("dirs", ctypes.c_void_p), ("bg", ctypes.c_void_p), ("bg_value", ctypes.c_float),
                ("opaque_background", c_i32), ("origins", ctypes.c_void_p), ("radii", ctypes.c_void_p)]


class Strokes(ctypes.Structure):
    _fields_ = [("sdf_ids", ctypes.c_void_p), ("shape_params", ctypes.c_void_p), ("param_stride", c_i32),
                ("color_params", ctypes.c_void_p), ("density", ctypes.c_void_p),
                ("sdf_delta", ctypes.c_void_p), ("use_laplace_transform", c_i32),
                ("inv_scale_radius", c_i32), ("stroke_window", ctypes.c_void_p), ("base_mask", ctypes.c_uint32)]


class Options(ctypes.Structure):
    _fields_ = [("cull_alpha", ctypes.c_float), ("chunk_fwd", c_i32), ("chunk_bwd", c_i32),
                ("warps", c_i32), ("schedule", c_i32), ("grad_mode", c_i32),
                ("timing_events", ctypes.POINTER(ctypes.c_void_p)), ("warps_bwd", c_i32),
                ("forward_only", c_i32), ("count_pairs", c_i32), ("wait_limit_us", c_i32),
                ("test_stall_staging", c_i32), ("rays_per_item", c_i32)]


class DensityNet(ctypes.Structure):
    _fields_ = [("table", ctypes.c_void_p), ("offsets", ctypes.c_void_p), ("n_levels", c_u32),
                ("level_dim", c_u32), ("log2_per_level_scale", ctypes.c_float), ("base_resolution", c_u32),
                ("gridtype", c_u32), ("align_corners", c_i32), ("w1", ctypes.c_void_p), ("b1", ctypes.c_void_p),
                ("w2", ctypes.c_void_p), ("b2", ctypes.c_void_p), ("density_bias", ctypes.c_float),
                ("warp", c_i32), ("warp_scale", ctypes.c_float), ("grid_bound", ctypes.c_float),
                ("raw_output", c_i32), ("status", ctypes.c_void_p), ("wait_limit_us", c_i32), ("test_stall", c_i32)]


_P = ctypes.c_void_p
_DN = ctypes.POINTER(DensityNet)
_SIGS = {
    "n3ds_last_error": (ctypes.c_char_p, []),
    "n3ds_version": (ctypes.c_int, []),
    "n3ds_stroke_workspace_bytes": (c_size_t, [c_i64]),
    "n3ds_stroke_forward": (ctypes.c_int, [_P, _P, _P, _P, c_i64, _P, _P, _P, _P, _P, c_i64, c_i64, c_i64, c_i64,
                                           c_i64, c_u32, c_u32, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                           _P, c_size_t, _P]),
    "n3ds_stroke_backward": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, c_i64, c_i64,
                                            c_i64, c_i64, c_i64, c_u32, c_u32, ctypes.c_float, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, _P, c_size_t, _P]),
    "n3ds_compose_forward": (ctypes.c_int, [_P, _P, _P, _P, _P, c_i64, c_i64, c_i64, _P]),
    "n3ds_compose_workspace_bytes": (c_size_t, [c_i64, c_i64, ctypes.c_int]),
    "n3ds_compose_backward": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, c_i64, c_i64, c_i64,
                                             ctypes.c_int, _P, c_size_t, _P]),
    "n3ds_default_options": (None, [ctypes.POINTER(Options)]),
    "n3ds_field_workspace_bytes": (c_size_t, [ctypes.POINTER(Batch), ctypes.POINTER(Options)]),
    "n3ds_field_forward": (ctypes.c_int, [ctypes.POINTER(Batch), ctypes.POINTER(Rays), ctypes.POINTER(Strokes),
                                          ctypes.POINTER(Options), _P, _P, _P, _P, c_size_t, _P]),
    "n3ds_field_backward": (ctypes.c_int, [ctypes.POINTER(Batch), ctypes.POINTER(Rays),
                                           ctypes.POINTER(Strokes), ctypes.POINTER(Options), _P, _P, _P,
                                           _P, _P, _P, _P, _P, _P, c_size_t, _P]),
    "n3ds_field_read_status": (ctypes.c_int, [_P, ctypes.POINTER(c_i32), ctypes.POINTER(ctypes.c_uint64), _P]),
    "n3ds_adam_step": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, c_i64, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_float, ctypes.c_float, _P, _P]),
    "n3ds_fp32_probe": (ctypes.c_int, [_P, c_i32, c_i32, _P]),
    "n3ds_field_read_pair_counts": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64), _P]),
    "n3ds_field_read_backward_pairs": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64), _P]),
    "n3ds_max_dilate_weights": (ctypes.c_int, [_P, _P, _P, _P, c_i64, c_i32, ctypes.c_float, ctypes.c_float,
                                               ctypes.c_float, c_i32, _P]),
    "n3ds_sample_intervals": (ctypes.c_int, [_P, _P, _P, c_i64, c_i32, c_i32, _P, c_i32, ctypes.c_float,
                                             ctypes.c_float, _P]),
    "n3ds_resample_intervals": (ctypes.c_int, [_P, _P, _P, _P, c_i64, c_i32, c_i32, ctypes.c_float,
                                               ctypes.c_float, _P, c_i32, ctypes.c_float, ctypes.c_float, _P, _P,
                                               _P]),
    "n3ds_insert_workspace_bytes": (c_size_t, [_P, _P]),
    "n3ds_insert_step": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, c_i64, c_i32, ctypes.c_float, _P, _P, c_i64,
                                        _P, c_size_t, _P]),
    "n3ds_ema_update": (ctypes.c_int, [_P, _P, c_i64, ctypes.c_float, _P]),
    "n3ds_clip_columns": (ctypes.c_int, [_P, c_i64, c_i32, ctypes.POINTER(ctypes.c_float),
                                         ctypes.POINTER(ctypes.c_float), _P]),
    "n3ds_texture_forward": (ctypes.c_int, [_P, _P, _P, _P, _P, c_i64, _P, c_i32, c_i32, c_i32, ctypes.c_float,
                                            c_i32, _P]),
    "n3ds_texture_backward": (ctypes.c_int, [_P, _P, _P, _P, _P, c_i64, _P, c_i32, c_i32, c_i32, ctypes.c_float,
                                             c_i32, _P]),
    "n3ds_texture_pack": (ctypes.c_int, [_P, _P, c_i32, c_i32, c_i32, _P]),
    "n3ds_texture_forward_packed": (ctypes.c_int, [_P, _P, _P, _P, _P, c_i64, _P, c_i32, c_i32, c_i32,
                                                   ctypes.c_float, c_i32, _P]),
    "n3ds_texture_backward_packed": (ctypes.c_int, [_P, _P, _P, _P, _P, c_i64, _P, c_i32, c_i32, c_i32,
                                                    ctypes.c_float, c_i32, _P]),
    "n3ds_field_launch_count": (ctypes.c_int, [ctypes.POINTER(Batch), ctypes.POINTER(Options),
                                               ctypes.POINTER(c_i32), ctypes.POINTER(c_i32)]),
    "n3ds_field_resolve_options": (ctypes.c_int, [ctypes.POINTER(Options), ctypes.POINTER(Options)]),
    "n3ds_compose_mode_forward": (ctypes.c_int, [ctypes.c_int, _P, _P, _P, _P, _P, c_i64, c_i64, c_i64, _P]),
    "n3ds_compose_mode_backward": (ctypes.c_int, [ctypes.c_int, _P, _P, _P, _P, _P, _P, _P, _P, c_i64, c_i64,
                                                  c_i64, _P]),
    "n3ds_grid_encode_forward": (ctypes.c_int, [_P, _P, _P, _P, c_u32, c_u32, c_u32, c_u32, ctypes.c_float, c_u32,
                                                _P, c_u32, c_i32, c_u32, c_i32, _P]),
    "n3ds_grid_encode_backward": (ctypes.c_int, [_P, _P, _P, _P, _P, c_u32, c_u32, c_u32, c_u32, ctypes.c_float,
                                                 c_u32, _P, _P, c_u32, c_i32, c_u32, c_i32, _P]),
    "n3ds_grid_total_variation": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_float, c_u32, c_u32, c_u32, c_u32,
                                                 ctypes.c_float, c_u32, c_u32, c_i32, c_i32, _P]),
    "n3ds_density_net_feature_stride": (ctypes.c_int, [c_u32, c_u32]),
    "n3ds_density_net_resident_ctas": (ctypes.c_int, [c_i32]),
    "n3ds_density_net_forward": (ctypes.c_int, [_DN, _P, c_i64, _P, _P, _P, _P]),
    "n3ds_density_net_backward": (ctypes.c_int, [_DN, _P, _P, _P, c_i64, _P, _P, _P, _P, _P, _P]),
    "n3ds_grid_level_mean_sq": (ctypes.c_int, [_P, _P, c_u32, c_u32, c_i32, _P, _P]),
    "n3ds_grid_level_mean_sq_backward": (ctypes.c_int, [_P, _P, c_u32, c_u32, c_i32, _P, _P, _P]),
    "n3ds_stroke_forward_static": (ctypes.c_int, [_P, _P, _P, _P, c_i64, _P, _P, _P, _P, _P, c_i64, c_i64, c_i64,
                                                  c_i64, c_i64, c_u32, c_u32, ctypes.c_float, ctypes.c_int,
                                                  ctypes.c_int, _P]),
}

EXPORTED = tuple(_SIGS)

_lib = None
_lock = threading.Lock()


def load():
    """Load (once) and return the ctypes handle; raises if the library is not built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"{LIB_PATH} is missing: build it with "
                                   f"`python -m neural3dstrokes_b200.build` (no CPU fallback exists)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(rc):
    if rc != N3DS_OK:
        msg = load().n3ds_last_error().decode()
        raise RuntimeError(f"n3ds error {rc}: {msg}")


def ptr(t):
    """Device pointer of a tensor, or None for None / empty tensors."""
    if t is None or t.numel() == 0:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr(device=None):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def workspace(nbytes, device):
    """A 256-byte aligned byte buffer from torch's caching allocator."""
    buf = torch.empty(max(int(nbytes), 1) + 256, dtype=torch.uint8, device=device)
    off = (-buf.data_ptr()) % 256
    return buf[off:off + max(int(nbytes), 1)]


def default_options(**kw):
    o = Options()
    load().n3ds_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o
