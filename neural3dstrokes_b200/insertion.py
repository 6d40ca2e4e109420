"""Stroke insertion and reset on the device: StrokeField.step_update
(source/models.py:586-658) and clip_params (576-584) without host round trips.

``StrokeInserter`` owns the stroke parameters of one field ([max_num_strokes, ...]
tensors that callers may wrap as parameters), the shape-gradient EMA and, in device
memory, the stroke count and the step of the last update. ``step_update(cur_step,
max_step, shape_grad=None, errors=None, error_coords=None)`` runs the reference's
update: EMA of the shape gradients, detection of strokes whose density fell under
``reset_density``, the update decision, new strokes centred on the top error samples
(or split from the top shape-gradient rows), resets, and the clamp, as three to four
kernel launches with no synchronisation (``n3ds_ema_update``, ``n3ds_insert_step``,
``n3ds_clip_columns``).

Differences, deliberate: the error field is the caller's (as in the reference, an MLP
outside the stroke path): draw points with ``sample_error_coords()``, evaluate them and
pass the errors every step (the reference evaluates only when it updates, which needs
the update decision on the host); random draws come from a counter-based hash on the
device, so individual values differ from the reference's host RNG while their
distributions match.
"""
import ctypes
import math
from typing import Optional

import torch

from . import _lib
from . import strokes as _strokes

_BASE_SAMPLER = {"roundcube": (1, 0, 0), "roundbox": (1, 0, 0), "cappedtorus": (2, 0, 0), "capsule": (3, 0, 0),
                 "scapsule": (3, 0, 0), "line": (4, 0, 0), "triprism": (5, 0, 0),
                 "quadratic_bezier": (6, 3, 2), "cubic_bezier": (6, 4, 2), "catmull_rom": (6, 4, 2)}
_INIT = {"recon": 0, "gen_box": 1, "gen_sphere": 2}
_COLOR_SAMPLER = {"constant_rgb": 0, "gradient_rgb": 1, "constant_sh2": 2, "constant_sh3": 2}


class _Sampler(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("n_shape", "n_color", "base_sampler", "spline_points", "spline_radii",
                                               "t", "r", "s1", "s3", "init_type", "color_sampler")]


class _Config(ctypes.Structure):
    _fields_ = [("max_num_strokes", ctypes.c_int32), ("init_num_strokes", ctypes.c_int32),
                ("reset_density", ctypes.c_float), ("use_error_field", ctypes.c_int32),
                ("use_shape_grads", ctypes.c_int32), ("shape_split_update_rate", ctypes.c_float),
                ("min_update_interval", ctypes.c_int32), ("min_reset_interval", ctypes.c_int32),
                ("max_reset_frac", ctypes.c_float), ("seed", ctypes.c_uint64)]


def _bounds(ranges):
    lo = [float("nan") if a is None else float(a) for a, _ in ranges]
    hi = [float("nan") if b is None else float(b) for _, b in ranges]
    return (ctypes.c_float * len(ranges))(*lo), (ctypes.c_float * len(ranges))(*hi)


class StrokeInserter:
    """Device-side StrokeField.step_update; attribute names follow the reference."""

    def __init__(self, shape_type="sphere", color_type="constant_rgb", init_type="recon", max_num_strokes=500,
                 init_num_strokes=10, reset_density=0.01, use_error_field=True, use_shape_grads=False,
                 shape_grad_ema=0.99, shape_split_update_rate=0.05, min_update_interval=2, min_reset_interval=50,
                 max_reset_frac=0.95, error_point_samples=30000, step_power=0.5, bbox_size=2.0,
                 train_density=True, seed=0, device="cuda"):
        if shape_type not in _strokes._SHAPES:
            raise KeyError(shape_type)
        if init_type not in _INIT:
            raise ValueError(f"Unknown init type {init_type}")
        _, d_shape, d_color, self.shape_param_ranges, self.color_param_ranges, _, _ = \
            _strokes.get_stroke(shape_type, color_type, init_type)
        _, _, _, t, r, s1, s3 = _strokes._SHAPES[shape_type]
        base, pts, rad = _BASE_SAMPLER.get(shape_type, (0, 0, 0))
        self.sampler = _Sampler(d_shape, d_color, base, pts, rad, int(bool(t)), int(bool(r)), int(bool(s1)),
                                int(bool(s3)), _INIT[init_type], _COLOR_SAMPLER[color_type])
        self.max_num_strokes, self.init_num_strokes, self.step_power = int(max_num_strokes), int(init_num_strokes), \
            float(step_power)
        self.shape_grad_ema = float(shape_grad_ema)
        self.error_point_samples, self.bbox_size = int(error_point_samples), float(bbox_size)
        self.use_error_field = bool(use_error_field)
        self.config = _Config(self.max_num_strokes, self.init_num_strokes,
                              float(reset_density) if train_density else float("-inf"), int(self.use_error_field),
                              int(bool(use_shape_grads)), float(shape_split_update_rate), int(min_update_interval),
                              int(min_reset_interval), float(max_reset_frac), int(seed) & (2 ** 64 - 1))
        dev = torch.device(device)
        self.device = dev
        m = self.max_num_strokes
        # models.py:564-570: zero shape / colour parameters, unit densities, empty field
        self.shape_params = torch.zeros(m, d_shape, device=dev)
        self.color_params = torch.zeros(m, d_color, device=dev)
        self.density_params = torch.ones(m, device=dev)
        self.shape_params_grad = torch.zeros(m, d_shape, device=dev)
        self.stroke_step = torch.zeros(1, dtype=torch.int32, device=dev)
        self.last_update_step = torch.zeros(1, dtype=torch.int32, device=dev)
        lib = _lib.load()
        self._ws = torch.empty(int(lib.n3ds_insert_workspace_bytes(ctypes.byref(self.config),
                                                                  ctypes.byref(self.sampler))),
                               dtype=torch.uint8, device=dev)
        self._shape_bounds = _bounds(self.shape_param_ranges) if d_shape else None
        self._color_bounds = _bounds(self.color_param_ranges)
        self._density_bounds = _bounds([(0.0, None)])

    def next_target(self, cur_step: int, max_step: int):
        """models.py:589-594 up to the max with the current count (taken on the device)."""
        steps_per_stroke = max_step // self.max_num_strokes
        if steps_per_stroke <= 1:
            raise ValueError(f"Too few steps per stroke: {steps_per_stroke}")
        train_frac = cur_step / (max_step - steps_per_stroke)
        nxt = int(self.max_num_strokes * min(max(train_frac, 0.0), 1.0) ** self.step_power)
        return min(nxt + self.init_num_strokes, self.max_num_strokes), train_frac

    def sample_error_coords(self, n: Optional[int] = None):
        """Points to evaluate the caller's error field at (models.py:613-616): normalised
        coordinates in [-1, 1]^3 and their unwarped positions (identity warp: * bbox/2)."""
        c = torch.rand(n or self.error_point_samples, 3, device=self.device) * 2 - 1
        return c, c * (self.bbox_size / 2)

    def step_update(self, cur_step: int, max_step: int, shape_grad: Optional[torch.Tensor] = None,
                    errors: Optional[torch.Tensor] = None, error_coords: Optional[torch.Tensor] = None):
        """StrokeField.step_update (models.py:586-658) on the device; ``errors`` [E] at
        ``error_coords`` [E, 3] (normalised, from sample_error_coords) when the error
        field is used, ``shape_grad`` [max, n_shape] the current shape gradient."""
        lib = _lib.load()
        nt, train_frac = self.next_target(int(cur_step), int(max_step))
        st = _lib.stream_ptr()
        with torch.cuda.device(self.device):
            if shape_grad is not None:
                g = shape_grad.detach().float().contiguous()
                if g.shape != self.shape_params_grad.shape:
                    raise ValueError("shape_grad must match shape_params")
                _lib.check(lib.n3ds_ema_update(_lib.ptr(self.shape_params_grad), _lib.ptr(g),
                                               self.shape_params_grad.numel(), self.shape_grad_ema, st))
            e = c = None
            n_err = 0
            if errors is not None:
                e = errors.detach().float().contiguous().reshape(-1)
                c = error_coords.detach().float().contiguous().reshape(-1, 3)
                if c.shape[0] != e.shape[0]:
                    raise ValueError("errors and error_coords must have the same length")
                n_err = e.shape[0]
            _lib.check(lib.n3ds_insert_step(ctypes.byref(self.config), ctypes.byref(self.sampler),
                                            _lib.ptr(self.shape_params), _lib.ptr(self.color_params),
                                            _lib.ptr(self.density_params), _lib.ptr(self.shape_params_grad),
                                            _lib.ptr(self.stroke_step), _lib.ptr(self.last_update_step),
                                            int(cur_step), int(nt), float(train_frac), _lib.ptr(e), _lib.ptr(c),
                                            n_err, _lib.ptr(self._ws), self._ws.numel(), st))
            self.clip_params()

    def clip_params(self):
        """models.py:576-584: clamp shape / colour columns to their ranges, densities >= 0."""
        lib = _lib.load()
        st = _lib.stream_ptr()
        m = self.max_num_strokes
        for x, b in ((self.shape_params, self._shape_bounds), (self.color_params, self._color_bounds),
                     (self.density_params, self._density_bounds)):
            if b is None:
                continue
            cols = 1 if x.dim() == 1 else x.shape[1]
            _lib.check(lib.n3ds_clip_columns(_lib.ptr(x), m, cols, b[0], b[1], st))
