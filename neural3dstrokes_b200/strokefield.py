"""Drop-in for the stroke level of the reference model: StrokeField.predict_density
(source/models.py:660-711) followed by the render step of Model.forward
(models.py:206-235: compute_alpha_weights + volumetric_rendering, render.py:29-88),
fused into one forward and one adjoint backward.

``render_stroke_field(field, coords, radius, tdist, directions, ...)`` reads the
reference StrokeField's own attributes, so a model keeps its module, parameters and
checkpoints:

- ``shape_params`` [max_num_strokes, d_shape], ``color_params`` [max, 3],
  ``density_params`` [max] (the nn.Parameters), ``stroke_step`` (int32 buffer),
- ``max_num_strokes``, ``max_opt_strokes``, ``stroke_step_limit``,
  ``density_scale``, ``sdf_delta``, ``sdf_delta_eval``, ``training``,
  ``use_laplace_transform``, ``inv_scale_radius``, ``warp_fn``, ``bbox_size``,
  ``shape_type``, and (checked) ``color_type``, ``composition_type``,
  ``stroke_texture``.

What predict_density does, and how it is done here:
- coordinates warped into [-1, 1] (``_warp_coords`` models.py:19-33): the same torch
  ops, before the fused kernels; the sample radius is not warped (models.py:681);
- truncation to ``stroke_step`` (models.py:666-673): the reference reads the count
  to the host (``.item()``); here it stays on the device as a stroke window the
  kernels read, so the call has no host synchronisation (and can be graph-captured);
- the no-grad fixed strokes below ``stroke_step - max_opt_strokes`` concatenated
  before the optimised ones (models.py:686-702): the same stroke order, composited,
  with no gradient of their own and none into the coordinates;
- ``density_scale`` (models.py:673) and the training-time ``sdf_delta`` annealing
  towards ``sdf_delta_eval`` (models.py:675-680), computed on the device in float64
  and rounded to float32 as the reference's Python arithmetic is;
- 'over' composition (models.py:709), then compute_alpha_weights and
  volumetric_rendering with the background colour (models.py:206-235).

Returns rgb [R,3], acc [R] (opacity) and depth [R]. Constant-rgb colour, 'over'
composition and no stroke texture (the reference configs' setting) run fused; other
settings raise NotImplementedError (the drop-in ``_strokelib`` operators cover them).
"""
from typing import Optional

import torch

from . import strokes as _strokes
from .field import FieldOptions, render_strokes


def _contract(x):
    """coord.contract (source/utils/coord.py:5-11), the same torch ops."""
    eps = torch.finfo(x.dtype).eps
    x_mag_sq = torch.sum(x ** 2, dim=-1, keepdim=True).clamp_min(eps)
    return torch.where(x_mag_sq <= 1, x, ((2 * torch.sqrt(x_mag_sq) - 1) / x_mag_sq) * x)


def warp_coords(warp_fn, coords, bbox_size=2.0, no_warp=False):
    """_warp_coords (models.py:19-33): coordinates into [-1, 1]."""
    if no_warp:
        return coords
    if warp_fn is None:
        bound = bbox_size / 2
        return coords / bound
    if warp_fn == "contract":
        return _contract(coords) / 2.0
    raise NotImplementedError(f"Unknown warp function {warp_fn}")


def stroke_window(field):
    """(frozen, active) of the field's single scene as a device int32 [1, 2] tensor,
    from the device stroke count: active = stroke_step, frozen = max(0, stroke_step -
    max_opt_strokes), both capped by stroke_step_limit (models.py:666-670)."""
    step = field.stroke_step.reshape(1).to(torch.int32)
    fixed = (step - int(field.max_opt_strokes)).clamp_min(0)
    if getattr(field, "stroke_step_limit", None) is not None:
        lim = int(field.stroke_step_limit)
        step = step.clamp_max(lim)
        fixed = fixed.clamp_max(lim)
    return torch.cat([fixed, step]).reshape(1, 2)


def annealed_delta(field, window):
    """sdf_delta of this call: while training, lerp(sdf_delta, sdf_delta_eval,
    clamp(stroke_step / max_num_strokes, 0, 1)) (models.py:675-678) with the truncated
    count, in float64 then float32 (a device 0-d tensor); sdf_delta_eval otherwise."""
    dev = window.device
    if not field.training:
        return torch.tensor(float(field.sdf_delta_eval), device=dev, dtype=torch.float32)
    frac = (window[0, 1].to(torch.float64) / float(field.max_num_strokes)).clamp(0.0, 1.0)
    d = float(field.sdf_delta) * (1 - frac) + float(field.sdf_delta_eval) * frac
    return d.to(torch.float32)


def render_stroke_field(field, coords: torch.Tensor, radius: torch.Tensor, tdist: torch.Tensor,
                        directions: torch.Tensor, bg=1.0, opaque_background: bool = False, no_warp: bool = False,
                        options: Optional[FieldOptions] = None):
    """predict_density + the render step of the stroke level for one scene.

    coords [R,N,3], radius [R,N] (cast_rays' outputs, render.py:5-26), tdist [R,N+1],
    directions [R,3]; bg a float or [R,3]. Gradients flow to field.shape_params,
    color_params and density_params (rows of the optimised window only) and to
    coords."""
    if getattr(field, "color_type", "constant_rgb") != "constant_rgb":
        raise NotImplementedError("the fused stroke field computes constant_rgb colour")
    if getattr(field, "composition_type", "over") != "over":
        raise NotImplementedError("the fused stroke field composites with 'over'")
    if getattr(field, "stroke_texture", None) is not None:
        raise NotImplementedError("the fused stroke field has no stroke texture")
    dev = coords.device
    S = int(field.shape_params.shape[0])
    sdf_id = _strokes.sdf_id_of(field.shape_type)
    ids = getattr(field, "_n3ds_sdf_ids", None)
    if ids is None or ids.device != dev or ids.numel() != S or int(getattr(field, "_n3ds_sdf_id", -1)) != sdf_id:
        ids = torch.full((S,), sdf_id, dtype=torch.int32, device=dev)
        field._n3ds_sdf_ids, field._n3ds_sdf_id = ids, sdf_id
    window = stroke_window(field)
    delta = annealed_delta(field, window).expand(S)
    density = field.density_params * field.density_scale
    x = warp_coords(getattr(field, "warp_fn", None), coords, float(getattr(field, "bbox_size", 2.0)), no_warp)
    return render_strokes(x, radius, tdist, directions, field.shape_params, ids, field.color_params, density, delta,
                          bool(field.use_laplace_transform), bool(field.inv_scale_radius), bg, opaque_background,
                          options, stroke_window=window)


class StrokeField(torch.nn.Module):
    """The reference StrokeField's parameters and settings (models.py:526-574) for a
    caller without the reference module; ``render`` is ``render_stroke_field``."""

    def __init__(self, shape_type="sphere", max_num_strokes=500, max_opt_strokes=500, density_scale=20.0,
                 sdf_delta=7.0, sdf_delta_eval=1.0, use_laplace_transform=False, inv_scale_radius=True,
                 bbox_size=4.0, warp_fn=None, stroke_step_limit=None):
        super().__init__()
        self.shape_type = shape_type
        self.color_type = "constant_rgb"
        self.composition_type = "over"
        self.stroke_texture = None
        self.max_num_strokes = int(max_num_strokes)
        self.max_opt_strokes = int(max_opt_strokes)
        self.density_scale = float(density_scale)
        self.sdf_delta = float(sdf_delta)
        self.sdf_delta_eval = float(sdf_delta_eval)
        self.use_laplace_transform = bool(use_laplace_transform)
        self.inv_scale_radius = bool(inv_scale_radius)
        self.bbox_size = float(bbox_size)
        self.warp_fn = warp_fn
        self.stroke_step_limit = stroke_step_limit
        d_shape = _strokes.num_shape_params(shape_type)
        self.shape_params = torch.nn.Parameter(torch.zeros(self.max_num_strokes, d_shape))
        self.color_params = torch.nn.Parameter(torch.zeros(self.max_num_strokes, 3))
        self.density_params = torch.nn.Parameter(torch.ones(self.max_num_strokes))
        self.register_buffer("stroke_step", torch.tensor(0, dtype=torch.int32))

    def render(self, coords, radius, tdist, directions, bg=1.0, opaque_background=False, no_warp=False,
               options=None):
        return render_stroke_field(self, coords, radius, tdist, directions, bg, opaque_background, no_warp,
                                   options)
