"""Restatement of source/utils/render.py (volume rendering) plus the whole-path oracle.

TEST INFRASTRUCTURE ONLY: used by tests, smoke() and the bench's CPU legs.

- ``cast_rays``              <- render.py:5-26
- ``compute_alpha_weights``  <- render.py:29-48
- ``volumetric_rendering``   <- render.py:51-88 (rgb, depth, acc; the extras are out
  of scope)
- ``render_strokes``: the stroke-field path end to end, as models.py drives it
  (StrokeField.predict_density models.py:660-711 -> compute_alpha_weights ->
  volumetric_rendering, models.py:206-235): per-group stroke evaluation, 'over'
  compositing, then volume rendering.
"""
import torch

from . import strokefield as sf


def cast_rays(tdist, origins, directions, radii):
    t = 0.5 * (tdist[..., :-1] + tdist[..., 1:])
    coords = directions[..., None, :] * t[..., None] + origins[..., None, :]
    radius = radii * t
    return coords, radius, t


def compute_alpha_weights(density, tdist, dirs, opaque_background=False):
    t_delta = tdist[..., 1:] - tdist[..., :-1]
    delta = t_delta * torch.norm(dirs[..., None, :], dim=-1)
    density_delta = density * delta
    if opaque_background:
        density_delta = torch.cat([density_delta[..., :-1],
                                   torch.full_like(density_delta[..., -1:], torch.inf)], dim=-1)
    alpha = 1 - torch.exp(-density_delta)
    trans = torch.exp(-torch.cat([torch.zeros_like(density_delta[..., :1]),
                                  torch.cumsum(density_delta[..., :-1], dim=-1)], dim=-1))
    weights = alpha * trans
    return weights, alpha, trans


def volumetric_rendering(rgbs, weights, tdist, bg_rgbs, eps=None):
    """render.py:51-88; ``eps`` defaults to the machine epsilon of the input dtype as
    the reference does (render.py:76)."""
    if eps is None:
        eps = torch.finfo(rgbs.dtype).eps
    acc = weights.sum(dim=-1)
    bg_w = (1 - acc[..., None]).clamp_min(0.)
    rgb = (weights[..., None] * rgbs).sum(dim=-2) + bg_w * bg_rgbs
    t_mids = 0.5 * (tdist[..., :-1] + tdist[..., 1:])
    depth = torch.clip(torch.nan_to_num((weights * t_mids).sum(dim=-1) / acc.clamp_min(eps), torch.inf),
                       tdist[..., 0], tdist[..., -1])
    return rgb, depth, acc


def render_strokes(x, radius, tdist, dirs, shape_params, sdf_ids, color_params, density,
                   sdf_delta, use_laplace=True, inv_scale_radius=True, bg=1.0,
                   opaque_background=False):
    """Whole stroke-field path for one scene.

    x [R,N,3], radius [R,N], tdist [R,N+1], dirs [R,3]; shape_params [S,Pmax] padded,
    sdf_ids [S]; color_params [S,3]; density [S] (already times density_scale).
    Returns rgb [R,3], acc [R], depth [R]. Differentiable by torch.autograd.

    The depth guard max(acc, eps) uses float32's epsilon whatever the oracle dtype:
    the reference path runs in float32 (render.py:76 takes eps from the input dtype),
    so that constant is part of the function being reproduced.
    """
    R, N, _ = x.shape
    xf = x.reshape(-1, 3)
    rf = radius.reshape(-1)
    alpha, color = sf.stroke_forward_mixed(xf, rf, shape_params, sdf_ids, color_params,
                                           sdf_delta, use_laplace, inv_scale_radius)
    dens, col = sf.compose_forward(alpha, color, density)
    weights = compute_alpha_weights(dens.reshape(R, N), tdist, dirs, opaque_background)[0]
    rgb, depth, acc = volumetric_rendering(col.reshape(R, N, -1), weights, tdist, bg,
                                           eps=float(torch.finfo(torch.float32).eps))
    return rgb, acc, depth
