"""The reference Model's ray-sampling loop (source/models.py:125-200) over this
package's kernels, for a model whose last level is the stroke field.

Per proposal level:
  * one resampling launch (stepfun.resample_intervals): the dilation of the previous
    level's weights (after the first level), the logits
    ``where(s[1:] > s[:-1], log(w + padding), -inf)``, sample_intervals and the
    identity ray warp s -> t = s * far + (1 - s) * near (models.py:147-185,
    coord.py:56-99 with raydist_fn None, the Model default);
  * cast_rays (render.py:5-26) and the proposal network (mlp.PropMLP: coordinate warp,
    hash-grid encoding and density layers in one launch);
  * compute_alpha_weights (render.py:29-48: elementwise ops and a cumulative sum over
    [R, N], torch ops as in the reference).
The last level's intervals are resampled the same way and returned: the stroke field
casts its samples from them inside its kernels (field.render_rays), so the last
level's [R, N, 3] positions are never written to memory.

Sampling is not differentiated (the reference's stop_level_grad, models.py:181-183,
is on by default): the intervals are data for the next level, while each proposal
level's density and weights stay differentiable with respect to that network's
parameters for the caller's interlevel loss.
"""
import dataclasses
from typing import List, Sequence

import torch

from . import stepfun


def compute_alpha_weights(density: torch.Tensor, tdist: torch.Tensor, dirs: torch.Tensor,
                          opaque_background: bool = False):
    """render.py:29-48: (weights, alpha, trans) of interval densities [..., N] over the
    fence posts tdist [..., N + 1] of rays with directions dirs [..., 3]."""
    t_delta = tdist[..., 1:] - tdist[..., :-1]
    density_delta = density * (t_delta * torch.norm(dirs[..., None, :], dim=-1))
    if opaque_background:
        density_delta = torch.cat([density_delta[..., :-1], torch.full_like(density_delta[..., -1:], torch.inf)], -1)
    alpha = 1 - torch.exp(-density_delta)
    trans = torch.exp(-torch.cat([torch.zeros_like(density_delta[..., :1]),
                                  torch.cumsum(density_delta[..., :-1], dim=-1)], dim=-1))
    return alpha * trans, alpha, trans


@dataclasses.dataclass
class RaySamples:
    sdist: torch.Tensor  # [R, N + 1] normalised fence posts of the last level
    tdist: torch.Tensor  # [R, N + 1] metric fence posts of the last level
    levels: List[dict]   # per proposal level: sdist, tdist, density [R, n], weights [R, n]


def sample_rays(origins: torch.Tensor, directions: torch.Tensor, radii: torch.Tensor, near: torch.Tensor,
                far: torch.Tensor, prop_mlps: Sequence[torch.nn.Module], num_prop_samples: int = 64,
                num_nerf_samples: int = 32, dilation_bias: float = 0.0025, dilation_multiplier: float = 0.5,
                resample_padding: float = 0.0, single_jitter: bool = True, rand: bool = False,
                opaque_background: bool = False) -> RaySamples:
    """The proposal levels of Model.forward (models.py:125-200) for rays origins /
    directions [R, 3], radii / near / far [R] or [R, 1], one proposal network per level
    (the Model's prop_mlp_0, prop_mlp_1); then the last level's resampling.
    ``num_nerf_samples`` is the last level's sample count as the caller's schedule has
    it (the reference scales it while training, models.py:140-144). ``rand`` draws the
    jitter (training); without it the samples are the deterministic centred ones."""
    R = int(origins.shape[0])
    if origins.shape != (R, 3) or directions.shape != (R, 3):
        raise ValueError("expected origins / directions [R, 3]")
    if radii.numel() != R or near.numel() != R or far.numel() != R:
        raise ValueError("expected radii / near / far with one value per ray")
    if not origins.is_cuda:
        raise RuntimeError("sample_rays runs on CUDA tensors only (the resampling and network kernels)")
    init_s_near, init_s_far = 0.0, 1.0
    near = near.reshape(R)
    far = far.reshape(R)
    sdist = torch.cat([torch.full((R, 1), init_s_near, device=origins.device),
                       torch.full((R, 1), init_s_far, device=origins.device)], -1)
    weights = torch.ones(R, 1, device=origins.device)
    use_dilation = dilation_bias > 0 or dilation_multiplier > 0
    prod_num_samples = 1
    levels = []
    n_levels = len(prop_mlps) + 1
    for i in range(n_levels):
        is_prop = i < n_levels - 1
        if is_prop and num_prop_samples == 0:  # no proposal sampling (models.py:137-138)
            continue
        n = num_prop_samples if is_prop else num_nerf_samples
        dilation = dilation_bias + dilation_multiplier * (init_s_far - init_s_near) / prod_num_samples
        prod_num_samples *= n
        sdist, tdist = stepfun.resample_intervals(sdist, weights.detach(), n, rand=rand, single_jitter=single_jitter,
                                                  dilation=dilation if (i > 0 and use_dilation) else 0.0,
                                                  resample_padding=resample_padding,
                                                  domain=(init_s_near, init_s_far), near=near, far=far)
        if not is_prop:
            return RaySamples(sdist, tdist, levels)
        t = (tdist[:, :-1] + tdist[:, 1:]) / 2
        coords = directions[:, None, :] * t[..., None] + origins[:, None, :]
        radius = radii.reshape(R, 1) * t
        density = prop_mlps[i](coords.reshape(-1, 3), radius.reshape(-1))["density"].reshape(R, n)
        weights = compute_alpha_weights(density, tdist, directions, opaque_background)[0]
        levels.append(dict(sdist=sdist, tdist=tdist, density=density, weights=weights))
    raise AssertionError("unreachable")
