"""Torch restatement of the reference's proposal resampling (source/utils/stepfun.py),
TEST INFRASTRUCTURE ONLY: imported by tests, never by the product package.

Dtype-generic, vectorised over rays. Randomness is explicit: where the reference
draws ``torch.rand`` inside ``sample`` (stepfun.py:237-242), these functions take the
drawn values as ``jitter`` ([..., 1] for single_jitter, [..., N] otherwise; None for
the deterministic centred samples). Pinned against tests/golden/stepfun_golden.npz,
which the reference itself produced (tests/golden/make_golden.py --stepfun).
"""
import math

import torch


def _eps(x):
    return torch.finfo(x.dtype).eps


def interp_sorted(x, xp, fp):
    """sorted_interp (stepfun.py:5-24): per ray, the last post with xp <= x and the
    first with xp > x (by masks), linear in between, offset nan->0 and clipped."""
    le = x[..., None, :] >= xp[..., :, None]                        # [..., P, Q]
    lo_f = torch.where(le, fp[..., :, None], fp[..., :1, None]).max(-2).values
    hi_f = torch.where(~le, fp[..., :, None], fp[..., -1:, None]).min(-2).values
    lo_x = torch.where(le, xp[..., :, None], xp[..., :1, None]).max(-2).values
    hi_x = torch.where(~le, xp[..., :, None], xp[..., -1:, None]).min(-2).values
    off = torch.clip(torch.nan_to_num((x - lo_x) / (hi_x - lo_x), 0), 0, 1)
    return lo_f + off * (hi_f - lo_f)


def cdf_of(w):
    """integrate_weights (stepfun.py:150-171): [0, min(cumsum(w[:-1]), 1), 1]."""
    c = torch.cumsum(w[..., :-1], -1).clamp_max(1)
    z = torch.zeros(c.shape[:-1] + (1,), dtype=w.dtype, device=w.device)
    return torch.cat([z, c, torch.ones_like(z)], -1)


def max_dilate_weights(t, w, dilation, domain=(-math.inf, math.inf), renormalize=False):
    """stepfun.py:120-147: pdf -> max-pooled pdf over the dilated intervals -> weights."""
    eps = _eps(w)
    p = w / (t[..., 1:] - t[..., :-1]).clamp_min(eps)
    lo_edges = t[..., :-1] - dilation
    hi_edges = t[..., 1:] + dilation
    posts = torch.sort(torch.cat([t, lo_edges, hi_edges], -1), -1).values.clip(*domain)
    inside = (lo_edges[..., None, :] <= posts[..., None]) & (hi_edges[..., None, :] > posts[..., None])
    p_d = torch.where(inside, p[..., None, :], torch.zeros_like(p[..., None, :])).max(-1).values[..., :-1]
    w_d = p_d * (posts[..., 1:] - posts[..., :-1])
    if renormalize:
        w_d = w_d / w_d.sum(-1, keepdim=True).clamp_min(eps)
    return posts, w_d


def sample_intervals(jitter, t, w_logits, num_samples, single_jitter=False, domain=(-math.inf, math.inf)):
    """stepfun.py:220-243, 280-317: centred (jitter None) or jittered inverse-CDF
    samples, then the intervals between them with reflected, clamped end posts."""
    eps = _eps(t)
    n = num_samples
    if jitter is None:
        pad = 1 / (2 * n)
        u = torch.linspace(pad, 1. - pad - eps, n, dtype=t.dtype, device=t.device).expand(t.shape[:-1] + (n,))
    else:
        u_max = eps + (1 - eps) / n
        max_jitter = (1 - u_max) / (n - 1) - eps
        u = torch.linspace(0, 1 - u_max, n, dtype=t.dtype, device=t.device) + jitter.to(t) * max_jitter
    w = torch.softmax(w_logits, -1)
    centers = interp_sorted(u, cdf_of(w), t)
    mid = (centers[..., 1:] + centers[..., :-1]) / 2
    first = (2 * centers[..., :1] - mid[..., :1]).clamp_min(domain[0])
    last = (2 * centers[..., -1:] - mid[..., -1:]).clamp_max(domain[1])
    return torch.cat([first, mid, last], -1)


def resample_level(sdist, weights, num_samples, jitter=None, single_jitter=True, dilation=0.0, padding=0.0,
                   domain=(0.0, 1.0), near=None, far=None):
    """One proposal level (models.py:156-185): optional dilation + [1:-1] slice,
    logits, sampling, and the identity s -> t warp (coord.py:96-99)."""
    if dilation > 0:
        sdist, weights = max_dilate_weights(sdist, weights, dilation, domain=domain, renormalize=True)
        sdist, weights = sdist[..., 1:-1], weights[..., 1:-1]
    logits = torch.where(sdist[..., 1:] > sdist[..., :-1], torch.log(weights + padding),
                         torch.full_like(sdist[..., :-1], -math.inf))
    s = sample_intervals(jitter, sdist, logits, num_samples, single_jitter, domain)
    t = None if near is None else s * far + (1 - s) * near
    return s, t
