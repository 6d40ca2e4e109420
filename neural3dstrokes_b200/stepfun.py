"""Proposal resampling of ray intervals: the functions of source/utils/stepfun.py on
the stroke path (models.py:147-185), one CUDA warp per ray.

``max_dilate_weights(t, w, dilation, domain, renormalize)`` and
``sample_intervals(rand, t, w_logits, num_samples, single_jitter, domain)`` take and
return what the reference functions do; ``resample_intervals`` runs one whole
proposal level (dilation, [1:-1] slice, logits with padding, sampling and the
identity s -> t warp) in one launch. With ``rand`` the jitter is drawn with
``torch.rand`` of the same shape the reference draws, so with the same generator
state the samples are the reference's.

Not differentiable: the reference detaches the resampled distances
(``stop_level_grad``, models.py:183-185).
"""
import math
from typing import Optional, Tuple

import torch

from . import _lib


def _prep(t, w):
    if t.dim() < 1 or w.shape[:-1] != t.shape[:-1] or t.shape[-1] != w.shape[-1] + 1:
        raise ValueError("expected t [..., n+1] and w [..., n]")
    if not t.is_cuda:
        raise RuntimeError("stepfun kernels run on CUDA tensors")
    pre = t.shape[:-1]
    n = w.shape[-1]
    R = int(math.prod(pre)) if len(pre) else 1
    return pre, n, R, t.detach().contiguous().float().reshape(R, n + 1), w.detach().contiguous().float().reshape(R, n)


def max_dilate_weights(t: torch.Tensor, w: torch.Tensor, dilation: float,
                       domain: Tuple[float, float] = (-math.inf, math.inf),
                       renormalize: bool = False) -> Tuple[torch.Tensor, torch.Tensor]:
    """stepfun.max_dilate_weights (stepfun.py:136-147): t [..., n+1], w [..., n] ->
    (t_dilate [..., 3n+1], w_dilate [..., 3n])."""
    pre, n, R, tc, wc = _prep(t, w)
    t_out = torch.empty(R, 3 * n + 1, device=t.device)
    w_out = torch.empty(R, 3 * n, device=t.device)
    with torch.cuda.device(t.device):
        _lib.check(_lib.load().n3ds_max_dilate_weights(_lib.ptr(t_out), _lib.ptr(w_out), _lib.ptr(tc), _lib.ptr(wc),
                                                       R, n, float(dilation), float(domain[0]), float(domain[1]),
                                                       int(bool(renormalize)), _lib.stream_ptr()))
    return t_out.reshape(*pre, 3 * n + 1), w_out.reshape(*pre, 3 * n)


def _jitter(rand, shape_pre, num_samples, single_jitter, device):
    if not rand:
        return None
    d = 1 if single_jitter else num_samples
    return torch.rand(shape_pre + (d,), device=device).contiguous()


def sample_intervals(rand, t: torch.Tensor, w_logits: torch.Tensor, num_samples: int, single_jitter: bool = False,
                     domain: Tuple[float, float] = (-math.inf, math.inf)) -> torch.Tensor:
    """stepfun.sample_intervals (stepfun.py:280-317): [..., num_samples + 1] fence posts."""
    if num_samples <= 1:
        raise ValueError(f"num_samples must be > 1, is {num_samples}.")
    pre, n, R, tc, lc = _prep(t, w_logits)
    jit = _jitter(rand, tuple(pre), num_samples, single_jitter, t.device)
    out = torch.empty(R, num_samples + 1, device=t.device)
    with torch.cuda.device(t.device):
        _lib.check(_lib.load().n3ds_sample_intervals(_lib.ptr(out), _lib.ptr(tc), _lib.ptr(lc), R, n, num_samples,
                                                     _lib.ptr(jit), int(bool(single_jitter)), float(domain[0]),
                                                     float(domain[1]), _lib.stream_ptr()))
    return out.reshape(*pre, num_samples + 1)


def resample_intervals(sdist: torch.Tensor, weights: torch.Tensor, num_samples: int, rand=False,
                       single_jitter: bool = True, dilation: float = 0.0, resample_padding: float = 0.0,
                       domain: Tuple[float, float] = (0.0, 1.0), near: Optional[torch.Tensor] = None,
                       far: Optional[torch.Tensor] = None):
    """One proposal level of the reference's loop (models.py:156-185) in one launch:
    ``dilation > 0`` dilates (renormalised) and drops the first and last posts, then
    the logits ``where(s[1:] > s[:-1], log(w + resample_padding), -inf)`` are sampled
    into ``num_samples`` intervals. Returns (sdist_new [..., N+1], tdist [..., N+1] or
    None), tdist = s * far + (1 - s) * near when near / far [...] (or [..., 1]) are given."""
    if num_samples <= 1:
        raise ValueError(f"num_samples must be > 1, is {num_samples}.")
    pre, n, R, sc, wc = _prep(sdist, weights)
    jit = _jitter(rand, tuple(pre), num_samples, single_jitter, sdist.device)
    s_out = torch.empty(R, num_samples + 1, device=sdist.device)
    t_out = None
    nr = fr = None
    if near is not None or far is not None:
        if near is None or far is None:
            raise ValueError("near and far go together")
        nr = near.detach().float().contiguous().reshape(R)
        fr = far.detach().float().contiguous().reshape(R)
        t_out = torch.empty(R, num_samples + 1, device=sdist.device)
    with torch.cuda.device(sdist.device):
        _lib.check(_lib.load().n3ds_resample_intervals(_lib.ptr(s_out), _lib.ptr(t_out), _lib.ptr(sc), _lib.ptr(wc),
                                                       R, n, num_samples, float(dilation), float(resample_padding),
                                                       _lib.ptr(jit), int(bool(single_jitter)), float(domain[0]),
                                                       float(domain[1]), _lib.ptr(nr), _lib.ptr(fr),
                                                       _lib.stream_ptr()))
    s_out = s_out.reshape(*pre, num_samples + 1)
    return s_out, (t_out.reshape(*pre, num_samples + 1) if t_out is not None else None)
