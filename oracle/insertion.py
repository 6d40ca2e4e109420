"""Restatement of the deterministic part of the reference's StrokeField.step_update
(source/models.py:586-658), TEST INFRASTRUCTURE ONLY (imported by tests).

``plan`` returns what the reference decides for one call: the next stroke count,
whether it updates, the reset indices (torch.nonzero order), and the order in which
error samples (torch.topk) or shape-gradient rows feed the new and reset strokes.
The random parameter draws themselves are not restated (the device draws its own).
"""
import math

import torch


def plan(prev, last_update_step, cur_step, max_step, density, cfg, errors=None, grad_ema=None):
    """cfg: dict with max_num_strokes, init_num_strokes, step_power, reset_density,
    train_density, use_error_field, use_shape_grads, min_update_interval,
    min_reset_interval, max_reset_frac."""
    m = cfg["max_num_strokes"]
    steps_per_stroke = max_step // m
    assert steps_per_stroke > 1
    train_frac = cur_step / (max_step - steps_per_stroke)
    nxt = int(m * min(max(train_frac, 0.0), 1.0) ** cfg["step_power"])
    nxt = min(max(nxt + cfg["init_num_strokes"], prev), m)
    reset_density = cfg["reset_density"] if cfg.get("train_density", True) else -math.inf
    resets = torch.nonzero(density[:prev] < reset_density).squeeze(1)
    n_reset = resets.numel()
    update = nxt - prev >= cfg["min_update_interval"] or (
        n_reset > 0 and cur_step - last_update_step >= cfg["min_reset_interval"] and train_frac < cfg["max_reset_frac"])
    out = {"next": nxt if update else prev, "update": update, "resets": resets, "mode": None, "top": None,
           "last": cur_step if update else last_update_step}
    if not update:
        return out
    k = nxt - prev + n_reset
    if prev > cfg["init_num_strokes"] and cfg["use_error_field"] and errors is not None:
        out["mode"] = "error"
        out["top"] = torch.topk(errors, k=min(k, errors.numel())).indices
    elif prev > cfg["init_num_strokes"] and cfg["use_shape_grads"] and grad_ema is not None:
        scores = grad_ema[:prev].sum(-1)
        scores[resets] = -math.inf
        out["mode"] = "grad"
        out["top"] = torch.topk(scores, k=min(k, prev - n_reset)).indices
    return out
