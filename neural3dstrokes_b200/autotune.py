"""Autotuner for the fused stroke-field kernels.

Times one forward + backward of a :class:`~neural3dstrokes_b200.train.BatchedField`
on its own data for each candidate launch configuration and keeps the fastest:

* work decomposition (``schedule``): 32-sample segments with every lane evaluating
  each surviving stroke, or 64-sample units with packed (sample, stroke) pairs;
* warps per CTA (rays in flight per SM), forward and backward separately (the
  segment kernels fit 32 warps; the backward's 32-warp build is held to 64 registers
  and spills a little: on config 3 its backward alone measured 5.12 against 5.27 ms
  and a whole tuned step within noise of 24 warps, on Bezier tubes (config 2) 26.2
  against 25.1 ms, so the tuner decides per workload; the run kernels 16);
* strokes per shared-memory stage: the largest that fits, or half of it (more passes,
  less shared memory per CTA);
* samples per warp claim (segment schedule): a warp takes 1, 2 or 4 rays (64, 128 or
  256 samples) per atomic on its scene's work counter; tried on the best of the
  configurations above.

Results are cached per workload signature (scene count, per-scene stroke counts, ray
counts rounded to powers of two, samples per ray, primitive mix, step mode) in memory
and, when ``N3DS_TUNE_CACHE`` names a file, in that JSON file across processes.
Timing uses CUDA events on the field's stream after one untimed warm-up per
candidate; the field's parameters are not changed (forward and backward only).
"""
import dataclasses
import json
import math
import os
import threading
from typing import Dict, List, Optional

import torch

from .field import FieldOptions

_lock = threading.Lock()
_memo: Dict[str, dict] = {}
last_results: List[tuple] = []  # (milliseconds, options) of the last tuning pass


def signature(field) -> str:
    """Workload key: what the best launch configuration depends on."""
    kinds = sorted(set(field.kinds))
    rays = [1 << max(0, int(round(math.log2(max(1, r))))) for r in field.scene_rays]
    return json.dumps({"strokes": list(field.scene_strokes), "rays": rays, "n": field.n_samples, "kinds": kinds,
                       "laplace": field.laplace, "inv": field.inv_scale, "grad": field.options.grad_mode},
                      sort_keys=True)


def candidates(grad_mode: str = "exact", cull_alpha: float = 1e-9, forward_only: bool = False,
               count_pairs: bool = False) -> List[FieldOptions]:
    out = []
    # (schedule, forward warps, backward warps): up to 32 warps per CTA for the
    # segment kernels, 16 for the run kernels
    shapes = [("segments", 32, 32), ("segments", 32, 24), ("segments", 32, 20), ("segments", 24, 16),
              ("segments", 16, 16), ("runs", 16, 16)]
    for schedule, wf, wb in shapes:
        for half in (False, True):
            # chunk 0 = the largest stage that fits; the halved stage (-1) is resolved later
            out.append(FieldOptions(cull_alpha=cull_alpha, warps=wf, warps_bwd=wb, schedule=schedule,
                                    grad_mode=grad_mode, chunk_fwd=-1 if half else 0, chunk_bwd=-1 if half else 0,
                                    forward_only=forward_only, count_pairs=count_pairs))
    return out


def _load_file(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _time_step(field, reps: int) -> float:
    dev = field.device
    field.forward()
    field.backward()
    torch.cuda.synchronize(dev)
    best = float("inf")
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        field.forward()
        field.backward()
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def _resolve_half(field, opt: FieldOptions) -> FieldOptions:
    """Replace the 'half stage' marker (-1) by half of the largest stage that fits."""
    if opt.chunk_fwd >= 0:
        return opt
    full = resolved(dataclasses.replace(opt, chunk_fwd=0, chunk_bwd=0))
    return dataclasses.replace(opt, chunk_fwd=max(32, full.chunk_fwd // 64 * 32),
                               chunk_bwd=max(32, full.chunk_bwd // 64 * 32))


def resolved(opt: FieldOptions) -> FieldOptions:
    """The launch configuration the library will use for ``opt`` on the current device
    (auto stage sizes, warps and schedule filled in)."""
    import ctypes
    from . import _lib
    out = _lib.Options()
    _lib.check(_lib.load().n3ds_field_resolve_options(ctypes.byref(opt.c()), ctypes.byref(out)))
    return dataclasses.replace(opt, chunk_fwd=int(out.chunk_fwd), chunk_bwd=int(out.chunk_bwd),
                               schedule={1: "segments", 2: "runs"}[int(out.schedule)],
                               rays_per_item=int(out.rays_per_item))


def tune(field, reps: int = 3, cands: Optional[List[FieldOptions]] = None, use_cache: bool = True,
         verbose: bool = False) -> FieldOptions:
    """Pick the fastest launch configuration for ``field`` and install it
    (``field.options``). Returns the chosen options."""
    key = signature(field)
    path = os.environ.get("N3DS_TUNE_CACHE")
    with _lock:
        hit = _memo.get(key)
        if hit is None and use_cache and path:
            hit = _load_file(path).get(key)
    if use_cache and hit is not None:
        best = FieldOptions(**hit["options"])
        field.options = best
        field._bind()
        return best
    base = field.options
    results = []
    for opt in cands or candidates(base.grad_mode, base.cull_alpha, base.forward_only, base.count_pairs):
        opt = _resolve_half(field, opt)
        field.options = opt
        field._bind()
        ms = _time_step(field, reps)
        results.append((ms, opt))
        if verbose:
            print(f"autotune {opt.schedule:8s} warps={opt.warps:2d}/{opt.warps_bwd:2d} "
                  f"chunk={opt.chunk_fwd}/{opt.chunk_bwd}: "
                  f"{ms:.3f} ms", flush=True)
    ms, best = min(results, key=lambda t: t[0])
    if cands is None and best.schedule == "segments":
        for rpi in (2, 4):
            opt = dataclasses.replace(best, rays_per_item=rpi)
            field.options = opt
            field._bind()
            t = _time_step(field, reps)
            results.append((t, opt))
            if verbose:
                print(f"autotune segments rays_per_item={rpi}: {t:.3f} ms", flush=True)
    last_results[:] = results
    ms, best = min(results, key=lambda t: t[0])
    field.options = best
    field._bind()
    entry = {"options": {k: v for k, v in dataclasses.asdict(best).items() if not k.startswith("_")},
             "ms": ms, "tried": len(results)}
    with _lock:
        _memo[key] = entry
        if path:
            data = _load_file(path)
            data[key] = entry
            tmp = path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
            os.replace(tmp, path)
    return best
