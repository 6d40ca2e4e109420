"""Autotuner: option resolution on the host (CPU) and a tuning pass on a small batch
(GPU) that must leave the results unchanged. Tolerance: forward 1e-5 (helpers)."""
import dataclasses
import json

import pytest
import torch

from helpers import FWD_TOL, rel
from neural3dstrokes_b200 import autotune, scenes
from neural3dstrokes_b200.field import FieldOptions


def test_resolved_options_fill_in_auto_values():
    for schedule in ("segments", "runs"):
        r = autotune.resolved(FieldOptions(schedule=schedule))
        assert r.schedule == schedule
        assert r.chunk_fwd >= 32 and r.chunk_fwd % 32 == 0
        assert r.chunk_bwd >= 32 and r.chunk_bwd % 32 == 0
    assert autotune.resolved(FieldOptions()).schedule == "segments"
    # explicit stages are kept
    r = autotune.resolved(FieldOptions(chunk_fwd=64, chunk_bwd=96))
    assert (r.chunk_fwd, r.chunk_bwd) == (64, 96)


def test_rays_per_item_resolves_to_one_two_or_four():
    got = [autotune.resolved(FieldOptions(rays_per_item=r)).rays_per_item for r in (0, 1, 2, 3, 4, 9)]
    assert got == [1, 1, 2, 2, 4, 4]


@pytest.mark.gpu
@pytest.mark.parametrize("rpi", [2, 4])
def test_rays_per_item_keeps_results(cuda, rpi):
    """Larger work claims change which warp renders which ray, nothing else: forward
    outputs bit-equal, gradients equal up to the order of float atomics."""
    from neural3dstrokes_b200.train import BatchedField
    w = scenes.config(3, scale=0.02)
    out = []
    for r in (1, rpi):
        f = BatchedField(w.scenes[:5], w.rays[:5], options=FieldOptions(rays_per_item=r), device=cuda)
        g = torch.Generator().manual_seed(1)
        f.g_rgb.copy_(torch.randn(f.rgb.shape, generator=g))
        f.g_acc.copy_(torch.randn(f.acc.shape, generator=g))
        f.forward()
        f.backward()
        torch.cuda.synchronize()
        out.append((f.rgb.clone(), f.acc.clone(), f.grad_shape.clone(), f.grad_x.clone() if f.grad_x is not None
                    else None))
    (r1, a1, s1, x1), (r2, a2, s2, x2) = out
    assert torch.equal(r1, r2) and torch.equal(a1, a2)
    assert rel(s2, s1) < 1e-5
    if x1 is not None:
        assert torch.equal(x1, x2)


def test_candidate_set_covers_schedules_warps_and_stages():
    c = autotune.candidates()
    assert {o.schedule for o in c} == {"segments", "runs"}
    assert {o.warps for o in c} >= {16, 24, 32} and {o.warps_bwd for o in c} >= {16, 20, 24}
    assert {o.chunk_fwd for o in c} == {0, -1}


class _FakeField:
    """Stands in for BatchedField in the cache logic (no device work)."""

    def __init__(self):
        self.kinds = ["cube", "sphere"]
        self.scene_rays = [1000, 70]
        self.scene_strokes = [2, 0]
        self.n_samples = 64
        self.laplace = True
        self.inv_scale = True
        self.options = FieldOptions()
        self.binds = 0

    def _bind(self):
        self.binds += 1


def test_signature_rounds_ray_counts_and_cache_file(tmp_path, monkeypatch):
    f = _FakeField()
    key = autotune.signature(f)
    assert json.loads(key)["rays"] == [1024, 64]
    path = tmp_path / "tune.json"
    best = FieldOptions(schedule="runs", chunk_fwd=64, chunk_bwd=32)
    path.write_text(json.dumps({key: {"options": dataclasses.asdict(best), "ms": 1.0, "tried": 8}}))
    monkeypatch.setenv("N3DS_TUNE_CACHE", str(path))
    got = autotune.tune(f)
    assert got == best and f.options == best and f.binds == 1


@pytest.mark.gpu
def test_tuning_keeps_results(cuda):
    from neural3dstrokes_b200.train import BatchedField
    w = scenes.config(3, scale=0.02)
    field = BatchedField(w.scenes[:4], w.rays[:4], device=cuda)
    field.forward()
    torch.cuda.synchronize()
    ref = field.rgb.clone()
    best = autotune.tune(field, reps=1, use_cache=False)
    assert field.options == best
    field.forward()
    torch.cuda.synchronize()
    assert rel(field.rgb, ref) < FWD_TOL
