"""Device stroke insertion (n3ds_insert_step / n3ds_ema_update / n3ds_clip_columns)
against the reference's update decisions (oracle/insertion.py, models.py:586-658):
stroke counts, update steps, resets, and which error samples / gradient rows feed
which strokes are exact; the random draws are checked against the samplers' ranges."""
import math

import pytest
import torch

from oracle import insertion as oin
from neural3dstrokes_b200 import insertion, scenes

pytestmark = pytest.mark.gpu


def cfg_of(ins, **kw):
    c = ins.config
    d = {"max_num_strokes": c.max_num_strokes, "init_num_strokes": c.init_num_strokes, "step_power": ins.step_power,
         "reset_density": c.reset_density, "use_error_field": bool(c.use_error_field),
         "use_shape_grads": bool(c.use_shape_grads), "min_update_interval": c.min_update_interval,
         "min_reset_interval": c.min_reset_interval, "max_reset_frac": c.max_reset_frac}
    d.update(kw)
    return d


def clipped(x, ranges):
    """clip_params (models.py:576-584) applied to every row, as the reference does."""
    lo = torch.tensor([a if a is not None else -math.inf for a, _ in ranges], device=x.device)
    hi = torch.tensor([b if b is not None else math.inf for _, b in ranges], device=x.device)
    return torch.maximum(torch.minimum(x, hi), lo)


def distinct_errors(E, g, dev):
    return (torch.randperm(E, generator=g).float() / E).to(dev)


def test_error_field_sequence_matches_reference_decisions(cuda):
    ins = insertion.StrokeInserter("sphere", "constant_rgb", "recon", max_num_strokes=64, init_num_strokes=4,
                                   min_reset_interval=5, error_point_samples=2000, seed=3, device=cuda)
    cfg = cfg_of(ins)
    g = torch.Generator().manual_seed(0)
    prev, last = 0, 0
    updates = resets_seen = 0
    for cur in range(0, 900, 7):
        if cur % 35 == 0 and prev > 6:  # some strokes fade out
            idx = torch.randint(0, prev, (3,), generator=g)
            ins.density_params[idx.to(cuda)] = 0.001
        coords, _ = ins.sample_error_coords()
        errors = distinct_errors(coords.shape[0], g, cuda)
        dens_before = ins.density_params.clone()
        shape_before = ins.shape_params.clone()
        p = oin.plan(prev, last, cur, 1000, dens_before.cpu(), cfg, errors.cpu())
        ins.step_update(cur, 1000, errors=errors, error_coords=coords)
        assert int(ins.stroke_step) == p["next"] and int(ins.last_update_step) == p["last"], cur
        if p["update"]:
            updates += 1
            new_rows = list(range(prev, p["next"]))
            rows = new_rows + p["resets"].tolist()
            resets_seen += p["resets"].numel()
            for q, row in enumerate(rows):
                if p["mode"] == "error":  # translation = the q-th largest error's coordinate
                    assert torch.allclose(ins.shape_params[row, 1:], coords[p["top"][q]]), (cur, q)
                s = float(ins.shape_params[row, 0])
                d = math.exp(-(prev + q if q < len(new_rows) else p["next"]) / 200)
                assert (0.02 + 0.12 * d) * math.sqrt(3) - 1e-6 <= s <= (0.04 + 0.18 * d) * math.sqrt(3) + 1e-6
            for row in p["resets"].tolist():
                assert float(ins.density_params[row]) == 1.0
            untouched = torch.ones(64, dtype=torch.bool)
            untouched[rows] = False
            want = clipped(shape_before, ins.shape_param_ranges)
            assert torch.equal(ins.shape_params[untouched.to(cuda)], want[untouched.to(cuda)])
        else:
            assert torch.equal(ins.shape_params, clipped(shape_before, ins.shape_param_ranges))
        prev, last = p["next"], p["last"]
    assert updates > 5 and resets_seen > 0 and prev == 64
    c = ins.color_params[:prev]
    assert float(c.min()) >= 0 and float(c.max()) <= 1 and float(c.std()) > 0.1


def test_shape_gradient_split_matches_reference(cuda):
    ins = insertion.StrokeInserter("ellipsoid", "constant_rgb", "recon", max_num_strokes=40, init_num_strokes=5,
                                   use_error_field=False, use_shape_grads=True, device=cuda, seed=1)
    cfg = cfg_of(ins)
    g = torch.Generator().manual_seed(2)
    prev, last = 0, 0
    checked = 0
    for cur in range(0, 700, 13):
        grad = torch.randn(40, ins.shape_params.shape[1], generator=g).to(cuda)
        ema_ref = ins.shape_params_grad * ins.shape_grad_ema + grad * (1 - ins.shape_grad_ema)
        shape_before = ins.shape_params.clone()
        p = oin.plan(prev, last, cur, 700, ins.density_params.cpu(), cfg, None, ema_ref.cpu())
        ins.step_update(cur, 700, shape_grad=grad)
        assert torch.allclose(ins.shape_params_grad, ema_ref, rtol=1e-6, atol=1e-7)
        assert int(ins.stroke_step) == p["next"]
        if p["update"] and p["mode"] == "grad":
            for q, row in enumerate(range(prev, p["next"])):
                if q < p["top"].numel():
                    want = clipped(shape_before[p["top"][q]] + ema_ref[q] * 0.05, ins.shape_param_ranges)
                    assert torch.allclose(ins.shape_params[row], want, atol=1e-6)
                    checked += 1
        prev, last = p["next"], p["last"]
    assert checked > 0


@pytest.mark.parametrize("init_type", ["recon", "gen_box", "gen_sphere"])
@pytest.mark.parametrize("shape_type", scenes.EVERY_KIND)
def test_samplers_stay_in_range(cuda, shape_type, init_type):
    color = {"sphere": "gradient_rgb", "capsule": "constant_sh2", "cubic_bezier": "constant_sh3"}.get(shape_type,
                                                                                                     "constant_rgb")
    ins = insertion.StrokeInserter(shape_type, color, init_type, max_num_strokes=300, init_num_strokes=300,
                                   device=cuda, seed=7)
    ins.step_update(0, 3000)
    assert int(ins.stroke_step) == 300
    sp = ins.shape_params
    assert torch.isfinite(sp).all() and torch.isfinite(ins.color_params).all()
    for j, (a, b) in enumerate(ins.shape_param_ranges):
        if a is not None:
            assert float(sp[:, j].min()) >= a
        if b is not None:
            assert float(sp[:, j].max()) <= b
        assert float(sp[:, j].std()) > 0 or sp.shape[0] == 1, (shape_type, j)  # every column is drawn
    if color == "constant_sh2":
        c = ins.color_params
        assert abs(float(c.mean())) < 0.15 and 0.85 < float(c.std()) < 1.15  # N(0, 1)


def test_large_topk_order(cuda):
    """k in the thousands out of 30000 samples: the kept coordinates follow torch.topk."""
    ins = insertion.StrokeInserter("sphere", "constant_rgb", "recon", max_num_strokes=4000, init_num_strokes=50,
                                   device=cuda, seed=5)
    g = torch.Generator().manual_seed(9)
    ins.step_update(0, 40000)  # the first strokes, no error field yet
    ins.step_update(100, 40000)
    prev = int(ins.stroke_step)
    assert prev > 50
    coords, _ = ins.sample_error_coords(30000)
    errors = distinct_errors(30000, g, cuda)
    cur = 8000
    nt, _ = ins.next_target(cur, 40000)
    ins.step_update(cur, 40000, errors=errors, error_coords=coords)
    nxt = int(ins.stroke_step)
    assert nxt == nt and nxt - prev > 1000
    top = torch.topk(errors, nxt - prev).indices
    assert torch.equal(ins.shape_params[prev:nxt, 1:], coords[top])


def test_step_update_does_not_synchronise(cuda):
    ins = insertion.StrokeInserter("capsule", "constant_rgb", "recon", max_num_strokes=100, init_num_strokes=5,
                                   device=cuda)
    grad = torch.randn(100, ins.shape_params.shape[1], device=cuda)
    coords, _ = ins.sample_error_coords(500)
    errors = torch.rand(500, device=cuda)
    torch.cuda.synchronize(cuda)
    torch.cuda.set_sync_debug_mode("error")
    try:
        for cur in range(0, 400, 10):
            ins.step_update(cur, 1000, shape_grad=grad, errors=errors, error_coords=coords)
    finally:
        torch.cuda.set_sync_debug_mode("default")
    assert int(ins.stroke_step) > 5
