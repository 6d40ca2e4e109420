"""Parity of the fused stroke field (CUDA, through the C ABI) with the float64 oracle.

Tolerances (helpers.rel, normwise): forward 1e-5, gradients 1e-4.
"""
import pytest
import torch

from helpers import (FWD_TOL, GRAD_TOL, depth_errors, depth_upstream, oracle_forward, oracle_grads, rel,
                     shape_param_mask, small_workload)
from neural3dstrokes_b200 import scenes
from neural3dstrokes_b200.field import FieldOptions, render_strokes

pytestmark = pytest.mark.gpu

KINDS = scenes.EVERY_KIND + ["mixed", "every"]


def run_field(sc, rays, dev, delta=0.02, laplace=True, inv=True, bg=1.0, opaque=False, opts=None,
              requires_grad=False, x_grad=True):
    x = rays.x.to(dev).requires_grad_(requires_grad and x_grad)
    sp = sc.shape_params.to(dev).requires_grad_(requires_grad)
    col = sc.color_params.to(dev).requires_grad_(requires_grad)
    den = sc.density.to(dev).requires_grad_(requires_grad)
    dl = torch.full((sc.n_strokes,), float(delta), device=dev, requires_grad=requires_grad)
    out = render_strokes(x, rays.radius.to(dev), rays.tdist.to(dev), rays.dirs.to(dev), sp, sc.sdf_ids.to(dev),
                         col, den, dl, laplace, inv, bg.to(dev) if torch.is_tensor(bg) else bg, opaque, opts)
    return out, (x, sp, col, den, dl)


SCHEDULES = ["runs", "segments"]


@pytest.mark.parametrize("schedule", SCHEDULES)
@pytest.mark.parametrize("kind", KINDS)
def test_forward_matches_oracle(cuda, kind, schedule):
    sc, rays = small_workload(kind)
    (rgb, acc, depth), _ = run_field(sc, rays, cuda, opts=FieldOptions(schedule=schedule))
    rgb_r, acc_r, depth_r = oracle_forward(sc, rays)
    assert rel(rgb, rgb_r) < FWD_TOL
    assert rel(acc, acc_r) < FWD_TOL
    e1, e2 = depth_errors(depth.cpu(), acc.cpu(), depth_r, acc_r)
    assert e1 < FWD_TOL and e2 < FWD_TOL


@pytest.mark.parametrize("x_grad", [True, False])
@pytest.mark.parametrize("schedule", SCHEDULES)
@pytest.mark.parametrize("kind", KINDS)
def test_backward_matches_float64_autograd(cuda, kind, schedule, x_grad):
    sc, rays = small_workload(kind, n_strokes=16, n_rays=64, n_samples=40, seed=3)
    g = torch.Generator().manual_seed(7)
    g_rgb = torch.randn(rays.n_rays, 3, generator=g)
    g_acc = torch.randn(rays.n_rays, generator=g)
    g_depth = depth_upstream(sc, rays, g)
    (rgb, acc, depth), (x, sp, col, den, dl) = run_field(sc, rays, cuda, requires_grad=True,
                                                         opts=FieldOptions(schedule=schedule), x_grad=x_grad)
    L = (rgb * g_rgb.to(cuda)).sum() + (acc * g_acc.to(cuda)).sum() + (depth * g_depth.to(cuda)).sum()
    L.backward()
    ref = oracle_grads(sc, rays, g_rgb, g_acc, g_depth)
    m = shape_param_mask(sc)
    errs = {
        "x": rel(x.grad, ref["x"]) if x_grad else 0.0,
        "shape": rel(sp.grad.cpu()[m], ref["shape"][m]),
        "color": rel(col.grad, ref["color"]),
        "density": rel(den.grad, ref["density"]),
        "delta": rel(dl.grad, ref["delta"]),
    }
    assert all(v < GRAD_TOL for v in errs.values()), errs
    # unused padding slots get exactly zero gradient
    assert float(sp.grad.cpu()[~m].abs().max()) == 0.0


def test_config0_forward(cuda):
    w = scenes.config(0, scale=0.25)
    sc, rays = w.scenes[0], w.rays[0]
    (rgb, acc, depth), _ = run_field(sc, rays, cuda)
    rgb_r, acc_r, depth_r = oracle_forward(sc, rays)
    assert rel(rgb, rgb_r) < FWD_TOL and rel(acc, acc_r) < FWD_TOL
    e1, e2 = depth_errors(depth.cpu(), acc.cpu(), depth_r, acc_r)
    assert e1 < FWD_TOL and e2 < FWD_TOL


@pytest.mark.parametrize("kind", ["mixed", "every", "ellipsoid", "capsule", "cube", "roundcube"])
@pytest.mark.parametrize("schedule", SCHEDULES)
def test_culling_is_invisible(cuda, schedule, kind):
    sc, rays = small_workload(kind, n_strokes=64, n_rays=256, n_samples=64, seed=11)
    (a, acc_a, _), _ = run_field(sc, rays, cuda, opts=FieldOptions(cull_alpha=1e-9, schedule=schedule))
    (b, acc_b, _), _ = run_field(sc, rays, cuda, opts=FieldOptions(cull_alpha=0.0, schedule=schedule))
    assert rel(a, b) < 1e-6 and rel(acc_a, acc_b) < 1e-6


@pytest.mark.parametrize("n_samples,shuffle", [(100, False), (64, True), (1, False), (33, True), (200, False)])
def test_schedules_agree(cuda, n_samples, shuffle):
    """Sample runs and 32-sample segments give the same outputs and gradients, also
    for partial 64-sample units, single-sample rays and samples out of ray order
    (which the run schedule must not cull by chord intervals)."""
    sc, rays = small_workload("mixed", n_strokes=150, n_rays=40, n_samples=n_samples, seed=21)
    if shuffle:
        perm = torch.randperm(n_samples, generator=torch.Generator().manual_seed(4))
        rays = scenes.RaySet(rays.origins, rays.dirs, rays.tdist, rays.x[:, perm].contiguous(),
                             rays.radius[:, perm].contiguous())
    g_rgb = torch.randn(rays.n_rays, 3, generator=torch.Generator().manual_seed(1)).to(cuda)
    outs = []
    for schedule in SCHEDULES:
        (rgb, acc, depth), (x, sp, col, den, dl) = run_field(sc, rays, cuda, requires_grad=True,
                                                             opts=FieldOptions(schedule=schedule))
        ((rgb * g_rgb).sum() + acc.sum()).backward()
        outs.append((rgb.detach(), acc.detach(), x.grad, sp.grad, col.grad, den.grad, dl.grad))
    for a, b in zip(*outs):
        assert rel(a, b) < 1e-5


@pytest.mark.parametrize("x_grad", [True, False])
def test_multipass_matches_single_pass(cuda, x_grad):
    """Several shared-memory stages per scene (also stage sizes that are not multiples
    of 32, which are rounded down) give the single-stage results."""
    sc, rays = small_workload("every", n_strokes=100, n_rays=96, n_samples=70, seed=5)
    g_rgb = torch.randn(rays.n_rays, 3, generator=torch.Generator().manual_seed(1)).to(cuda)
    outs = []
    for opts in (FieldOptions(), FieldOptions(chunk_fwd=32, chunk_bwd=32),
                 FieldOptions(chunk_fwd=32, chunk_bwd=32, schedule="segments"),
                 FieldOptions(chunk_fwd=100, chunk_bwd=70, schedule="segments")):
        (rgb, acc, depth), (x, sp, col, den, dl) = run_field(sc, rays, cuda, opts=opts, requires_grad=True,
                                                             x_grad=x_grad)
        (rgb * g_rgb).sum().backward()
        outs.append((rgb.detach(), x.grad if x_grad else rgb.detach(), sp.grad, col.grad, den.grad, dl.grad))
    for other in outs[1:]:
        for a, b in zip(other, outs[0]):
            assert rel(a, b) < 1e-5


def test_batched_scenes_match_individual(cuda):
    parts = [small_workload(k, n_strokes=n, n_rays=r, n_samples=48, seed=i)
             for i, (k, n, r) in enumerate([("mixed", 40, 64), ("cube", 7, 33), ("cubic_bezier", 19, 90)])]
    x = torch.cat([p[1].x for p in parts]).to(cuda).requires_grad_(True)
    sp = torch.cat([p[0].shape_params for p in parts]).to(cuda).requires_grad_(True)
    col = torch.cat([p[0].color_params for p in parts]).to(cuda)
    den = torch.cat([p[0].density for p in parts]).to(cuda)
    ids = torch.cat([p[0].sdf_ids for p in parts]).to(cuda)
    cat = lambda f: torch.cat([f(p[1]) for p in parts]).to(cuda)
    rgb, acc, depth = render_strokes(x, cat(lambda r: r.radius), cat(lambda r: r.tdist), cat(lambda r: r.dirs), sp,
                                     ids, col, den, 0.02,
                                     scene_sizes=[(p[1].n_rays, p[0].n_strokes) for p in parts])
    rgb.sum().backward()
    r0 = s0 = 0
    for sc, rays in parts:
        (rgb1, _, _), (x1, sp1, _, _, _) = run_field(sc, rays, cuda, requires_grad=True)
        rgb1.sum().backward()
        assert rel(rgb[r0:r0 + rays.n_rays], rgb1) < 1e-6
        assert rel(x.grad[r0:r0 + rays.n_rays], x1.grad) < 1e-5
        assert rel(sp.grad[s0:s0 + sc.n_strokes], sp1.grad) < 1e-5
        r0 += rays.n_rays
        s0 += sc.n_strokes


@pytest.mark.parametrize("laplace,delta,opaque", [(False, 0.05, False), (True, 0.02, True), (True, 0.0, False)])
def test_step_modes_and_opaque_background(cuda, laplace, delta, opaque):
    sc, rays = small_workload("mixed", n_strokes=20, n_rays=64, n_samples=32, seed=9)
    bg = torch.rand(rays.n_rays, 3, generator=torch.Generator().manual_seed(2))
    (rgb, acc, depth), _ = run_field(sc, rays, cuda, delta=delta, laplace=laplace, bg=bg, opaque=opaque)
    rgb_r, acc_r, depth_r = oracle_forward(sc, rays, delta=delta, laplace=laplace, bg=bg, opaque=opaque)
    assert rel(rgb, rgb_r) < FWD_TOL and rel(acc, acc_r) < FWD_TOL


def test_empty_scene_and_rays(cuda):
    sc, rays = small_workload("sphere", n_strokes=0, n_rays=16, n_samples=32)
    (rgb, acc, depth), _ = run_field(sc, rays, cuda)
    assert float(acc.abs().max()) == 0.0
    assert torch.allclose(rgb, torch.ones_like(rgb))
    sc2, rays2 = small_workload("sphere", n_strokes=4, n_rays=0, n_samples=32)
    (rgb2, acc2, _), _ = run_field(sc2, rays2, cuda)
    assert rgb2.shape == (0, 3) and acc2.shape == (0,)


def test_backward_without_matching_block_masks(cuda):
    """The backward reads the forward's stroke-block masks only when they were written
    with its skip threshold; after a forward of the run schedule (which writes none),
    a forward-only pass, or a forward at another threshold, it visits every block and
    gives the same gradients."""
    from neural3dstrokes_b200.train import BatchedField
    sc, rays = small_workload("every", n_strokes=90, n_rays=128, n_samples=64, seed=8)
    f = BatchedField([sc], [rays], device=cuda)
    g = torch.Generator().manual_seed(3)
    f.g_rgb.copy_(torch.randn(f.g_rgb.shape, generator=g))
    f.g_acc.copy_(torch.randn(f.g_acc.shape, generator=g))
    f.step()
    ref = [t.clone() for t in (f.grad_x, f.grad_shape, f.grad_color, f.grad_density, f.grad_delta)]
    seg = FieldOptions(schedule="segments")
    for first, second in ((FieldOptions(schedule="runs"), seg), (FieldOptions(forward_only=True), seg),
                          (seg, FieldOptions(schedule="segments", cull_alpha=1e-8))):
        f.c_opt = first.c()
        f.forward()
        f.c_opt = second.c()
        f.backward()
        for a, b in zip((f.grad_x, f.grad_shape, f.grad_color, f.grad_density, f.grad_delta), ref):
            assert rel(a, b) < 1e-5


def test_forward_only_outputs_are_identical(cuda):
    """A forward that records nothing for a backward (no input needs a gradient) gives
    the same outputs bit for bit."""
    sc, rays = small_workload("every", n_strokes=60, n_rays=100, n_samples=50, seed=4)
    (a, acc_a, d_a), _ = run_field(sc, rays, cuda, requires_grad=True)
    with torch.no_grad():
        (b, acc_b, d_b), _ = run_field(sc, rays, cuda)
    assert torch.equal(a.detach(), b) and torch.equal(acc_a.detach(), acc_b) and torch.equal(d_a.detach(), d_b)


def test_pair_counters_only_when_requested(cuda):
    """options.count_pairs fills the evaluated-pair counters (forward per base type,
    backward total); without it they stay 0 and the outputs are the same."""
    from neural3dstrokes_b200.train import BatchedField
    sc, rays = small_workload("mixed", n_strokes=60, n_rays=96, n_samples=64, seed=2)
    out = []
    for count in (True, False):
        f = BatchedField([sc], [rays], options=FieldOptions(count_pairs=count), device=cuda)
        f.g_rgb.fill_(1.0)
        f.step()
        st, pairs = f.status()
        per_base, bwd = f.pair_counts(), f.backward_pairs()
        assert st == 0
        if count:
            assert pairs > 0 and sum(per_base) == pairs and 0 < bwd <= pairs
        else:
            assert pairs == 0 and sum(per_base) == 0 and bwd == 0
        out.append((f.rgb.clone(), f.grad_shape.clone()))
    assert torch.equal(out[0][0], out[1][0])
    assert rel(out[0][1], out[1][1]) < 1e-5


@pytest.mark.parametrize("chunk", [0, 64])
def test_backward_warp_counts_agree(cuda, chunk):
    """The 32-warp backward build (64 registers) gives the 24-warp results."""
    sc, rays = small_workload("every", n_strokes=90, n_rays=80, n_samples=64, seed=8)
    g_rgb = torch.randn(rays.n_rays, 3, generator=torch.Generator().manual_seed(3)).to(cuda)
    outs = []
    for wb in (24, 32):
        opts = FieldOptions(schedule="segments", warps_bwd=wb, chunk_bwd=chunk)
        (rgb, acc, depth), (x, sp, col, den, dl) = run_field(sc, rays, cuda, opts=opts, requires_grad=True)
        ((rgb * g_rgb).sum() + acc.sum()).backward()
        outs.append((x.grad, sp.grad, col.grad, den.grad, dl.grad))
    for a, b in zip(*outs):
        assert rel(a, b) < 1e-5


@pytest.mark.parametrize("kind", ["mixed_primitives", "ellipsoid", "capsule"])
def test_common_primitive_build_matches_general_build(cuda, kind):
    """A field whose strokes are all common primitives (its kind list gives the base
    hint) runs the forward build that carries only their code; its outputs and the
    batched field's gradients match the general build (render_strokes passes no hint)
    on the same inputs."""
    from neural3dstrokes_b200.train import BatchedField
    g = torch.Generator().manual_seed(41)
    kinds = ([scenes.MIXED_PRIMS[i % 6] for i in range(60)] if kind == "mixed_primitives" else [kind] * 60)
    sc = scenes.make_strokes(kinds, g)
    rays = scenes.make_rays(80, 64, g)
    f = BatchedField([sc], [rays], device=cuda)
    assert f.c_strokes.base_mask != 0
    up = [torch.randn(t.shape, generator=g).to(cuda) for t in (f.g_rgb, f.g_acc, f.g_depth)]
    for dst, u in zip((f.g_rgb, f.g_acc, f.g_depth), up):
        dst.copy_(u)
    f.step()
    torch.cuda.synchronize()
    (rgb, acc, depth), leaves = run_field(sc, rays, cuda, requires_grad=True)
    assert rel(f.rgb, rgb) < 1e-6 and rel(f.acc, acc) < 1e-6
    assert f.status()[0] == 0
    torch.autograd.backward([rgb, acc, depth], up)
    for ours, leaf in zip((f.grad_x, f.grad_shape, f.grad_color, f.grad_density, f.grad_delta), leaves):
        assert rel(ours, leaf.grad) < 1e-5
