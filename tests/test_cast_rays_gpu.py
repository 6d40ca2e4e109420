"""The fused field with samples cast in the kernels from the rays (render_rays) against
render_strokes given the samples that cast_rays (render.py:5-26) computes, in float32
with the same operation order: x = directions * t + origins, radius = radii * t,
t = (t0 + t1) / 2.

Forward outputs agree bit for bit (same sample positions, same kernels); gradients
agree to 1e-6 (the stroke-parameter sums are accumulated with atomics whose order
varies between launches)."""
import pytest
import torch

from helpers import rel, small_workload
from neural3dstrokes_b200 import scenes
from neural3dstrokes_b200.field import FieldOptions, render_rays, render_strokes

pytestmark = pytest.mark.gpu


def cast(origins, dirs, radii, tdist):
    t = (tdist[:, :-1] + tdist[:, 1:]) / 2
    x = dirs[:, None, :] * t[..., None]
    x = x + origins[:, None, :]
    return x, radii[:, None] * t


def params(sc, dev, delta=0.02):
    sp = sc.shape_params.to(dev).requires_grad_(True)
    col = sc.color_params.to(dev).requires_grad_(True)
    den = sc.density.to(dev).requires_grad_(True)
    dl = torch.full((sc.n_strokes,), float(delta), device=dev, requires_grad=True)
    return sp, col, den, dl


def both(sc, rays, dev, opts, laplace=True, inv=True, scene_sizes=None, bg=1.0):
    g = torch.Generator().manual_seed(11)
    radii = (torch.rand(rays.n_rays, generator=g) * 0.4 + 0.1).to(dev)
    o, d, td = rays.origins.to(dev), rays.dirs.to(dev), rays.tdist.to(dev)
    outs, grads = [], []
    up = [torch.randn(rays.n_rays, 3, generator=g).to(dev), torch.randn(rays.n_rays, generator=g).to(dev),
          torch.randn(rays.n_rays, generator=g).to(dev) * 0.1]
    for mode in ("cast", "explicit"):
        sp, col, den, dl = params(sc, dev)
        if mode == "cast":
            out = render_rays(o, d, radii, td, sp, sc.sdf_ids.to(dev), col, den, dl, laplace, inv, bg,
                              options=opts, scene_sizes=scene_sizes)
        else:
            x, r = cast(o, d, radii, td)
            out = render_strokes(x, r, td, d, sp, sc.sdf_ids.to(dev), col, den, dl, laplace, inv, bg, False, opts,
                                 scene_sizes=scene_sizes)
        loss = sum((o_ * u).sum() for o_, u in zip(out, up))
        loss.backward()
        outs.append([t.detach() for t in out])
        grads.append([t.grad for t in (sp, col, den, dl)])
    return outs, grads


@pytest.mark.parametrize("schedule", ["segments", "runs"])
@pytest.mark.parametrize("kind", ["sphere", "capsule", "cubic_bezier", "every"])
def test_cast_matches_explicit_samples(cuda, kind, schedule):
    sc, rays = small_workload(kind, n_strokes=24, n_rays=96, n_samples=48, seed=5)
    outs, grads = both(sc, rays, cuda, FieldOptions(schedule=schedule))
    for a, b in zip(*outs):
        assert torch.equal(a, b)
    for a, b in zip(*grads):
        assert rel(a, b) < 1e-6


@pytest.mark.parametrize("laplace,inv", [(False, True), (True, False)])
def test_cast_step_modes(cuda, laplace, inv):
    sc, rays = small_workload("mixed", n_strokes=20, n_rays=64, n_samples=33, seed=9)
    outs, grads = both(sc, rays, cuda, FieldOptions(), laplace=laplace, inv=inv)
    for a, b in zip(*outs):
        assert torch.equal(a, b)
    for a, b in zip(*grads):
        assert rel(a, b) < 1e-6


def test_cast_batched_scenes(cuda):
    parts = [small_workload(k, n_strokes=s, n_rays=r, n_samples=40, seed=i)
             for i, (k, s, r) in enumerate([("sphere", 12, 50), ("every", 30, 70), ("capsule", 5, 33)])]
    sc = scenes.Scene(sum((p[0].kinds for p in parts), []),
                      *(torch.cat([getattr(p[0], f) for p in parts])
                        for f in ("sdf_ids", "shape_params", "color_params", "density")))
    rays = scenes.RaySet(*(torch.cat([getattr(p[1], f) for p in parts])
                           for f in ("origins", "dirs", "tdist", "x", "radius")))
    sizes = [(p[1].n_rays, p[0].n_strokes) for p in parts]
    outs, grads = both(sc, rays, cuda, FieldOptions(), scene_sizes=sizes)
    for a, b in zip(*outs):
        assert torch.equal(a, b)
    for a, b in zip(*grads):
        assert rel(a, b) < 1e-6


def test_cast_rejects_bad_shapes(cuda):
    sc, rays = small_workload("sphere", n_strokes=4, n_rays=8, n_samples=8)
    sp, col, den, dl = params(sc, cuda)
    with pytest.raises(ValueError):
        render_rays(rays.origins.to(cuda), rays.dirs.to(cuda)[:4], torch.ones(8, device=cuda), rays.tdist.to(cuda),
                    sp, sc.sdf_ids.to(cuda), col, den, dl)


@pytest.mark.parametrize("schedule", ["segments", "runs"])
def test_batched_field_cast_mode(cuda, schedule):
    from neural3dstrokes_b200.train import BatchedField
    g = torch.Generator().manual_seed(21)
    parts = [(scenes.make_strokes([scenes.EVERY_KIND[int(i)] for i in torch.randint(0, len(scenes.EVERY_KIND), (s,),
                                                                                    generator=g)], g),
              scenes.make_rays(r, 56, g, base_radius=0.25)) for s, r in [(30, 80), (9, 45)]]
    fields = [BatchedField([p[0] for p in parts], [p[1] for p in parts], options=FieldOptions(schedule=schedule),
                           device=cuda, cast=c) for c in (True, False)]
    up = torch.Generator().manual_seed(2)
    g_rgb = torch.randn(fields[0].g_rgb.shape, generator=up)
    g_acc = torch.randn(fields[0].g_acc.shape, generator=up)
    for f in fields:
        f.g_rgb.copy_(g_rgb)
        f.g_acc.copy_(g_acc)
        f.step()
    torch.cuda.synchronize(cuda)
    a, b = fields
    assert a.grad_x is None
    for name in ("rgb", "acc", "depth"):
        assert torch.equal(getattr(a, name), getattr(b, name)), name
    for name in ("grad_shape", "grad_color", "grad_density", "grad_delta"):
        assert rel(getattr(a, name), getattr(b, name)) < 1e-6, name
    assert a.status()[0] == 0


def test_in_kernel_cast_matches_reference_cast_rays_golden(cuda):
    """The samples the kernels cast from the rays are the reference cast_rays' own
    (tests/golden/cast_golden.npz, float32 outputs of render.py:5-26): render_rays on
    the golden rays equals render_strokes on the golden coords and radii, forward bit
    for bit and gradients to 1e-6, and both are within 1e-5 / 1e-4 of the float64
    oracle evaluated at the golden samples."""
    import os

    import numpy as np

    from helpers import GRAD_TOL, FWD_TOL, oracle_grads
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cast_golden.npz"))
    t = lambda k: torch.from_numpy(z[k])
    R = t("tdist").shape[0]
    g = torch.Generator().manual_seed(6)
    sc = scenes.make_strokes([scenes.MIXED_PRIMS[int(i)] for i in torch.randint(0, 6, (48,), generator=g)], g)
    delta = 2.0  # sample radii are ~0.01: a soft width comparable to the strokes
    up = [torch.randn(R, 3, generator=g), torch.randn(R, generator=g)]
    outs, grads = [], []
    for mode in ("cast", "explicit"):
        sp, col, den, dl = params(sc, cuda, delta)
        ids = sc.sdf_ids.to(cuda)
        if mode == "cast":
            out = render_rays(t("origins").to(cuda), t("directions").to(cuda), t("radii").to(cuda),
                              t("tdist").to(cuda), sp, ids, col, den, dl)
        else:
            out = render_strokes(t("coords").to(cuda), t("radius").to(cuda), t("tdist").to(cuda),
                                 t("directions").to(cuda), sp, ids, col, den, dl)
        ((out[0] * up[0].to(cuda)).sum() + (out[1] * up[1].to(cuda)).sum()).backward()
        outs.append([o.detach() for o in out])
        grads.append([p.grad for p in (sp, col, den, dl)])
    for a, b in zip(*outs):
        assert torch.equal(a, b)
    for a, b in zip(*grads):
        assert rel(a, b) < 1e-6
    rays = scenes.RaySet(t("origins"), t("directions"), t("tdist"), t("coords"), t("radius"))
    ref = oracle_grads(sc, rays, up[0], up[1], torch.zeros(R), delta=delta)
    assert rel(outs[0][0], ref["rgb"]) < FWD_TOL and rel(outs[0][1], ref["acc"]) < FWD_TOL
    assert rel(grads[0][0], ref["shape"]) < GRAD_TOL and rel(grads[0][1], ref["color"]) < GRAD_TOL
