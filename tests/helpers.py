"""Shared test utilities: error metrics, small seeded scenes, oracle wrappers.

Error metric (used for every tolerance in these tests): the normwise relative error
    rel(a, b) = max_i |a_i - b_i| / max(max_i |b_i|, 1e-30)
of a tensor against its oracle value b. Forward tolerance 1e-5, gradient 1e-4.
Depth is compared as acc * depth (the expected ray distance, well conditioned) on
all rays, and as depth itself on rays with acc >= 1e-2 (depth = D / acc is
ill-conditioned where a ray barely touches any stroke).
"""
import torch

from neural3dstrokes_b200 import scenes
from oracle import render as orr
from oracle import strokefield as sf

FWD_TOL = 1e-5
GRAD_TOL = 1e-4


def rel(a, b):
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    if b.numel() == 0:
        return 0.0
    return float((a - b).abs().max() / max(float(b.abs().max()), 1e-30))


def small_workload(kind, n_strokes=24, n_rays=128, n_samples=48, seed=0):
    g = torch.Generator().manual_seed(seed)
    if kind == "mixed":
        kinds = [scenes.ALL_KINDS[int(i)] for i in torch.randint(0, 8, (n_strokes,), generator=g)]
    elif kind == "every":
        n = len(scenes.EVERY_KIND)
        kinds = [scenes.EVERY_KIND[int(i)] for i in torch.randint(0, n, (n_strokes,), generator=g)]
    else:
        kinds = [kind] * n_strokes
    sc = scenes.make_strokes(kinds, g)
    rays = scenes.make_rays(n_rays, n_samples, g)
    return sc, rays


def oracle_forward(sc, rays, delta=0.02, laplace=True, inv=True, bg=1.0, opaque=False, dtype=torch.float64):
    d = lambda t: t.to(dtype)
    return orr.render_strokes(d(rays.x), d(rays.radius), d(rays.tdist), d(rays.dirs), d(sc.shape_params),
                              sc.sdf_ids, d(sc.color_params), d(sc.density), delta, laplace, inv,
                              bg if not torch.is_tensor(bg) else d(bg), opaque)


def depth_upstream(sc, rays, g, delta=0.02, thresh=0.05):
    """Random upstream depth gradient, zero on rays less than 5% opaque (where
    depth = D / acc is ill-conditioned and culling-sensitive)."""
    _, acc, _ = oracle_forward(sc, rays, delta=delta)
    return torch.randn(rays.n_rays, generator=g) * (acc > thresh).float()


def oracle_grads(sc, rays, g_rgb, g_acc, g_depth, delta=0.02, laplace=True, inv=True, bg=1.0, opaque=False):
    """Exact float64 gradients (torch.autograd of the oracle) of
    L = <rgb, g_rgb> + <acc, g_acc> + <depth, g_depth>."""
    d = lambda t: t.double()
    x = d(rays.x).requires_grad_(True)
    sp = d(sc.shape_params).requires_grad_(True)
    col = d(sc.color_params).requires_grad_(True)
    den = d(sc.density).requires_grad_(True)
    dl = torch.full((sc.n_strokes,), float(delta), dtype=torch.float64, requires_grad=True)
    rgb, acc, depth = orr.render_strokes(x, d(rays.radius), d(rays.tdist), d(rays.dirs), sp, sc.sdf_ids, col,
                                         den, dl, laplace, inv, bg if not torch.is_tensor(bg) else d(bg), opaque)
    L = (rgb * d(g_rgb)).sum() + (acc * d(g_acc)).sum() + (depth * d(g_depth)).sum()
    gx, gsp, gcol, gden, gdl = torch.autograd.grad(L, [x, sp, col, den, dl], allow_unused=True)
    z = lambda g, ref: torch.zeros_like(ref) if g is None else g
    return dict(x=z(gx, x), shape=z(gsp, sp), color=z(gcol, col), density=z(gden, den), delta=z(gdl, dl),
                rgb=rgb.detach(), acc=acc.detach(), depth=depth.detach())


def depth_errors(depth, acc, depth_ref, acc_ref):
    e1 = rel(depth * acc, depth_ref * acc_ref)
    m = acc_ref >= 1e-2
    e2 = rel(depth[m.to(depth.device)], depth_ref[m]) if bool(m.any()) else 0.0
    return e1, e2


def shape_param_mask(sc):
    """Boolean [S, 16] mask of the parameter slots each stroke actually uses."""
    m = torch.zeros_like(sc.shape_params, dtype=torch.bool)
    for i, sid in enumerate(sc.sdf_ids.tolist()):
        m[i, :sf.num_shape_params(sid)] = True
    return m
