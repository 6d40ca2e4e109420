"""The reference stroke-field step on CPU cores (labelled port) and on the GPU (the
unmodified reference op from oracle/_ref).

TEST / CPU-BASELINE INFRASTRUCTURE ONLY: used by tests and by bench.py's CPU-baseline
and reference legs, never by the product package.

Both run the chain the reference model runs for one training step of the stroke
field (models.py:660-711, 191-235; train.py:132-139):
  stroke_fn per primitive group (one sdf_id per call, models.py:681-684) -> alphas
  scattered into stroke order -> compose_strokes('over') -> compute_alpha_weights ->
  volumetric_rendering, then the backward in the opposite order (torch autograd for
  the render math, the reference compose and stroke adjoints).

``port_step``: float32, the torch restatement of the reference kernels
(oracle.strokefield) on the host cores.
``plain_op_step``: the reference CUDA extension (oracle/_ref/_strokelib*.so), ray
chunked so that P_chunk * S stays below 2**31 (its 32-bit thread index,
strokes_forward.cu:35-37) and its [P, S] tensors fit in memory.
"""
import glob
import importlib.machinery
import importlib.util
import os

import torch

from . import render as orr
from . import strokefield as sf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _groups(sdf_ids):
    ids = sdf_ids.tolist()
    out = {}
    for i, v in enumerate(ids):
        out.setdefault(int(v), []).append(i)
    return {k: torch.tensor(v, dtype=torch.long) for k, v in out.items()}


def port_step(scene, x, radius, tdist, dirs, g_rgb, g_acc, g_depth, delta=0.02, laplace=True, inv=True, bg=1.0):
    """One forward + backward of the reference chain in float32 on CPU.
    x [R,N,3] ... ; returns (rgb, acc, depth, grad_shape, grad_color, grad_density, grad_x)."""
    R, N, _ = x.shape
    P, S = R * N, scene.n_strokes
    xf, rf = x.reshape(-1, 3), radius.reshape(-1)
    groups = _groups(scene.sdf_ids)
    alphas = torch.zeros(P, S)
    for sid, idx in groups.items():
        ps = scene.shape_params[idx][:, :sf.num_shape_params(sid)]
        a, _ = sf.stroke_forward(xf, rf, ps, scene.color_params[idx], sid, delta, laplace, inv)
        alphas[:, idx] = a
    colors = scene.color_params[None].expand(P, S, 3)
    dens, col = sf.compose_forward(alphas, colors, scene.density)
    dens_t = dens.reshape(R, N).requires_grad_(True)
    col_t = col.reshape(R, N, 3).requires_grad_(True)
    w = orr.compute_alpha_weights(dens_t, tdist, dirs)[0]
    rgb, depth, acc = orr.volumetric_rendering(col_t, w, tdist, bg)
    L = (rgb * g_rgb).sum() + (acc * g_acc).sum() + (depth * g_depth).sum()
    g_dens, g_col = torch.autograd.grad(L, [dens_t, col_t])
    ga, gc, gd = sf.compose_backward_compat(g_dens.reshape(-1), g_col.reshape(-1, 3), alphas, colors,
                                            scene.density)
    grad_shape = torch.zeros_like(scene.shape_params)
    grad_color = torch.zeros_like(scene.color_params)
    grad_x = torch.zeros(P, 3)
    for sid, idx in groups.items():
        n = sf.num_shape_params(sid)
        ps = scene.shape_params[idx][:, :n]
        gs, gcol, gx = sf.stroke_backward_compat(ga[:, idx], gc[:, idx], xf, rf, alphas[:, idx], ps,
                                                 scene.color_params[idx], sid, delta, laplace, inv)
        grad_shape[idx, :n] = gs
        grad_color[idx] = gcol
        grad_x += gx
    return rgb.detach(), acc.detach(), depth.detach(), grad_shape, grad_color, gd, grad_x.reshape(R, N, 3)


def reference_extension():
    hits = sorted(glob.glob(os.path.join(ROOT, "oracle", "_ref", "_strokelib*.so")))
    if not hits:
        return None
    loader = importlib.machinery.ExtensionFileLoader("_strokelib", hits[0])
    spec = importlib.util.spec_from_file_location("_strokelib", hits[0], loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def plain_op_step(ref, scene, x, radius, tdist, dirs, g_rgb, g_acc, g_depth, delta=0.02, laplace=True, inv=True,
                  bg=1.0, max_pairs=1 << 29, return_grad_x=False):
    """One forward + backward through the reference CUDA op, ray-chunked, with the
    sample-position gradient requested as well. All tensors on the GPU. Returns
    (rgb, acc, depth, grad_shape, grad_color, grad_density), plus grad_x [R*N, 3]
    when ``return_grad_x``."""
    dev = x.device
    R, N, _ = x.shape
    S = scene.n_strokes
    groups = {k: v.to(dev) for k, v in _groups(scene.sdf_ids.cpu()).items()}
    chunk = max(1, min(R, max_pairs // max(1, S * N)))
    rgb = torch.empty(R, 3, device=dev)
    acc = torch.empty(R, device=dev)
    depth = torch.empty(R, device=dev)
    grad_shape = torch.zeros_like(scene.shape_params)
    grad_color = torch.zeros_like(scene.color_params)
    grad_density = torch.zeros_like(scene.density)
    empty = torch.empty(0, device=dev)
    grad_x = torch.empty(R * N, 3, device=dev) if return_grad_x else None
    for r0 in range(0, R, chunk):
        r1 = min(R, r0 + chunk)
        xc = x[r0:r1].reshape(-1, 3).contiguous()
        rc = radius[r0:r1].reshape(-1).contiguous()
        vd = dirs[r0:r1].contiguous()
        P = xc.shape[0]
        alphas = torch.empty(P, S, device=dev)
        saved = {}
        for sid, idx in groups.items():
            ps = scene.shape_params[idx][:, :sf.num_shape_params(sid)].contiguous()
            cp = scene.color_params[idx].contiguous()
            a = torch.empty(P, idx.numel(), device=dev)
            c = torch.empty(P, idx.numel(), 3, device=dev)
            ref.stroke_forward(a, c, empty, empty, xc, rc, vd, ps, cp, sid, 0, delta, laplace, inv)
            alphas[:, idx] = a
            saved[sid] = (a, ps, cp)
        colors = scene.color_params[None].expand(P, S, 3).contiguous()
        dens = torch.empty(P, device=dev)
        col = torch.empty(P, 3, device=dev)
        ref.compose_forward(dens, col, alphas, colors, scene.density)
        dens_t = dens.reshape(r1 - r0, N).requires_grad_(True)
        col_t = col.reshape(r1 - r0, N, 3).requires_grad_(True)
        w = orr.compute_alpha_weights(dens_t, tdist[r0:r1], dirs[r0:r1])[0]
        rg, dp, ac = orr.volumetric_rendering(col_t, w, tdist[r0:r1], bg)
        L = (rg * g_rgb[r0:r1]).sum() + (ac * g_acc[r0:r1]).sum() + (dp * g_depth[r0:r1]).sum()
        g_dens, g_col = torch.autograd.grad(L, [dens_t, col_t])
        rgb[r0:r1], acc[r0:r1], depth[r0:r1] = rg.detach(), ac.detach(), dp.detach()
        ga = torch.zeros_like(alphas)
        gc = torch.zeros_like(colors)
        ref.compose_backward(ga, gc, grad_density, g_dens.reshape(-1).contiguous(),
                             g_col.reshape(-1, 3).contiguous(), alphas, colors, scene.density)
        gx = torch.zeros(P, 3, device=dev)
        for sid, idx in groups.items():
            a, ps, cp = saved[sid]
            gs = torch.zeros_like(ps)
            gcol = torch.zeros_like(cp)
            ref.stroke_backward(gs, gcol, gx, ga[:, idx].contiguous(), gc[:, idx].contiguous(), empty, xc, rc,
                                vd, a, ps, cp, sid, 0, delta, laplace, inv)
            grad_shape[idx, :ps.shape[1]] += gs
            grad_color[idx] += gcol
        if return_grad_x:
            grad_x[r0 * N:r1 * N] = gx
    if return_grad_x:
        return rgb, acc, depth, grad_shape, grad_color, grad_density, grad_x
    return rgb, acc, depth, grad_shape, grad_color, grad_density


def plain_op_train(ref, scenes, rays, targets, steps, lr=1e-3, betas=(0.9, 0.99), eps=1e-15, delta=0.02,
                   laplace=True, inv=True, ranges=None):
    """MSE training of the stroke parameters through the reference CUDA op, as the
    reference trains the stroke field: per step and scene, forward and backward of
    the op chain (plain_op_step), then torch Adam (utils/training.py:119-136) over
    shape, colour and density, then the parameter clamp of StrokeField.clip_params
    (models.py:576-584). ``scenes``/``rays``/``targets`` on the GPU; ``ranges``: per
    scene (lo, hi) tensors of the shape parameters. Returns the loss of every step
    (before that step's update) and the trained scenes."""
    import copy
    scenes = [copy.copy(s) for s in scenes]
    params = []
    for s in scenes:
        s.shape_params = s.shape_params.clone().requires_grad_(True)
        s.color_params = s.color_params.clone().requires_grad_(True)
        s.density = s.density.clone().requires_grad_(True)
        params += [s.shape_params, s.color_params, s.density]
    opt = torch.optim.Adam(params, lr=lr, betas=betas, eps=eps)
    n_total = sum(t.numel() for t in targets)
    losses = []
    for _ in range(steps):
        loss = 0.0
        grads = []
        # plain_op_step differentiates the render math with torch autograd itself; the
        # stroke parameters go in detached (their gradients come from the reference op)
        for s, r, t in zip(scenes, rays, targets):
            det = copy.copy(s)
            det.shape_params, det.color_params, det.density = (s.shape_params.detach(), s.color_params.detach(),
                                                              s.density.detach())
            zr = torch.zeros(r.n_rays, 3, device=t.device)
            z = torch.zeros(r.n_rays, device=t.device)
            rgb = plain_op_step(ref, det, r.x, r.radius, r.tdist, r.dirs, zr, z, z, delta, laplace, inv)[0]
            diff = rgb - t
            loss += float((diff * diff).sum())
            g_rgb = diff * (2.0 / n_total)
            _, _, _, gs, gc, gd = plain_op_step(ref, det, r.x, r.radius, r.tdist, r.dirs, g_rgb, z, z, delta,
                                                laplace, inv)
            grads += [gs, gc, gd]
        losses.append(loss / n_total)
        for p, g in zip(params, grads):
            p.grad = torch.nan_to_num(g)
        opt.step()
        with torch.no_grad():
            for i, s in enumerate(scenes):
                lo, hi = ranges[i]
                s.shape_params.copy_(torch.minimum(torch.maximum(s.shape_params, lo), hi))
                s.color_params.clamp_(0.0, 1.0)
                s.density.clamp_(min=0.0)
    return losses, scenes
