"""Accuracy of the fused stroke field at a benchmark workload's own shape.

TEST / CHECKER INFRASTRUCTURE ONLY: used by tests and by bench.py's untimed accuracy
leg, never by the product package, and never timed.

Method (``subset_accuracy``). The GPU runs the WHOLE workload through the caller's
``BatchedField``: every ray and every stroke of every scene, with the launch
configuration the bench times (several shared-memory stages per scene, the
forward's stroke-block masks, persistent CTAs handing scenes over). The upstream
gradients are zero except on a fixed, evenly spaced subset of rays per scene, so
every output and gradient the backward produces depends on that subset only: the
stroke-parameter gradients are sums over the subset's samples, the position
gradient is zero on every other ray (checked). The float64 oracle
(``oracle.render.render_strokes`` + torch.autograd, the reference chain
models.py:660-711 -> render.py:29-88) evaluates the same subset with every stroke of
its scene, and the reference CUDA op (oracle/_ref, driven as models.py drives it)
evaluates it as well.

Error measure: normwise relative error max|a - b| / max|b| per tensor and scene, the
worst scene reported. Depth is compared as acc * depth on all rays and as depth on
rays at least 1 % opaque; the upstream depth gradient is zero on rays less than 5 %
opaque (depth = D / acc is ill-conditioned where a ray barely meets a stroke).

Against the reference op the gradients are compared in compat mode (the fused
kernels reproducing the reference's own backward formulas, strokes_backward.cu /
compositing.cu); the exact gradients differ from the reference op by its known
divergences (cube exterior normal, scale through the soft-step width, Bezier
adjoints). Strokes of the quadratic Bezier type are left out of that comparison:
the reference's quadratic-Bezier adjoint (strokes_sdf.h:709-1172) is not restated.

``plain_op_compare``: the same fused field at full size (all rays carry upstream
gradients) against one plain reference-op call per scene (config 3: 16 sequential
calls), compat gradients.

``fd_slice``: a slice of rays x strokes whose fused-kernel gradients are checked
against float64 central finite differences of the oracle.
"""
import dataclasses
import math

import torch

from . import render as orr
from . import strokefield as sf

FWD_TOL = 1e-5
GRAD_TOL = 1e-4
DEPTH_GRAD_FLOOR = 0.05  # upstream depth gradient only on rays at least this opaque
DEPTH_FLOOR = 1e-2       # depth itself compared on rays at least this opaque


def rel(a, b):
    """Normwise relative error of a against b (float64 on the host)."""
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    if b.numel() == 0:
        return 0.0
    return float((a - b).abs().max() / max(float(b.abs().max()), 1e-30))


def ray_subset(n_rays, k):
    """k evenly spaced ray indices of 0 .. n_rays - 1 (first and last included)."""
    k = max(1, min(int(k), int(n_rays)))
    return torch.linspace(0, n_rays - 1, k, dtype=torch.float64).round().long().unique()


def take_rays(rays, idx):
    from neural3dstrokes_b200.scenes import RaySet
    f = lambda t: None if t is None else t[idx].contiguous()
    return RaySet(f(rays.origins), f(rays.dirs), f(rays.tdist), f(rays.x), f(rays.radius), f(rays.radii))


def used_slots(scene):
    """Boolean [S, 16] mask of the parameter slots each stroke uses."""
    m = torch.zeros_like(scene.shape_params, dtype=torch.bool)
    for i, sid in enumerate(scene.sdf_ids.tolist()):
        m[i, :sf.num_shape_params(sid)] = True
    return m


def oracle_scene(scene, rays, g_rgb, g_acc, g_depth, delta, laplace, inv, bg=1.0):
    """Float64 outputs and exact gradients of L = <rgb, g_rgb> + <acc, g_acc> +
    <depth, g_depth'> where g_depth' is g_depth on rays >= DEPTH_GRAD_FLOOR opaque and
    zero elsewhere. Returns (dict of tensors, g_depth')."""
    d = lambda t: t.detach().double().cpu()
    x = d(rays.x).requires_grad_(True)
    sp = d(scene.shape_params).requires_grad_(True)
    col = d(scene.color_params).requires_grad_(True)
    den = d(scene.density).requires_grad_(True)
    dl = torch.full((scene.n_strokes,), float(delta), dtype=torch.float64, requires_grad=True)
    rgb, acc, depth = orr.render_strokes(x, d(rays.radius), d(rays.tdist), d(rays.dirs), sp, scene.sdf_ids.cpu(),
                                         col, den, dl, laplace, inv, bg)
    gd = g_depth.double().cpu() * (acc.detach() >= DEPTH_GRAD_FLOOR).double()
    L = (rgb * g_rgb.double().cpu()).sum() + (acc * g_acc.double().cpu()).sum() + (depth * gd).sum()
    grads = torch.autograd.grad(L, [x, sp, col, den, dl], allow_unused=True)
    z = lambda g, r: torch.zeros_like(r) if g is None else g
    out = dict(rgb=rgb.detach(), acc=acc.detach(), depth=depth.detach(), x=z(grads[0], x), shape=z(grads[1], sp),
               color=z(grads[2], col), density=z(grads[3], den), delta=z(grads[4], dl))
    return out, gd.float()


def _errors(ours, ref, mask, names, has_x=True):
    """Per-output normwise errors of one scene (ours / ref: dicts of host tensors)."""
    e = {}
    if "rgb" in names:
        e["rgb"] = rel(ours["rgb"], ref["rgb"])
        e["acc"] = rel(ours["acc"], ref["acc"])
        e["acc_x_depth"] = rel(ours["depth"] * ours["acc"], ref["depth"] * ref["acc"])
        m = ref["acc"] >= DEPTH_FLOOR
        e["depth"] = rel(ours["depth"][m], ref["depth"][m]) if bool(m.any()) else 0.0
    if "shape" in names:
        e["grad_shape"] = rel(ours["shape"][mask], ref["shape"][mask])
        e["grad_color"] = rel(ours["color"], ref["color"])
        e["grad_density"] = rel(ours["density"], ref["density"])
        if "delta" in ref:
            e["grad_delta"] = rel(ours["delta"], ref["delta"])
        if has_x and "x" in ref:
            e["grad_x"] = rel(ours["x"], ref["x"])
    return e


def _worst(per_scene):
    out = {}
    for e in per_scene:
        for k, v in e.items():
            out[k] = max(out.get(k, 0.0), v)
    return out


def _within(errs, fwd_tol=FWD_TOL, grad_tol=GRAD_TOL):
    return all(v <= (grad_tol if k.startswith("grad_") else fwd_tol) for k, v in errs.items())


def _run_gpu(field, seeds, grad_mode):
    """Forward + backward of the caller's field with the given seeds (full-size
    tensors) in the given gradient mode; returns host copies of everything."""
    saved_opt = field.c_opt
    saved = [t.clone() for t in (field.g_rgb, field.g_acc, field.g_depth)]
    try:
        field.g_rgb.copy_(seeds[0])
        field.g_acc.copy_(seeds[1])
        field.g_depth.copy_(seeds[2])
        field.c_opt = dataclasses.replace(field.options, grad_mode=grad_mode).c()
        field.forward()
        field.backward()
        if field.device.type == "cuda":
            torch.cuda.synchronize(field.device)
        st, _ = field.status()
        res = dict(rgb=field.rgb.cpu(), acc=field.acc.cpu(), depth=field.depth.cpu(),
                   shape=field.grad_shape.cpu(), color=field.grad_color.cpu(), density=field.grad_density.cpu(),
                   delta=field.grad_delta.cpu(), x=field.grad_x.cpu() if field.grad_x is not None else None,
                   status=st)
    finally:
        field.c_opt = saved_opt
        field.g_rgb.copy_(saved[0])
        field.g_acc.copy_(saved[1])
        field.g_depth.copy_(saved[2])
    return res


def _split(res, r0, r1, s0, s1, idx):
    out = dict(rgb=res["rgb"][r0:r1][idx], acc=res["acc"][r0:r1][idx], depth=res["depth"][r0:r1][idx],
               shape=res["shape"][s0:s1], color=res["color"][s0:s1], density=res["density"][s0:s1],
               delta=res["delta"][s0:s1])
    if res.get("x") is not None:
        out["x"] = res["x"][r0:r1][idx]
    return out


def workload_from_field(field, w):
    """A copy of workload ``w`` whose scenes carry the field's current parameters
    (after training steps have moved them away from the generated ones)."""
    import copy
    from neural3dstrokes_b200.scenes import Scene
    out = copy.copy(w)
    out.scenes = []
    s0 = 0
    shape, color, dens = field.shape.detach().cpu(), field.color.detach().cpu(), field.density.detach().cpu()
    for sc in w.scenes:
        n = sc.n_strokes
        out.scenes.append(Scene(sc.kinds, sc.sdf_ids, shape[s0:s0 + n].clone(), color[s0:s0 + n].clone(),
                                dens[s0:s0 + n].clone()))
        s0 += n
    return out


def subset_accuracy(field, w, rays_per_scene, seed=0, ref=None):
    """Accuracy statement of ``field`` (a BatchedField over workload ``w``) on a fixed
    subset of ``rays_per_scene`` evenly spaced rays per scene. ``ref``: the reference
    extension (oracle/_ref) or None. Returns a JSON-ready dict."""
    g = torch.Generator().manual_seed(1234 + seed)
    R_tot = field.rgb.shape[0]
    seeds = [torch.zeros(R_tot, 3), torch.zeros(R_tot), torch.zeros(R_tot)]
    plan, oracles = [], []
    r0 = s0 = 0
    sub_pairs = 0
    for sc, rays in zip(w.scenes, w.rays):
        R, S = rays.n_rays, sc.n_strokes
        idx = ray_subset(R, rays_per_scene)
        sub = take_rays(rays, idx)
        k = idx.numel()
        g_rgb, g_acc, g_depth = torch.randn(k, 3, generator=g), torch.randn(k, generator=g), torch.randn(k, generator=g)
        o, gd = oracle_scene(sc, sub, g_rgb, g_acc, g_depth, w.sdf_delta, w.use_laplace, w.inv_scale_radius,
                             field.bg_value)
        seeds[0][r0 + idx] = g_rgb
        seeds[1][r0 + idx] = g_acc
        seeds[2][r0 + idx] = gd
        plan.append((r0, r0 + R, s0, s0 + S, idx, sub, (g_rgb, g_acc, gd)))
        oracles.append(o)
        sub_pairs += S * k * rays.n_samples
        r0 += R
        s0 += S
    dev = field.device
    ours = _run_gpu(field, [t.to(dev) for t in seeds], "exact")
    per_scene = []
    outside_nonzero = 0
    if ours["x"] is not None:
        inside = torch.zeros(R_tot, dtype=torch.bool)
        for (a, b, _, _, idx, _, _) in plan:
            inside[a + idx] = True
        outside_nonzero = int((ours["x"][~inside] != 0).any(dim=-1).any(dim=-1).sum())
    for (a, b, c, d, idx, _, _), o, sc in zip(plan, oracles, w.scenes):
        mine = _split(ours, a, b, c, d, idx)
        per_scene.append(_errors(mine, o, used_slots(sc), ("rgb", "shape"), has_x=ours["x"] is not None))
    vs64 = _worst(per_scene)
    out = {"rays_per_scene": int(rays_per_scene), "scenes": len(w.scenes), "subset_pairs": int(sub_pairs),
           "subset": "evenly spaced rays of each scene (first and last included), every stroke of the scene",
           "upstream": "N(0,1) on rgb and opacity of the subset rays, on depth where the oracle's opacity >= "
                       f"{DEPTH_GRAD_FLOOR}; zero on every other ray (the GPU runs the whole workload)",
           "metric": "max over scenes of max|ours - ref| / max|ref|; depth on rays >= 1% opaque",
           "tolerance": {"forward": FWD_TOL, "gradient": GRAD_TOL},
           "vs_fp64_oracle": vs64, "status_word": int(ours["status"]),
           "grad_x_nonzero_outside_subset": outside_nonzero,
           "ok": _within(vs64) and outside_nonzero == 0 and ours["status"] == 0}
    if ref is None:
        out["vs_reference_op"] = "unavailable: reference extension not built (oracle/_ref)"
        return out
    from .cpu_port import plain_op_step
    compat = _run_gpu(field, [t.to(dev) for t in seeds], "compat")
    fwd_ours, fwd_ref64, grad_vs_ref = [], [], []
    quad_sid = 0x90
    for (a, b, c, d, idx, sub, sd), o, sc in zip(plan, oracles, w.scenes):
        sub_d = sub.to(dev)
        r = plain_op_step(ref, sc.to(dev), sub_d.x, sub_d.radius, sub_d.tdist, sub_d.dirs, *(t.to(dev) for t in sd),
                          w.sdf_delta, w.use_laplace, w.inv_scale_radius, field.bg_value, return_grad_x=True)
        rr = dict(rgb=r[0].cpu(), acc=r[1].cpu(), depth=r[2].cpu(), shape=r[3].cpu(), color=r[4].cpu(),
                  density=r[5].cpu(), x=r[6].cpu().reshape(idx.numel(), -1, 3))
        mine = _split(ours, a, b, c, d, idx)
        fwd_ours.append(_errors(mine, rr, None, ("rgb",)))
        fwd_ref64.append(_errors(rr, o, None, ("rgb",)))
        mc = _split(compat, a, b, c, d, idx)
        keep = sc.sdf_ids.cpu() != quad_sid
        mask = used_slots(sc) & keep[:, None]
        grad_vs_ref.append(_errors(mc, rr, mask, ("shape",), has_x=bool(keep.all()) and mc.get("x") is not None))
    f_ours, f_ref = _worst(fwd_ours), _worst(fwd_ref64)
    gv = _worst(grad_vs_ref)
    # forward: within tolerance of the reference op, or never further from it than the
    # reference op is from float64 (its float32 closed-form Bezier solve is the larger
    # error on curve scenes)
    fwd_ok = all(f_ours[k] <= FWD_TOL or f_ours[k] <= f_ref[k] + FWD_TOL for k in f_ours)
    has_quad = any(bool((sc.sdf_ids.cpu() == quad_sid).any()) for sc in w.scenes)
    out["vs_reference_op"] = {
        "forward": f_ours, "reference_op_vs_fp64_oracle": f_ref, "compat_gradients": gv,
        "note": "gradients in compat mode (the reference's backward formulas); quadratic-Bezier strokes left "
                "out of the gradient comparison (their reference adjoint is not restated), and grad_x compared "
                "only on scenes without them",
        "gradient_bar": "applied" if not has_quad else
        "reported only: the reference op's float32 quadratic-Bezier forward (closest-point error up to ~4e-3 "
        "in t) changes the alphas that every gradient of the scene depends on",
        "ok": bool(fwd_ok and (has_quad or _within(gv))),
    }
    return out


def plain_op_compare(field, w, ref, seed=0):
    """The fused field at full size in compat mode against one reference-op call per
    scene over all of its rays (the sequential plain-op baseline), same upstream
    gradients on every ray (depth where the plain op's opacity >= DEPTH_GRAD_FLOOR).
    Returns a JSON-ready dict."""
    from .cpu_port import plain_op_step
    dev = field.device
    g = torch.Generator().manual_seed(4321 + seed)
    R_tot = field.rgb.shape[0]
    g_rgb, g_acc, g_depth = torch.randn(R_tot, 3, generator=g), torch.randn(R_tot, generator=g), \
        torch.randn(R_tot, generator=g)
    # the depth mask needs the opacity: one forward of the fused field first
    field.forward()
    if dev.type == "cuda":
        torch.cuda.synchronize(dev)
    g_depth = g_depth * (field.acc.cpu() >= DEPTH_GRAD_FLOOR).float()
    seeds = [g_rgb.to(dev), g_acc.to(dev), g_depth.to(dev)]
    mine = _run_gpu(field, seeds, "compat")
    per_scene = []
    r0 = s0 = 0
    has_quad = False
    for sc, rays in zip(w.scenes, w.rays):
        R, S = rays.n_rays, sc.n_strokes
        rd = rays.to(dev)
        r = plain_op_step(ref, sc.to(dev), rd.x, rd.radius, rd.tdist, rd.dirs, seeds[0][r0:r0 + R],
                          seeds[1][r0:r0 + R], seeds[2][r0:r0 + R], w.sdf_delta, w.use_laplace, w.inv_scale_radius,
                          field.bg_value, return_grad_x=True)
        rr = dict(rgb=r[0].cpu(), acc=r[1].cpu(), depth=r[2].cpu(), shape=r[3].cpu(), color=r[4].cpu(),
                  density=r[5].cpu(), x=r[6].cpu().reshape(R, -1, 3))
        del r
        allr = torch.arange(R)
        m = _split(mine, r0, r0 + R, s0, s0 + S, allr)
        keep = sc.sdf_ids.cpu() != 0x90
        has_quad = has_quad or not bool(keep.all())
        per_scene.append(_errors(m, rr, used_slots(sc) & keep[:, None], ("rgb", "shape"),
                                 has_x=bool(keep.all()) and m.get("x") is not None))
        r0 += R
        s0 += S
        torch.cuda.empty_cache()
    errs = _worst(per_scene)
    return {"calls": len(w.scenes), "rays": int(R_tot), "compat_errors": errs,
            "upstream": f"N(0,1) on rgb and opacity of every ray, on depth where opacity >= {DEPTH_GRAD_FLOOR}",
            "ok": _within(errs), "quadratic_bezier_left_out": has_quad}


def fd_slice(scene, rays, n_rays=32, n_strokes=8, delta=0.02, laplace=True, inv=True, h=1e-6, n_x=32,
             device="cuda", seed=0):
    """Gradients of the fused field (per-scene op ``render_strokes``, exact mode) on a
    slice of ``n_rays`` evenly spaced rays and the ``n_strokes`` strokes nearest to
    them (half of each type present, so both Bezier kinds appear on the spline
    workload), against float64 central finite differences of the oracle: every
    parameter of the slice's strokes (shape, colour, density, softness) and ``n_x``
    sample coordinates. Returns a JSON-ready dict."""
    from neural3dstrokes_b200.field import render_strokes
    from neural3dstrokes_b200.scenes import Scene
    idx = ray_subset(rays.n_rays, n_rays)
    sub = take_rays(rays, idx)
    pts = sub.x.reshape(-1, 3)
    S = scene.n_strokes
    ctrl = torch.zeros(S, 3)
    for i, sid in enumerate(scene.sdf_ids.tolist()):
        n = sf.num_shape_params(sid)
        row = scene.shape_params[i, :n]
        if (sid >> 4) >= 9:  # curves: mean of the control points
            k = (n - 2) // 3
            ctrl[i] = row[:3 * k].reshape(k, 3).mean(0)
        else:  # translation is the row's last three entries
            ctrl[i] = row[n - 3:n]
    dist = torch.cdist(ctrl, pts).min(dim=1).values
    kinds = sorted(set(scene.sdf_ids.tolist()))
    per = max(1, n_strokes // len(kinds))
    pick = []
    for sid in kinds:
        cand = [i for i in dist.argsort().tolist() if int(scene.sdf_ids[i]) == sid]
        pick += cand[:per]
    pick = sorted(pick[:n_strokes])
    it = torch.tensor(pick, dtype=torch.long)
    sl = Scene([scene.kinds[i] for i in pick], scene.sdf_ids[it], scene.shape_params[it].clone(),
               scene.color_params[it].clone(), scene.density[it].clone())
    g = torch.Generator().manual_seed(77 + seed)
    k = idx.numel()
    g_rgb, g_acc, g_depth = torch.randn(k, 3, generator=g), torch.randn(k, generator=g), torch.randn(k, generator=g)
    o, gd = oracle_scene(sl, sub, g_rgb, g_acc, g_depth, delta, laplace, inv)

    dev = torch.device(device)
    x = sub.x.to(dev).clone().requires_grad_(True)
    sp = sl.shape_params.to(dev).requires_grad_(True)
    col = sl.color_params.to(dev).requires_grad_(True)
    den = sl.density.to(dev).requires_grad_(True)
    dl = torch.full((len(pick),), float(delta), device=dev, requires_grad=True)
    rgb, acc, depth = render_strokes(x, sub.radius.to(dev), sub.tdist.to(dev), sub.dirs.to(dev), sp,
                                     sl.sdf_ids.to(dev), col, den, dl, laplace, inv)
    L = (rgb * g_rgb.to(dev)).sum() + (acc * g_acc.to(dev)).sum() + (depth * gd.to(dev)).sum()
    L.backward()
    gpu = dict(shape=sp.grad.cpu(), color=col.grad.cpu(), density=den.grad.cpu(), delta=dl.grad.cpu(),
               x=x.grad.cpu())

    d64 = lambda t: t.detach().double().cpu()
    base = dict(x=d64(sub.x), shape=d64(sl.shape_params), color=d64(sl.color_params), density=d64(sl.density),
                delta=torch.full((len(pick),), float(delta), dtype=torch.float64))
    gr64, ga64, gd64 = g_rgb.double(), g_acc.double(), gd.double()

    def loss(v):
        with torch.no_grad():
            rgb_, acc_, dep_ = orr.render_strokes(v["x"], d64(sub.radius), d64(sub.tdist), d64(sub.dirs), v["shape"],
                                                  sl.sdf_ids, v["color"], v["density"], v["delta"], laplace, inv)
            return float((rgb_ * gr64).sum() + (acc_ * ga64).sum() + (dep_ * gd64).sum())

    def fd(name, flat_idx):
        out = torch.zeros(len(flat_idx), dtype=torch.float64)
        for j, fi in enumerate(flat_idx):
            v = {k_: t.clone() for k_, t in base.items()}
            ref_t = v[name].view(-1)
            step = h * max(1.0, abs(float(ref_t[fi])))
            ref_t[fi] += step
            lp = loss(v)
            ref_t[fi] -= 2 * step
            lm = loss(v)
            out[j] = (lp - lm) / (2 * step)
        return out

    mask = used_slots(sl).view(-1).nonzero().view(-1).tolist()
    res = {}
    fd_shape = fd("shape", mask)
    res["grad_shape"] = (gpu["shape"].view(-1)[mask], o["shape"].view(-1)[mask], fd_shape)
    for name in ("color", "density", "delta"):
        n = base[name].numel()
        res["grad_" + name] = (gpu[name].view(-1), o[name].view(-1), fd(name, list(range(n))))
    # sample coordinates: the n_x with the largest oracle gradient magnitude
    ox = o["x"].reshape(-1)
    xi = ox.abs().argsort(descending=True)[:n_x].tolist()
    res["grad_x"] = (gpu["x"].reshape(-1)[xi], ox[xi], fd("x", xi))
    errs = {k_: rel(v[0], v[2]) for k_, v in res.items()}
    oracle_fd = {k_: rel(v[1], v[2]) for k_, v in res.items()}
    return {"rays": int(k), "strokes": len(pick), "stroke_kinds": sorted(set(sl.kinds)),
            "parameters": int(sum(v[2].numel() for v in res.values())), "h": h,
            "fused_vs_fd": errs, "oracle_autograd_vs_fd": oracle_fd,
            "tolerance": GRAD_TOL, "ok": _within({k_: v for k_, v in errs.items()})}
