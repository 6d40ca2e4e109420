"""Generate the golden fixtures under tests/golden/ from the reference itself.

Three sources, each a seeded, small input set:

--layouts   (CPU, needs the reference checkout): imports the reference
            source/strokelib/strokes.py with a stub ``_strokelib`` module and records,
            per shape type, the sdf_id, parameter count and clamp ranges that
            get_stroke produces (strokes.py:95-106, 227-313). -> layouts.json
--render    (CPU, needs the reference checkout): imports the reference
            source/utils/render.py and runs compute_alpha_weights (plain and opaque
            background) and volumetric_rendering in float64 on seeded inputs.
            -> render_golden.npz
--cast      (CPU, needs the reference checkout): imports the reference
            source/utils/render.py and runs cast_rays (render.py:5-26) in float32 on
            rays of the benchmark geometry. -> cast_golden.npz
--strokespy (CPU, needs the reference checkout): imports the reference
            source/strokelib/strokes.py with a recording ``_strokelib`` (the oracle's
            float32 port) and drives get_stroke / stroke_fn / compose_strokes and the
            backward per shape type as models.py does; records every backend call's
            arguments and results. -> strokes_py_calls.json, strokes_py_calls.npz
--compose   (CPU, needs the reference checkout): imports the reference strokes.py with a
            stub ``_strokelib`` and runs its torch compositing modes (max,
            max_density_weighted, softmax, softmax_density_weighted,
            strokes.py:390-417) in float64 with autograd. -> compose_modes_golden.npz
--stepfun   (CPU, needs the reference checkout): imports the reference
            source/utils/stepfun.py and coord.py and runs, in float32, max_dilate_weights,
            sample_intervals (deterministic, single and per-sample jitter; the jitter
            draws are recorded by re-seeding) and the proposal-level chain of
            models.py:147-185 (dilate, slice, logits, sample, s_to_t).
            -> stepfun_golden.npz
--strokelib (GPU, needs oracle/_ref built from the reference sources by
            oracle/build_ref.py): runs the reference CUDA operators stroke_forward,
            stroke_backward, compose_forward, compose_backward on seeded inputs for
            every implemented primitive. -> strokelib_golden.npz
--gridlayout (CPU, needs the reference checkout): imports the reference
            source/gridencoder/grid.py with a stub ``_gridencoder`` module and records
            the parameter layout (offsets, grid_sizes, per-level idx counts, n_params,
            output_dim, per_level_scale) that GridEncoder.__init__ builds for the
            proposal / error networks' settings (models.py:305-333, 505-509) and
            other shapes. -> grid_layouts.json
--grid      (GPU, needs oracle/_ref/grid built by oracle/build_ref.py): runs the
            reference grid_encode_forward (with dy_dx), grid_encode_backward and
            grad_total_variation kernels on seeded small tables, hash and tiled,
            linear and smoothstep, both corner alignments, D 2 and 3, C 1 to 8, in
            float32, float64 and float16. -> grid_golden.npz

Usage: python tests/golden/make_golden.py [--layouts] [--render] [--cast] [--strokespy] [--compose] [--stepfun] [--strokelib]
       [--gridlayout] [--grid]
       [--ref PATH] [--out tests/golden]
"""
import argparse
import copy
import glob
import importlib.machinery
import importlib.util
import json
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def make_layouts(ref_root, out):
    sys.modules["_strokelib"] = types.ModuleType("_strokelib")  # stub backend: never called
    path = os.path.join(ref_root, "source", "strokelib", "strokes.py")
    spec = importlib.util.spec_from_file_location("ref_strokes", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    pristine = copy.deepcopy(mod._sdf_dict)
    res = {}
    for name in pristine:
        mod._sdf_dict = copy.deepcopy(pristine)  # get_stroke mutates the range lists in place
        base, _, _, t, r, s1, s3 = mod._sdf_dict[name]
        _, d_shape, d_color, sranges, cranges, _, _ = mod.get_stroke(name, "constant_rgb", "recon")
        res[name] = {
            "sdf_id": mod._make_sdf_id(base, t, r, s1, s3),
            "dim_shape": d_shape,
            "dim_color": d_color,
            "shape_ranges": [[None if a is None else float(a), None if b is None else float(b)] for a, b in sranges],
        }
    del sys.modules["_strokelib"]
    with open(os.path.join(out, "layouts.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)
    print("layouts:", len(res), "shape types")


def make_compose_modes(ref_root, out):
    sys.modules["_strokelib"] = types.ModuleType("_strokelib")  # stub backend: 'over' is not called
    path = os.path.join(ref_root, "source", "strokelib", "strokes.py")
    spec = importlib.util.spec_from_file_location("ref_strokes_compose", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    g = torch.Generator().manual_seed(77)
    arrays = {}
    for C in (1, 3):
        a = torch.rand(2, 16, 23, generator=g, dtype=torch.float64) ** 2
        c = torch.rand(2, 16, 23, C, generator=g, dtype=torch.float64)
        d = torch.rand(23, generator=g, dtype=torch.float64) * 10
        gd = torch.randn(2, 16, generator=g, dtype=torch.float64)
        gc = torch.randn(2, 16, C, generator=g, dtype=torch.float64)
        for k, v in dict(alphas=a, colors=c, density_params=d, g_density=gd, g_color=gc).items():
            arrays[f"c{C}/{k}"] = v.numpy()
        for mode in ("max", "max_density_weighted", "softmax", "softmax_density_weighted"):
            ta, tc, td = (t.clone().requires_grad_(True) for t in (a, c, d))
            dens, col = mod.compose_strokes(ta, tc, td, mode)
            ((dens * gd).sum() + (col * gc).sum()).backward()
            for k, v in dict(density=dens, color=col, grad_alphas=ta.grad, grad_colors=tc.grad,
                             grad_density_params=td.grad).items():
                arrays[f"c{C}/{mode}/{k}"] = v.detach().numpy()
    del sys.modules["_strokelib"]
    np.savez_compressed(os.path.join(out, "compose_modes_golden.npz"), **arrays)
    print("compose modes golden written:", len(arrays), "arrays")


def make_render(ref_root, out):
    sys.path.insert(0, ref_root)
    from source.utils import render as ref_render  # noqa: E402
    g = torch.Generator().manual_seed(1234)
    R, N = 96, 40
    density = (torch.rand(R, N, generator=g, dtype=torch.float64) ** 4) * 30
    density[torch.rand(R, N, generator=g) < 0.3] = 0
    rgbs = torch.rand(R, N, 3, generator=g, dtype=torch.float64)
    t0 = 2 + torch.rand(R, 1, generator=g, dtype=torch.float64)
    steps = torch.rand(R, N, generator=g, dtype=torch.float64) * 0.2 + 0.01
    tdist = torch.cat([t0, t0 + torch.cumsum(steps, -1)], -1)
    dirs = torch.randn(R, 3, generator=g, dtype=torch.float64)
    bg = torch.rand(R, 3, generator=g, dtype=torch.float64)
    w, a, tr = ref_render.compute_alpha_weights(density, tdist, dirs)
    wo, ao, tro = ref_render.compute_alpha_weights(density, tdist, dirs, opaque_background=True)
    rend = ref_render.volumetric_rendering(rgbs, w, tdist, bg, tdist[..., -1:], False)
    rend1 = ref_render.volumetric_rendering(rgbs, wo, tdist, 1.0, tdist[..., -1:], False)
    np.savez_compressed(os.path.join(out, "render_golden.npz"), density=density.numpy(), rgbs=rgbs.numpy(),
                        tdist=tdist.numpy(), dirs=dirs.numpy(), bg=bg.numpy(), weights=w.numpy(),
                        alpha=a.numpy(), trans=tr.numpy(), weights_opaque=wo.numpy(), rgb=rend["rgb"].numpy(),
                        depth=rend["depth"].numpy(), acc=rend["acc"].numpy(), rgb_opaque=rend1["rgb"].numpy(),
                        depth_opaque=rend1["depth"].numpy(), acc_opaque=rend1["acc"].numpy())
    print("render golden written")


def make_cast(ref_root, out):
    """The reference cast_rays (render.py:5-26) in float32 on rays of the benchmark
    geometry (origins on the radius-4 sphere, jittered directions, stratified fence
    posts in [2, 6]) with per-ray base radii [R, 1] as batch['radii']."""
    sys.path.insert(0, ref_root)
    from source.utils import render as ref_render  # noqa: E402
    from neural3dstrokes_b200 import scenes
    g = torch.Generator().manual_seed(4321)
    R, N = 256, 48
    rays = scenes.make_rays(R, N, g)
    radii = (torch.rand(R, 1, generator=g) * 0.004 + 0.001).float()
    tdist, origins, dirs = rays.tdist.float(), rays.origins.float(), rays.dirs.float()
    coords, radius, t = ref_render.cast_rays(tdist, origins, dirs, radii)
    np.savez_compressed(os.path.join(out, "cast_golden.npz"), tdist=tdist.numpy(), origins=origins.numpy(),
                        directions=dirs.numpy(), radii=radii.numpy(), coords=coords.numpy(),
                        radius=radius.numpy(), t=t.numpy())
    print("cast golden written")


# output arguments (written by the call) of each _strokelib function, by position
STROKELIB_OUTPUTS = {"stroke_forward": (0, 1, 2, 3), "stroke_backward": (0, 1, 2), "compose_forward": (0, 1),
                     "compose_backward": (0, 1, 2)}


class _RecordingBackend(types.ModuleType):
    """A ``_strokelib`` module whose four functions compute with the oracle's float32
    port on the host and record every call the reference strokes.py makes: each
    argument's shape, dtype and value (outputs before and after the call)."""

    def __init__(self):
        super().__init__("_strokelib")
        self.calls, self.arrays = [], {}
        from oracle import strokefield as sf
        self.sf = sf

    def _record(self, name, args, fn):
        k = len(self.calls)
        outs = STROKELIB_OUTPUTS[name]
        meta = []
        for i, a in enumerate(args):
            if torch.is_tensor(a):
                key = f"c{k}/a{i}"
                meta.append({"tensor": key, "shape": list(a.shape), "dtype": str(a.dtype).replace("torch.", ""),
                             "contiguous": bool(a.is_contiguous()), "output": i in outs,
                             "zero_before": bool(a.numel() == 0 or not bool(a.any()))})
                if i not in outs:
                    self.arrays[key] = a.detach().numpy().copy()
            else:
                meta.append({"value": a, "type": type(a).__name__})
        fn()
        for i in outs:
            self.arrays[f"c{k}/a{i}"] = args[i].detach().numpy().copy()
        self.calls.append({"fn": name, "args": meta})

    def stroke_forward(self, *args):
        def run():
            a, c, sdf, tex, x, r, vd, ps, cp, sid, cid, delta, lap, inv = args
            aa, cc = self.sf.stroke_forward(x, r, ps, cp, sid, delta, lap, inv, color_id=cid, viewdir=vd)
            a.copy_(aa)
            c.copy_(cc)
        self._record("stroke_forward", args, run)

    def stroke_backward(self, *args):
        def run():
            gs, gcol, gx, ga, gc, gsdf, x, r, vd, a, ps, cp, sid, cid, delta, lap, inv = args
            s_, c_, x_ = self.sf.stroke_backward_compat(ga, gc, x, r, a, ps, cp, sid, delta, lap, inv)
            gs += s_
            gcol += c_
            if gx.numel():
                gx += x_
        self._record("stroke_backward", args, run)

    def compose_forward(self, *args):
        def run():
            d, c, alphas, colors, dp = args
            dd, cc = self.sf.compose_forward(alphas, colors, dp)
            d.copy_(dd)
            c.copy_(cc)
        self._record("compose_forward", args, run)

    def compose_backward(self, *args):
        def run():
            ga, gc, gdp, gd, gcol, alphas, colors, dp = args
            a_, c_, p_ = self.sf.compose_backward_compat(gd, gcol, alphas, colors, dp)
            ga += a_
            gc += c_
            gdp += p_
        self._record("compose_backward", args, run)


def make_strokes_py(ref_root, out):
    """The reference's own strokes.py (source/strokelib/strokes.py) driven as the
    model drives it (models.py:681-684, 709): per shape type, get_stroke(type,
    'constant_rgb', 'recon'), stroke_fn(coords, radius, viewdirs, shape, colour,
    sdf_delta, laplace, inv_scale_radius, True, False), compose_strokes(..., 'over'),
    and a backward. Its backend is a recording module, so the log holds exactly the
    calls strokes.py makes into _strokelib. -> strokes_py_calls.json / .npz"""
    from neural3dstrokes_b200 import scenes
    rec = _RecordingBackend()
    saved = sys.modules.get("_strokelib")
    sys.modules["_strokelib"] = rec
    try:
        path = os.path.join(ref_root, "source", "strokelib", "strokes.py")
        spec = importlib.util.spec_from_file_location("ref_strokes_recorded", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        assert mod._backend is rec
        g = torch.Generator().manual_seed(99)
        groups = []
        for kind in scenes.EVERY_KIND:
            stroke_fn, d_shape, _, _, _, _, _ = mod.get_stroke(kind, "constant_rgb", "recon")
            R, N, S = 4, 8, 5
            sc = scenes.make_strokes([kind] * S, g)
            rays = scenes.make_rays(R, N, g)
            # centre every stroke on a sample of the rays, so that each call carries
            # alphas well above any culling threshold
            pts = rays.x.reshape(-1, 3)
            pick = torch.randint(0, pts.shape[0], (S,), generator=g)
            # (off the sample itself: the per-axis radius factor is 0/0 at a stroke's centre)
            pts = pts.clone()
            pts[pick] += torch.randn(S, 3, generator=g) * 0.03
            n = sc.shape_params.shape[1]
            for i in range(S):
                k = scenes.N_PARAMS[kind]
                row = sc.shape_params[i]
                if kind in ("quadratic_bezier", "cubic_bezier", "catmull_rom"):
                    m = (k - 2) // 3
                    ctrl = row[:3 * m].reshape(m, 3)
                    row[:3 * m] = (ctrl - ctrl.mean(0) + pts[pick[i]]).reshape(-1)
                else:
                    row[k - 3:k] = pts[pick[i]]
            x = rays.x.clone().requires_grad_(True)
            shape = sc.shape_params[:, :d_shape].clone().requires_grad_(True)
            color = sc.color_params.clone().requires_grad_(True)
            dens = (torch.rand(S, generator=g) * 0.8 + 0.2).requires_grad_(True)
            first = len(rec.calls)
            alphas, colors, _, _ = stroke_fn(x, rays.radius, rays.dirs, shape, color, 0.05, True, True, True, False)
            density, col = mod.compose_strokes(alphas, colors, dens * 20.0, "over")
            w1, w2 = torch.randn(density.shape, generator=g), torch.randn(col.shape, generator=g)
            ((density * w1).sum() + (col * w2).sum()).backward()
            groups.append({"kind": kind, "calls": list(range(first, len(rec.calls)))})
    finally:
        if saved is None:
            sys.modules.pop("_strokelib", None)
        else:
            sys.modules["_strokelib"] = saved
    with open(os.path.join(out, "strokes_py_calls.json"), "w") as f:
        json.dump({"source": "source/strokelib/strokes.py (reference), recorded backend", "groups": groups,
                   "calls": rec.calls}, f)
    np.savez_compressed(os.path.join(out, "strokes_py_calls.npz"), **rec.arrays)
    print("strokes.py call log written:", len(rec.calls), "calls")


def make_stepfun(ref_root, out):
    sys.path.insert(0, ref_root)
    from source.utils import coord as ref_coord  # noqa: E402
    from source.utils import stepfun as ref_stepfun  # noqa: E402
    g = torch.Generator().manual_seed(77)
    R, M = 48, 64
    # level-0 style posts in [0, 1] with a few zero-width bins, peaked weights with zeros
    steps = torch.rand(R, M, generator=g) + 0.05
    steps[torch.rand(R, M, generator=g) < 0.05] = 0.0
    t = torch.cat([torch.zeros(R, 1), torch.cumsum(steps, -1)], -1)
    t = t / t[:, -1:]
    w = torch.rand(R, M, generator=g) ** 6
    w[torch.rand(R, M, generator=g) < 0.2] = 0.0
    w[0] = 0.0
    w[0, 17] = 1.0  # all weight in one bin
    w = w / w.sum(-1, keepdim=True).clamp_min(1e-12)
    dilation = 0.0025 + 0.5 / 64
    td, wd = ref_stepfun.max_dilate_weights(t, w, dilation, domain=(0.0, 1.0), renormalize=True)
    sd, wsl = td[..., 1:-1], wd[..., 1:-1]
    logits = torch.where(sd[..., 1:] > sd[..., :-1], torch.log(wsl + 0.0), torch.full_like(sd[..., :-1], -torch.inf))
    res = {"t": t, "w": w, "dilation": np.float64(dilation), "t_dilate": td, "w_dilate": wd, "logits": logits}
    N = 32
    res["s_det"] = ref_stepfun.sample_intervals(False, sd, logits, N, single_jitter=True, domain=(0.0, 1.0))
    for name, single in (("single", True), ("multi", False)):
        torch.manual_seed(5)
        res["s_" + name] = ref_stepfun.sample_intervals(True, sd, logits, N, single_jitter=single, domain=(0.0, 1.0))
        torch.manual_seed(5)
        res["jit_" + name] = torch.rand(R, 1 if single else N)
    # the first level: one interval [0, 1] of weight 1, 64 proposal samples, then s_to_t
    near = 2.0 + torch.rand(R, 1, generator=g)
    far = near + 1.0 + 3 * torch.rand(R, 1, generator=g)
    _, s_to_t = ref_coord.construct_ray_warps(None, near, far)
    s0 = torch.cat([torch.zeros(R, 1), torch.ones(R, 1)], -1)
    l0 = torch.log(torch.ones(R, 1) + 0.0)
    torch.manual_seed(9)
    s1 = ref_stepfun.sample_intervals(True, s0, l0, 64, single_jitter=True, domain=(0.0, 1.0))
    torch.manual_seed(9)
    res["jit_level0"] = torch.rand(R, 1)
    res.update(near=near, far=far, s_level0=s1, t_level0=s_to_t(s1))
    np.savez_compressed(os.path.join(out, "stepfun_golden.npz"),
                        **{k: (v.numpy() if torch.is_tensor(v) else v) for k, v in res.items()})
    print("stepfun golden written")


KINDS = ["sphere", "ellipsoid", "aacube", "cube", "aabb", "obb", "roundcube", "roundbox", "cappedtorus", "capsule",
         "scapsule", "line", "triprism", "octahedron", "tetrahedron", "quadratic_bezier", "cubic_bezier", "catmull_rom"]


def make_strokelib(out):
    from neural3dstrokes_b200 import scenes
    from oracle import strokefield as sf
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "_strokelib*.so"))
    if not hits:
        raise SystemExit("oracle/_ref/_strokelib*.so missing: run python oracle/build_ref.py")
    loader = importlib.machinery.ExtensionFileLoader("_strokelib", hits[0])
    spec = importlib.util.spec_from_file_location("_strokelib", hits[0], loader=loader)
    ref = importlib.util.module_from_spec(spec)
    loader.exec_module(ref)
    dev = torch.device("cuda:0")
    arrays = {}
    for ki, kind in enumerate(KINDS):
        g = torch.Generator().manual_seed(500 + ki)
        sc = scenes.make_strokes([kind] * 12, g)
        rays = scenes.make_rays(20, 16, g)
        sid = scenes.SDF_ID[kind]
        ps = sc.shape_params[:, :sf.num_shape_params(sid)].contiguous()
        x = rays.x.reshape(-1, 3).contiguous()
        r = rays.radius.reshape(-1).contiguous()
        P, S = x.shape[0], ps.shape[0]
        # laplace step with delta 0.02 (the benchmark softness); linear step with a wide
        # delta 0.5 so that samples fall inside its 0 < alpha < 0.9999 band
        for lap, inv, delta in [(True, True, 0.02), (False, False, 0.5)]:
            tag = f"{kind}_{int(lap)}{int(inv)}"
            a = torch.empty(P, S, device=dev)
            c = torch.empty(P, S, 3, device=dev)
            sdf = torch.empty(P, S, device=dev)
            ref.stroke_forward(a, c, sdf, torch.empty(0, device=dev), x.to(dev), r.to(dev), rays.dirs.to(dev),
                               ps.to(dev), sc.color_params.to(dev), sid, 0, delta, lap, inv)
            ga = torch.randn(P, S, generator=g)
            gc = torch.randn(P, S, 3, generator=g)
            gps = torch.zeros_like(ps, device=dev)
            gcol = torch.zeros(S, 3, device=dev)
            gx = torch.zeros(P, 3, device=dev)
            ref.stroke_backward(gps, gcol, gx, ga.to(dev), gc.to(dev), torch.empty(0, device=dev), x.to(dev),
                                r.to(dev), rays.dirs.to(dev), a, ps.to(dev), sc.color_params.to(dev), sid, 0, delta,
                                lap, inv)
            for k, v in dict(x=x, radius=r, shape=ps, color=sc.color_params, alpha=a, colors=c, sdf=sdf,
                             g_alpha=ga, g_color=gc, grad_shape=gps, grad_color=gcol, grad_x=gx).items():
                arrays[f"{tag}/{k}"] = v.detach().cpu().numpy()
            arrays[f"{tag}/sdf_id"] = np.array(sid)
            arrays[f"{tag}/delta"] = np.array(delta)
    # colour fields: gradient rgb (unit-frame positions), SH2, SH3 (view directions)
    for kind in ("sphere", "obb", "capsule", "cubic_bezier"):
        for cid, npc in ((1, 12), (2, 12), (3, 27)):
            g = torch.Generator().manual_seed(700 + 10 * cid + len(kind))
            sc = scenes.make_strokes([kind] * 9, g)
            rays = scenes.make_rays(16, 12, g)
            sid = scenes.SDF_ID[kind]
            ps = sc.shape_params[:, :sf.num_shape_params(sid)].contiguous()
            if cid == 1:
                cp = torch.cat([torch.rand(9, 6, generator=g) * 2 - 1, torch.rand(9, 6, generator=g)], -1)
            else:
                cp = torch.randn(9, npc, generator=g)
            x = rays.x.reshape(-1, 3).contiguous()
            r = rays.radius.reshape(-1).contiguous()
            vd = (rays.dirs / rays.dirs.norm(dim=-1, keepdim=True)).contiguous()
            P, S = x.shape[0], ps.shape[0]
            tag = f"{kind}_c{cid}"
            a = torch.empty(P, S, device=dev)
            c = torch.empty(P, S, 3, device=dev)
            ref.stroke_forward(a, c, torch.empty(0, device=dev), torch.empty(0, device=dev), x.to(dev), r.to(dev),
                               vd.to(dev), ps.to(dev), cp.to(dev), sid, cid, 0.02, True, True)
            ga = torch.randn(P, S, generator=g)
            gc = torch.randn(P, S, 3, generator=g)
            gps = torch.zeros_like(ps, device=dev)
            gcol = torch.zeros_like(cp, device=dev)
            gx = torch.zeros(P, 3, device=dev)
            ref.stroke_backward(gps, gcol, gx, ga.to(dev), gc.to(dev), torch.empty(0, device=dev), x.to(dev),
                                r.to(dev), vd.to(dev), a, ps.to(dev), cp.to(dev), sid, cid, 0.02, True, True)
            for k, v in dict(x=x, radius=r, viewdir=vd, shape=ps, color=cp, alpha=a, colors=c, g_alpha=ga,
                             g_color=gc, grad_shape=gps, grad_color=gcol, grad_x=gx).items():
                arrays[f"{tag}/{k}"] = v.detach().cpu().numpy()
            arrays[f"{tag}/sdf_id"] = np.array(sid)
            arrays[f"{tag}/color_id"] = np.array(cid)
    # texture coordinates (the shapes with a texcoord mapping, their per-axis-scale
    # variants, and one without)
    for kind in ("sphere", "ellipsoid", "cube", "aabb", "roundbox", "capsule", "scapsule", "line", "octahedron"):
        g = torch.Generator().manual_seed(900 + len(kind))
        sc = scenes.make_strokes([kind] * 7, g)
        rays = scenes.make_rays(12, 10, g)
        sid = scenes.SDF_ID[kind]
        ps = sc.shape_params[:, :sf.num_shape_params(sid)].contiguous()
        x = rays.x.reshape(-1, 3).contiguous()
        r = rays.radius.reshape(-1).contiguous()
        P, S = x.shape[0], ps.shape[0]
        a = torch.empty(P, S, device=dev)
        c = torch.empty(P, S, 3, device=dev)
        tex = torch.empty(P, S, 2, device=dev)
        ref.stroke_forward(a, c, torch.empty(0, device=dev), tex, x.to(dev), r.to(dev), rays.dirs.to(dev),
                           ps.to(dev), sc.color_params.to(dev), sid, 0, 0.02, True, True)
        tag = f"{kind}_tex"
        for k, v in dict(x=x, radius=r, shape=ps, color=sc.color_params, texcoord=tex).items():
            arrays[f"{tag}/{k}"] = v.detach().cpu().numpy()
        arrays[f"{tag}/sdf_id"] = np.array(sid)
    g = torch.Generator().manual_seed(99)
    P, S = 300, 37
    al = torch.rand(P, S, generator=g) ** 3
    al[torch.rand(P, S, generator=g) < 0.3] = 0
    co = torch.rand(P, S, 3, generator=g)
    dp = torch.rand(S, generator=g) * 10
    dens = torch.empty(P, device=dev)
    col = torch.empty(P, 3, device=dev)
    ref.compose_forward(dens, col, al.to(dev), co.to(dev), dp.to(dev))
    gd = torch.randn(P, generator=g)
    gcol = torch.randn(P, 3, generator=g)
    ga = torch.zeros(P, S, device=dev)
    gc = torch.zeros(P, S, 3, device=dev)
    gdp = torch.zeros(S, device=dev)
    ref.compose_backward(ga, gc, gdp, gd.to(dev), gcol.to(dev), al.to(dev), co.to(dev), dp.to(dev))
    for k, v in dict(alphas=al, colors=co, density_params=dp, density=dens, color=col, g_density=gd, g_color=gcol,
                     grad_alphas=ga, grad_colors=gc, grad_density_params=gdp).items():
        arrays[f"compose/{k}"] = v.detach().cpu().numpy()
    np.savez_compressed(os.path.join(out, "strokelib_golden.npz"), **arrays)
    print("strokelib golden written:", len(arrays), "arrays")


# (name, GridEncoder kwargs): the proposal and error networks' grids and other shapes
GRID_LAYOUTS = [
    ("proposal", dict(input_dim=3, num_levels=10, level_dim=4, base_resolution=16, desired_resolution=8192,
                      log2_hashmap_size=21, gridtype="hash", align_corners=False)),
    ("error", dict(input_dim=3, num_levels=10, level_dim=2, base_resolution=16, desired_resolution=8192,
                   log2_hashmap_size=20, gridtype="hash", align_corners=False)),
    ("default", dict()),
    ("fractional_scale", dict(input_dim=3, num_levels=12, level_dim=2, base_resolution=16,
                              desired_resolution=2048, log2_hashmap_size=17)),
    ("tiled_2d_aligned", dict(input_dim=2, num_levels=6, level_dim=8, per_level_scale=1.5, base_resolution=8,
                              log2_hashmap_size=14, gridtype="tiled", align_corners=True)),
    ("smooth_4d", dict(input_dim=4, num_levels=5, level_dim=1, base_resolution=4, log2_hashmap_size=12,
                       interpolation="smoothstep")),
]


def _load_ref_grid(ref_root):
    sys.modules["_gridencoder"] = types.ModuleType("_gridencoder")  # stub backend: never called
    path = os.path.join(ref_root, "source", "gridencoder", "grid.py")
    spec = importlib.util.spec_from_file_location("ref_grid", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_grid_layouts(ref_root, out):
    mod = _load_ref_grid(ref_root)
    res = {}
    for name, kw in GRID_LAYOUTS:
        enc = mod.GridEncoder(**kw)
        res[name] = dict(kwargs=kw, offsets=enc.offsets.tolist(), grid_sizes=enc.grid_sizes.tolist(),
                         idx_counts=torch.bincount(enc.idx, minlength=enc.num_levels).tolist(),
                         n_params=int(enc.n_params), output_dim=int(enc.output_dim),
                         per_level_scale=float(enc.per_level_scale), embeddings_shape=list(enc.embeddings.shape),
                         repr=repr(enc))
    with open(os.path.join(out, "grid_layouts.json"), "w") as f:
        json.dump(res, f, indent=1)
    print("grid layouts written:", list(res))


# (tag, D, C, L, S, H, log2 rows per level, gridtype, align_corners, interp, dtype)
GRID_CASES = [
    ("h3c4", 3, 4, 5, 1.0, 4, 10, 0, False, 0, "float32"),
    ("h3c2_smooth", 3, 2, 4, 0.6, 5, 9, 0, False, 1, "float32"),
    ("t3c1_align", 3, 1, 4, 0.5, 3, 11, 1, True, 0, "float32"),
    ("h2c8", 2, 8, 6, 0.75, 4, 8, 0, False, 0, "float32"),
    ("t2c4_smooth_align", 2, 4, 3, 1.0, 6, 12, 1, True, 1, "float32"),
    ("h3c4_f64", 3, 4, 4, 0.8, 4, 10, 0, False, 0, "float64"),
    ("h3c4_f16", 3, 4, 4, 1.0, 4, 10, 0, False, 0, "float16"),
]


def grid_case_inputs(D, C, L, S, H, log2_rows, align, dtype, seed, B=96):
    """Seeded inputs of one case: points mostly in [0, 1] with a few outside, a table
    whose levels hold min(2^log2_rows, dense size) rows (rounded up to 8), grads."""
    g = torch.Generator().manual_seed(seed)
    offsets = [0]
    for lv in range(L):
        scale = 2.0 ** (lv * S) * H - 1
        res = int(np.ceil(scale)) + 1
        dense = (res if align else res + 1) ** D
        offsets.append(offsets[-1] + int(np.ceil(min(2 ** log2_rows, dense) / 8) * 8))
    x = torch.rand(B, D, generator=g)
    x[:4] = x[:4] * 1.4 - 0.2          # some points outside [0, 1]
    x[4] = 1.0                         # the upper boundary
    x[5] = 0.0
    emb = (torch.rand(offsets[-1], C, generator=g) * 2 - 1).to(getattr(torch, dtype))
    grad = torch.randn(L, B, C, generator=g).to(getattr(torch, dtype))
    return x, emb, torch.tensor(offsets, dtype=torch.int32), grad


def make_grid(out):
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "grid", "_gridencoder*.so"))
    if not hits:
        raise SystemExit("oracle/_ref/grid/_gridencoder*.so missing: run python oracle/build_ref.py --only grid")
    loader = importlib.machinery.ExtensionFileLoader("_gridencoder", hits[0])
    spec = importlib.util.spec_from_file_location("_gridencoder", hits[0], loader=loader)
    ref = importlib.util.module_from_spec(spec)
    loader.exec_module(ref)
    dev = torch.device("cuda:0")
    arrays = {}
    for i, (tag, D, C, L, S, H, lr, gt, al, it, dt) in enumerate(GRID_CASES):
        x, emb, offs, grad = grid_case_inputs(D, C, L, S, H, lr, al, dt, 1000 + i)
        B = x.shape[0]
        xd, ed, od = x.to(dev), emb.to(dev), offs.to(dev)
        outp = torch.empty(L, B, C, device=dev, dtype=emb.dtype)
        dydx = torch.empty(B, L * D * C, device=dev, dtype=emb.dtype)
        ref.grid_encode_forward(xd, ed, od, outp, B, D, C, L, S, H, dydx, gt, al, it)
        gemb = torch.zeros_like(ed)
        gin = torch.zeros(B, D, device=dev, dtype=emb.dtype)
        ref.grid_encode_backward(grad.to(dev), xd, ed, od, gemb, B, D, C, L, S, H, dydx, gin, gt, al, it)
        tv = torch.zeros_like(ed)
        if dt != "float16":  # the reference's TV reads inputs as the table type
            ref.grad_total_variation(xd.to(emb.dtype), ed, tv, od, 1e-3, B, D, C, L, S, H, gt, al)
        torch.cuda.synchronize()
        for k, v in dict(inputs=x, embeddings=emb, offsets=offs, grad=grad, outputs=outp, dy_dx=dydx,
                         grad_embeddings=gemb, grad_inputs=gin, tv=tv).items():
            arrays[f"{tag}/{k}"] = v.detach().cpu().numpy()
        arrays[f"{tag}/meta"] = np.array([D, C, L, S, H, gt, int(al), it], dtype=np.float64)
    np.savez_compressed(os.path.join(out, "grid_golden.npz"), **arrays)
    print("grid golden written:", len(arrays), "arrays")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--layouts", action="store_true")
    ap.add_argument("--render", action="store_true")
    ap.add_argument("--cast", action="store_true")
    ap.add_argument("--strokespy", action="store_true")
    ap.add_argument("--strokelib", action="store_true")
    ap.add_argument("--compose", action="store_true")
    ap.add_argument("--stepfun", action="store_true")
    ap.add_argument("--gridlayout", action="store_true")
    ap.add_argument("--grid", action="store_true")
    ap.add_argument("--ref", default=None, help="reference checkout (default: oracle.build_ref.reference_root())")
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if a.ref is None:
        from oracle.build_ref import reference_root
        a.ref = reference_root()
    os.makedirs(a.out, exist_ok=True)
    if a.layouts:
        make_layouts(a.ref, a.out)
    if a.render:
        make_render(a.ref, a.out)
    if a.cast:
        make_cast(a.ref, a.out)
    if a.strokespy:
        make_strokes_py(a.ref, a.out)
    if a.strokelib:
        make_strokelib(a.out)
    if a.compose:
        make_compose_modes(a.ref, a.out)
    if a.stepfun:
        make_stepfun(a.ref, a.out)
    if a.gridlayout:
        make_grid_layouts(a.ref, a.out)
    if a.grid:
        make_grid(a.out)
