"""The fused stroke field as a torch.autograd.Function over the C ABI.

One forward call replaces, for one scene or a batch of uneven scenes, the reference
chain StrokeField.predict_density -> stroke_fn per primitive group -> compose_strokes
('over') -> compute_alpha_weights -> volumetric_rendering (models.py:660-711, 191-235;
render.py:29-88): it returns rgb, opacity (acc) and depth per ray without any
[samples x strokes] tensor. The backward is the hand-written exact adjoint (or the
reference's formulas with ``grad_mode='compat'``) and returns gradients for the sample
positions and every stroke parameter: shape (translation, rotation, scale, base
parameters, Bezier control points and radii), colour, density and softness.
"""
import ctypes
import dataclasses
from dataclasses import dataclass
from typing import Optional, Sequence

import torch

from . import _lib


@dataclass
class FieldOptions:
    cull_alpha: float = 1e-9   # strokes whose alpha provably stays below this are skipped; 0 disables
    chunk_fwd: int = 0         # strokes per shared-memory stage (0: auto)
    chunk_bwd: int = 0
    warps: int = 0             # warps per CTA, forward: 4, 8, 16, 24, 32 (0: auto)
    warps_bwd: int = 0         # warps per CTA, backward: 4, 8, 16, 20, 24 (0: auto)
    schedule: str = "auto"     # 'segments' (auto): lane = sample; 'runs': packed (sample, stroke) pairs
    grad_mode: str = "exact"   # 'exact' or 'compat'
    forward_only: bool = False  # no backward follows: skip the bookkeeping the backward reads
    count_pairs: bool = False   # count evaluated pairs (statistics; a few % of the forward's work)
    wait_limit_us: int = 0      # limit of the device's bounded waits (0: one second)
    test_stall_staging: bool = False  # test of the wait limit only: every staging wait runs out
    rays_per_item: int = 0      # rays a warp claims at once, segment schedule: 1, 2, 4 (0: 1)

    def c(self, events=None):
        """ctypes options; ``events``: optional 4 torch.cuda.Event(enable_timing=True)
        recorded around the forward and backward segment kernels."""
        ev = None
        if events is not None:
            for e in events:
                if not e.cuda_event:  # torch creates the event on its first record
                    e.record()
            arr = (ctypes.c_void_p * 4)(*[ctypes.c_void_p(e.cuda_event) for e in events])
            ev = ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p))
            self._ev_keepalive = arr
        return _lib.Options(float(self.cull_alpha), int(self.chunk_fwd), int(self.chunk_bwd), int(self.warps),
                            {"auto": 0, "segments": 1, "runs": 2}[self.schedule],
                            _lib.N3DS_GRAD_COMPAT if self.grad_mode == "compat" else _lib.N3DS_GRAD_EXACT, ev,
                            int(self.warps_bwd), int(bool(self.forward_only)), int(bool(self.count_pairs)),
                            int(self.wait_limit_us), int(bool(self.test_stall_staging)), int(self.rays_per_item))


class _Native:
    """ctypes argument blocks for one call (kept alive for the call's duration)."""

    def __init__(self, scene_rays, scene_strokes, n_samples, x, radius, tdist, dirs, bg, bg_value, opaque,
                 sdf_ids, shape_params, color_params, density, delta, laplace, inv_scale, options, origins=None,
                 radii=None, window=None):
        n = len(scene_rays)
        self.nr = (ctypes.c_int64 * n)(*[int(v) for v in scene_rays])
        self.ns = (ctypes.c_int32 * n)(*[int(v) for v in scene_strokes])
        self.batch = _lib.Batch(n, self.nr, self.ns, int(n_samples))
        self.rays = _lib.Rays(_lib.ptr(x), _lib.ptr(radius), _lib.ptr(tdist), _lib.ptr(dirs), _lib.ptr(bg),
                              float(bg_value), int(bool(opaque)), _lib.ptr(origins), _lib.ptr(radii))
        self.strokes = _lib.Strokes(_lib.ptr(sdf_ids), _lib.ptr(shape_params), int(shape_params.shape[1]),
                                    _lib.ptr(color_params), _lib.ptr(density), _lib.ptr(delta), int(bool(laplace)),
                                    int(bool(inv_scale)), _lib.ptr(window))
        self.opt = options.c()

    def ws_bytes(self):
        return _lib.load().n3ds_field_workspace_bytes(ctypes.byref(self.batch), ctypes.byref(self.opt))


def _f32(t, name):
    if not (t.is_cuda and t.dtype == torch.float32):
        raise RuntimeError(f"{name} must be a CUDA float32 tensor")
    return t.contiguous()


class _FieldFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, radius, tdist, dirs, shape_params, color_params, density, delta, bg_t, sdf_ids,
                scene_rays, scene_strokes, bg_value, opaque, laplace, inv_scale, options, origins=None, radii=None,
                window=None):
        R, N = tdist.shape[0], tdist.shape[1] - 1
        tdist, dirs = _f32(tdist, "tdist"), _f32(dirs, "dirs")
        if x is not None:
            x, radius = _f32(x, "x"), _f32(radius, "radius")
        else:  # samples cast in-kernel from the rays
            origins, radii = _f32(origins, "origins"), _f32(radii, "radii")
        shape_params, color_params, density, delta = (
            _f32(t, n) for t, n in ((shape_params, "shape_params"), (color_params, "color_params"),
                                    (density, "density"), (delta, "sdf_delta")))
        if sdf_ids.dtype != torch.int32 or not sdf_ids.is_cuda:
            raise RuntimeError("sdf_ids must be a CUDA int32 tensor")
        sdf_ids = sdf_ids.contiguous()
        if window is not None:
            if window.dtype != torch.int32 or not window.is_cuda or window.numel() != 2 * len(scene_rays):
                raise RuntimeError("stroke_window must be a CUDA int32 tensor of (frozen, active) per scene")
            window = window.contiguous()
        bg_c = _f32(bg_t, "bg") if bg_t is not None else None
        # without any input that needs a gradient no backward can follow
        fwd_opts = options if any(ctx.needs_input_grad) else dataclasses.replace(options, forward_only=True)
        nat = _Native(scene_rays, scene_strokes, N, x, radius, tdist, dirs, bg_c, bg_value, opaque, sdf_ids,
                      shape_params, color_params, density, delta, laplace, inv_scale, fwd_opts, origins, radii,
                      window)
        lib = _lib.load()
        dev = tdist.device
        with torch.cuda.device(dev):
            ws_bytes = nat.ws_bytes()
            if ws_bytes == 0:
                raise RuntimeError("invalid batch description")
            ws = _lib.workspace(ws_bytes, dev)
            rgb = torch.empty(R, 3, device=dev)
            acc = torch.empty(R, device=dev)
            depth = torch.empty(R, device=dev)
            rc = lib.n3ds_field_forward(ctypes.byref(nat.batch), ctypes.byref(nat.rays), ctypes.byref(nat.strokes),
                                        ctypes.byref(nat.opt), _lib.ptr(rgb), _lib.ptr(acc), _lib.ptr(depth),
                                        _lib.ptr(ws), ws_bytes, _lib.stream_ptr())
        _lib.check(rc)
        ctx.save_for_backward(x, radius, tdist, dirs, shape_params, color_params, density, delta, sdf_ids, origins,
                              radii, window)
        ctx.bg = bg_c
        ctx.ws, ctx.ws_bytes = ws, ws_bytes
        ctx.meta = (scene_rays, scene_strokes, bg_value, opaque, laplace, inv_scale, options)
        return rgb, acc, depth

    @staticmethod
    def backward(ctx, g_rgb, g_acc, g_depth):
        x, radius, tdist, dirs, shape_params, color_params, density, delta, sdf_ids, origins, radii, window = \
            ctx.saved_tensors
        scene_rays, scene_strokes, bg_value, opaque, laplace, inv_scale, options = ctx.meta
        N = tdist.shape[1] - 1
        nat = _Native(scene_rays, scene_strokes, N, x, radius, tdist, dirs, ctx.bg, bg_value, opaque, sdf_ids,
                      shape_params, color_params, density, delta, laplace, inv_scale, options, origins, radii,
                      window)
        gx = torch.empty_like(x) if (x is not None and ctx.needs_input_grad[0]) else None
        gshape = torch.empty_like(shape_params)
        gcol = torch.empty_like(color_params)
        gden = torch.empty_like(density)
        gdel = torch.empty_like(delta)
        g = [t.contiguous().float() if t is not None else None for t in (g_rgb, g_acc, g_depth)]
        lib = _lib.load()
        with torch.cuda.device(tdist.device):
            rc = lib.n3ds_field_backward(ctypes.byref(nat.batch), ctypes.byref(nat.rays), ctypes.byref(nat.strokes),
                                         ctypes.byref(nat.opt), _lib.ptr(g[0]), _lib.ptr(g[1]), _lib.ptr(g[2]),
                                         _lib.ptr(gx), _lib.ptr(gshape), _lib.ptr(gcol), _lib.ptr(gden),
                                         _lib.ptr(gdel), _lib.ptr(ctx.ws), ctx.ws_bytes, _lib.stream_ptr())
        _lib.check(rc)
        return (gx, None, None, None, gshape, gcol, gden, gdel, None, None, None, None, None, None, None, None,
                None, None, None, None)


def render_strokes(x: torch.Tensor, radius: torch.Tensor, tdist: torch.Tensor, dirs: torch.Tensor,
                   shape_params: torch.Tensor, sdf_ids: torch.Tensor, color_params: torch.Tensor,
                   density: torch.Tensor, sdf_delta, use_laplace_transform: bool = True,
                   inv_scale_radius: bool = True, bg=1.0, opaque_background: bool = False,
                   options: Optional[FieldOptions] = None, scene_sizes: Optional[Sequence] = None,
                   stroke_window: Optional[torch.Tensor] = None):
    """Render rays through a stroke field.

    x [R,N,3] sample positions, radius [R,N], tdist [R,N+1], dirs [R,3];
    shape_params [S,P] in the reference layout (zero-padded rows), sdf_ids int32 [S],
    color_params [S,3], density [S] (already multiplied by density_scale), sdf_delta a
    float, a 0-d tensor or a per-stroke [S] tensor. ``scene_sizes``: list of
    (n_rays, n_strokes) for a batch of scenes concatenated along rays and strokes
    (default: one scene). bg: float or [R,3] tensor. ``stroke_window``: optional CUDA
    int32 [n_scenes, 2] of (frozen, active) per scene, read on the device: strokes at
    or beyond ``active`` are absent, strokes below ``frozen`` are composited but get
    no gradient and pass none to ``x`` (the truncation of
    StrokeField.predict_density, models.py:665-702, without a host read of the count).
    Returns rgb [R,3], acc [R], depth [R].
    """
    S = int(sdf_ids.numel())
    R = int(x.shape[0])
    dev = x.device
    if torch.is_tensor(sdf_delta):
        delta = sdf_delta.to(dev, torch.float32)
        if delta.dim() == 0:
            delta = delta.expand(S)
    else:
        delta = torch.full((S,), float(sdf_delta), device=dev)
    if scene_sizes is None:
        scene_sizes = [(R, S)]
    scene_rays = [int(a) for a, _ in scene_sizes]
    scene_strokes = [int(b) for _, b in scene_sizes]
    if sum(scene_rays) != R or sum(scene_strokes) != S:
        raise ValueError("scene_sizes do not add up to the ray / stroke counts")
    if x.dim() != 3 or x.shape[2] != 3 or radius.shape != x.shape[:2] or tdist.shape != (R, x.shape[1] + 1) \
            or dirs.shape != (R, 3):
        raise ValueError("expected x [R,N,3], radius [R,N], tdist [R,N+1], dirs [R,3]")
    if shape_params.dim() != 2 or shape_params.shape[0] != S or color_params.shape != (S, 3) or \
            density.shape != (S,):
        raise ValueError("expected shape_params [S,P], color_params [S,3], density [S]")
    bg_t, bg_value = (bg, 0.0) if torch.is_tensor(bg) else (None, float(bg))
    opts = options or FieldOptions()
    return _FieldFn.apply(x, radius, tdist, dirs, shape_params, color_params, density, delta, bg_t, sdf_ids,
                          scene_rays, scene_strokes, bg_value, opaque_background, use_laplace_transform,
                          inv_scale_radius, opts, None, None, stroke_window)


def render_rays(origins: torch.Tensor, directions: torch.Tensor, radii: torch.Tensor, tdist: torch.Tensor,
                shape_params: torch.Tensor, sdf_ids: torch.Tensor, color_params: torch.Tensor, density: torch.Tensor,
                sdf_delta, use_laplace_transform: bool = True, inv_scale_radius: bool = True, bg=1.0,
                opaque_background: bool = False, options: Optional[FieldOptions] = None,
                scene_sizes: Optional[Sequence] = None):
    """render_strokes with the samples cast in the kernels from the rays, as
    cast_rays does (render.py:5-26): x = directions * t + origins, radius = radii * t,
    t the interval midpoints of tdist. origins / directions [R,3], radii [R] or [R,1],
    tdist [R,N+1]. Gradients flow to the stroke parameters and sdf_delta (the rays are
    data in the reference's training step, models.py:183-191)."""
    R = int(tdist.shape[0])
    S = int(sdf_ids.numel())
    dev = tdist.device
    if origins.shape != (R, 3) or directions.shape != (R, 3) or radii.numel() != R or tdist.dim() != 2:
        raise ValueError("expected origins / directions [R,3], radii [R], tdist [R,N+1]")
    if torch.is_tensor(sdf_delta):
        delta = sdf_delta.to(dev, torch.float32)
        if delta.dim() == 0:
            delta = delta.expand(S)
    else:
        delta = torch.full((S,), float(sdf_delta), device=dev)
    if scene_sizes is None:
        scene_sizes = [(R, S)]
    scene_rays = [int(a) for a, _ in scene_sizes]
    scene_strokes = [int(b) for _, b in scene_sizes]
    if sum(scene_rays) != R or sum(scene_strokes) != S:
        raise ValueError("scene_sizes do not add up to the ray / stroke counts")
    bg_t, bg_value = (bg, 0.0) if torch.is_tensor(bg) else (None, float(bg))
    return _FieldFn.apply(None, None, tdist, directions, shape_params, color_params, density, delta, bg_t, sdf_ids,
                          scene_rays, scene_strokes, bg_value, opaque_background, use_laplace_transform,
                          inv_scale_radius, options or FieldOptions(), origins, radii.reshape(R))


def field_status(workspace):
    """(status, evaluated pairs) of the last forward that used ``workspace`` (synchronises)."""
    st = ctypes.c_int32(0)
    pairs = ctypes.c_uint64(0)
    _lib.check(_lib.load().n3ds_field_read_status(_lib.ptr(workspace), ctypes.byref(st), ctypes.byref(pairs),
                                                  _lib.stream_ptr()))
    return int(st.value), int(pairs.value)
