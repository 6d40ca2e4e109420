"""The reference Python operator API of the stroke field, over the B200 backend.

Same names, arguments and behaviour as source/strokelib/strokes.py:
``get_stroke(shape_type, color_type, init_type)`` returns
(stroke_fn, dim_shape, dim_color, shape_param_ranges, color_param_ranges,
shape_sampler, color_sampler) and ``compose_strokes(alphas, colors, density_params,
composition_type)`` composites; both autograd-differentiable through the drop-in
operators of ``neural3dstrokes_b200.strokelib``.

Differences, all deliberate: the shape/colour tables are this module's own; calling
get_stroke repeatedly does not grow the range lists (the reference mutates them in
place, strokes.py:245-252); the non-'over' composition modes run on their own CUDA
kernels (torch ops in the reference).
"""
import math

import torch
from torch.autograd.function import once_differentiable

from . import _lib
from . import strokelib as _backend

_BASE = {"unit_sphere": 0, "unit_cube": 1, "unit_round_cube": 2, "unit_capped_torus": 3, "unit_capsule": 4,
         "unit_line": 5, "unit_triprism": 6, "unit_octahedron": 7, "unit_tetrahedron": 8,
         "quadratic_bezier": 9, "cubic_bezier": 10, "catmull_rom": 11}
_IMPLEMENTED_BASES = set(range(12))

_PI = math.pi


def _spline_sampler(n_points, n_radii):
    def sample(scale_min, scale_max, centre):
        s = torch.rand(1) * (scale_max - scale_min) + scale_min
        pts = [centre + (torch.rand(3) - 0.5) * s for _ in range(n_points)]
        return torch.cat(pts + [(0.2 + 0.2 * torch.rand(n_radii)) * s])
    return sample


# name -> (base, base-param ranges, base-param sampler, T, R, S1, S3)
_SHAPES = {
    "sphere": ("unit_sphere", [], None, 1, 0, 1, 0),
    "ellipsoid": ("unit_sphere", [], None, 1, 1, 0, 1),
    "aacube": ("unit_cube", [], None, 1, 0, 1, 0),
    "cube": ("unit_cube", [], None, 1, 1, 1, 0),
    "aabb": ("unit_cube", [], None, 1, 0, 0, 1),
    "obb": ("unit_cube", [], None, 1, 1, 0, 1),
    "roundcube": ("unit_round_cube", [(0, 1)], lambda *a: 0.8 * torch.rand(1), 1, 1, 1, 0),
    "roundbox": ("unit_round_cube", [(0, 1)], lambda *a: 0.8 * torch.rand(1), 1, 1, 0, 1),
    "cappedtorus": ("unit_capped_torus", [(0, _PI), (0, None)], lambda *a: torch.rand(2), 1, 1, 1, 0),
    "capsule": ("unit_capsule", [(0.25, None)], lambda *a: torch.rand(1) + 0.25, 1, 1, 1, 0),
    "scapsule": ("unit_capsule", [(0.25, None)], lambda *a: torch.rand(1) + 0.25, 1, 1, 0, 1),
    "line": ("unit_line", [(0.25, None), (-0.8, 0.8)],
             lambda *a: torch.cat([torch.rand(1) + 0.25, torch.rand(1) - 0.5]), 1, 1, 1, 0),
    "triprism": ("unit_triprism", [(0, None)], lambda *a: torch.rand(1), 1, 1, 1, 0),
    "octahedron": ("unit_octahedron", [], None, 1, 1, 1, 0),
    "tetrahedron": ("unit_tetrahedron", [], None, 1, 1, 1, 0),
    "quadratic_bezier": ("quadratic_bezier", [(-1, 1)] * 9 + [(0.001, 0.2)] * 2, _spline_sampler(3, 2),
                         0, 0, 0, 0),
    "cubic_bezier": ("cubic_bezier", [(-1, 1)] * 12 + [(0.001, 0.2)] * 2, _spline_sampler(4, 2), 0, 0, 0, 0),
    "catmull_rom": ("catmull_rom", [(-1, 1)] * 12 + [(0.001, 0.2)] * 2, _spline_sampler(4, 2), 0, 0, 0, 0),
}

# name -> (color_id, parameter ranges, sampler) (strokes.py:84-91)
_COLORS = {
    "constant_rgb": (0, [(0, 1)] * 3, lambda: torch.rand(3)),
    "gradient_rgb": (1, [(-1, 1)] * 6 + [(0, 1)] * 6, lambda: torch.cat([torch.rand(6) - 0.5, torch.rand(6)], dim=-1)),
    "constant_sh2": (2, [(None, None)] * 12, lambda: torch.randn(12)),
    "constant_sh3": (3, [(None, None)] * 27, lambda: torch.randn(27)),
}
_COLOR_DIM = 3


def make_sdf_id(base_name, t, r, s1, s3):
    """Reference sdf_id packing (strokes.py:95-106): base << 4 | T | R << 1 | S1 << 2 | S3 << 3."""
    return (_BASE[base_name] << 4) | (1 if t else 0) | (2 if r else 0) | (4 if s1 else 0) | (8 if s3 else 0)


def sdf_id_of(shape_type: str) -> int:
    """The sdf_id get_stroke binds for a shape type."""
    base, _, _, t, r, s1, s3 = _SHAPES[shape_type]
    return make_sdf_id(base, t, r, s1, s3)


def num_shape_params(shape_type: str) -> int:
    """The shape-parameter count (dim_shape) get_stroke returns for a shape type."""
    base, base_ranges, _, t, r, s1, s3 = _SHAPES[shape_type]
    return len(base_ranges) + (1 if s1 else 3 if s3 else 0) + (3 if r else 0) + (3 if t else 0)


class _StrokeFn(torch.autograd.Function):
    """alpha / colour of a batch of strokes of one sdf_id at the samples
    (reference _stroke_fn, strokes.py:109-224)."""

    @staticmethod
    def forward(ctx, x, radius, viewdir, shape_params, color_params, sdf_id, color_id, sdf_delta,
                use_laplace_transform=False, inv_scale_radius=False, no_sdf=True, return_texcoord=False):
        if x.shape[-1] != 3:
            raise ValueError("x must have shape [..., num_samples, 3]")
        if shape_params.dim() != 2 or color_params.dim() != 2 or shape_params.shape[0] != color_params.shape[0]:
            raise ValueError("shape_params / color_params must be [num_strokes, n] with equal num_strokes")
        pre = x.shape[:-1]
        x = x.contiguous().reshape(-1, 3).float()
        radius = radius.contiguous().reshape(-1).float()
        viewdir = viewdir.contiguous().reshape(-1, 3).float()
        shape_params = shape_params.contiguous().float()
        color_params = color_params.contiguous().float()
        S = shape_params.shape[0]
        alpha = torch.empty(x.shape[0], S, device=x.device)
        color = torch.empty(x.shape[0], S, _COLOR_DIM, device=x.device)
        sdf = torch.empty(0 if no_sdf else (x.shape[0], S), device=x.device)
        tex = torch.empty((x.shape[0], S, 2) if return_texcoord else 0, device=x.device)
        _backend.stroke_forward(alpha, color, sdf, tex, x, radius, viewdir, shape_params, color_params, sdf_id,
                                color_id, sdf_delta, use_laplace_transform, inv_scale_radius)
        ctx.save_for_backward(x, radius, viewdir, alpha, shape_params, color_params)
        ctx.args = (sdf_id, color_id, sdf_delta, use_laplace_transform, inv_scale_radius, pre)
        if return_texcoord:
            ctx.mark_non_differentiable(tex)
        return (alpha.reshape(*pre, S), color.reshape(*pre, S, _COLOR_DIM),
                None if no_sdf else sdf.reshape(*pre, S), tex.reshape(*pre, S, 2) if return_texcoord else None)

    @staticmethod
    @once_differentiable
    def backward(ctx, g_alpha, g_color, g_sdf=None, g_tex=None):
        x, radius, viewdir, alpha, shape_params, color_params = ctx.saved_tensors
        sdf_id, color_id, sdf_delta, lap, inv, pre = ctx.args
        S = shape_params.shape[0]
        dev = x.device
        g_alpha = torch.zeros_like(alpha) if g_alpha is None else g_alpha.contiguous().float().reshape(-1, S)
        g_color = (torch.zeros(x.shape[0], S, _COLOR_DIM, device=dev) if g_color is None
                   else g_color.contiguous().float().reshape(-1, S, _COLOR_DIM))
        g_sdf = torch.empty(0, device=dev) if g_sdf is None else g_sdf.contiguous().float().reshape(-1, S)
        gs = torch.zeros_like(shape_params)
        gc = torch.zeros_like(color_params)
        gx = torch.zeros_like(x) if ctx.needs_input_grad[0] else torch.empty(0, device=dev)
        _backend.stroke_backward(gs, gc, gx, g_alpha, g_color, g_sdf, x, radius, viewdir, alpha, shape_params,
                                 color_params, sdf_id, color_id, sdf_delta, lap, inv)
        gx = gx.reshape(*pre, 3) if ctx.needs_input_grad[0] else None
        return gx, None, None, gs, gc, None, None, None, None, None, None, None


def get_stroke(shape_type: str, color_type: str, init_type: str):
    """Stroke function and its parameter tables (reference strokes.py:227-313)."""
    if shape_type not in _SHAPES:
        raise KeyError(shape_type)
    if color_type not in _COLORS:
        raise KeyError(color_type)
    base, base_ranges, base_sampler, t, r, s1, s3 = _SHAPES[shape_type]
    if _BASE[base] not in _IMPLEMENTED_BASES:
        raise NotImplementedError(f"shape type {shape_type} is outside the implemented set")
    color_id, color_ranges, color_sampler = _COLORS[color_type]
    sdf_id = make_sdf_id(base, t, r, s1, s3)
    ranges = list(base_ranges)
    if s1:
        ranges += [(0.01, 0.5)]
    elif s3:
        ranges += [(0.01, 0.5)] * 3
    if r:
        ranges += [(-_PI, _PI)] * 3
    if t:
        ranges += [(-1.0, 1.0)] * 3

    def shape_sampler(stroke_step, error_coord=None):
        decay = math.exp(-stroke_step / 200)
        if init_type == "recon":
            lo, hi = torch.full((3,), -0.5), torch.full((3,), 0.5)
            span = float(torch.linalg.vector_norm(hi - lo))
            smin, smax = (0.02 + 0.12 * decay) * span, (0.04 + 0.18 * decay) * span
            centre = error_coord if error_coord is not None else lo + (hi - lo) * torch.rand(3)
        elif init_type == "gen_box":
            lo, hi = torch.full((3,), -0.6), torch.full((3,), 0.6)
            span = float(torch.linalg.vector_norm(hi - lo))
            centre = lo + (hi - lo) * torch.rand(3)
            dist = 1 - 2.0 * float(torch.linalg.vector_norm(centre)) / span
            smin, smax = 0.05 * span * 4 ** -dist, 0.10 * span * 4 ** -dist
        elif init_type == "gen_sphere":
            smin, smax = 0.04 + 0.06 * decay, 0.06 + 0.09 * decay
            th, ph = torch.rand(1) * 2 * _PI, torch.rand(1) * 2 * _PI
            rad = 1.0 * (1 - decay)
            centre = torch.cat([rad * torch.sin(ph) * torch.cos(th), rad * torch.sin(ph) * torch.sin(th),
                                rad * torch.cos(ph)])
        else:
            raise ValueError(init_type)
        parts = []
        if base_sampler is not None:
            parts.append(base_sampler(smin, smax, centre))
        if s1:
            parts.append(torch.rand(1) * (smax - smin) + smin)
        elif s3:
            parts.append(torch.rand(3) * (smax - smin) + smin)
        if r:
            parts.append((torch.rand(3) * 2 - 1) * _PI)
        if t:
            parts.append(centre)
        return torch.cat(parts) if parts else torch.empty(0)

    def stroke_fn(x, radius, viewdir, shape_params, color_params, *args):
        return _StrokeFn.apply(x, radius, viewdir, shape_params, color_params, sdf_id, color_id, *args)

    return stroke_fn, len(ranges), len(color_ranges), ranges, list(color_ranges), shape_sampler, color_sampler


class _ComposeFn(torch.autograd.Function):
    """'over' compositing (reference _compositing_fn, strokes.py:316-373)."""

    @staticmethod
    def forward(ctx, alphas, colors, density_params):
        if density_params.dim() != 1 or alphas.shape[:-1] != colors.shape[:-2] or \
                alphas.shape[-1] != colors.shape[-2] or alphas.shape[-1] != density_params.shape[0]:
            raise ValueError("expected alphas [..., S], colors [..., S, C], density_params [S]")
        pre = alphas.shape[:-1]
        S = density_params.shape[0]
        C = colors.shape[-1]
        a = alphas.contiguous().reshape(-1, S).float()
        c = colors.contiguous().reshape(-1, S, C).float()
        d = density_params.contiguous().float()
        dens = torch.empty(a.shape[0], device=a.device)
        col = torch.empty(a.shape[0], C, device=a.device)
        _backend.compose_forward(dens, col, a, c, d)
        ctx.save_for_backward(a, c, d)
        ctx.pre = pre
        return dens.reshape(*pre), col.reshape(*pre, C)

    @staticmethod
    @once_differentiable
    def backward(ctx, g_dens, g_col):
        a, c, d = ctx.saved_tensors
        dev = a.device
        gd = torch.zeros(0, device=dev) if g_dens is None else g_dens.contiguous().float().reshape(-1)
        gc = torch.zeros(0, device=dev) if g_col is None else g_col.contiguous().float().reshape(-1, c.shape[-1])
        ga, gcs, gdp = torch.zeros_like(a), torch.zeros_like(c), torch.zeros_like(d)
        _backend.compose_backward(ga, gcs, gdp, gd, gc, a, c, d)
        S = d.shape[0]
        return ga.reshape(*ctx.pre, S), gcs.reshape(*ctx.pre, S, c.shape[-1]), gdp


_COMPOSE_MODES = {"max": 1, "max_density_weighted": 2, "softmax": 3, "softmax_density_weighted": 4}


class _ComposeModeFn(torch.autograd.Function):
    """max / max_density_weighted / softmax / softmax_density_weighted compositing
    (reference strokes.py:390-417, torch ops there; one CUDA kernel per direction here)."""

    @staticmethod
    def forward(ctx, alphas, colors, density_params, mode):
        if density_params.dim() != 1 or alphas.shape[:-1] != colors.shape[:-2] or \
                alphas.shape[-1] != colors.shape[-2] or alphas.shape[-1] != density_params.shape[0]:
            raise ValueError("expected alphas [..., S], colors [..., S, C], density_params [S]")
        pre = alphas.shape[:-1]
        S = density_params.shape[0]
        C = colors.shape[-1]
        a = alphas.contiguous().reshape(-1, S).float()
        c = colors.contiguous().reshape(-1, S, C).float()
        d = density_params.contiguous().float()
        dens = torch.empty(a.shape[0], device=a.device)
        col = torch.empty(a.shape[0], C, device=a.device)
        lib = _lib.load()
        with torch.cuda.device(a.device):
            _lib.check(lib.n3ds_compose_mode_forward(mode, _lib.ptr(dens), _lib.ptr(col), _lib.ptr(a), _lib.ptr(c),
                                                     _lib.ptr(d), a.shape[0], S, C, _lib.stream_ptr()))
        ctx.save_for_backward(a, c, d)
        ctx.pre, ctx.mode = pre, mode
        return dens.reshape(*pre), col.reshape(*pre, C)

    @staticmethod
    @once_differentiable
    def backward(ctx, g_dens, g_col):
        a, c, d = ctx.saved_tensors
        S, C = d.shape[0], c.shape[-1]
        gd = None if g_dens is None else g_dens.contiguous().float().reshape(-1)
        gc = None if g_col is None else g_col.contiguous().float().reshape(-1, C)
        ga, gcs, gdp = torch.empty_like(a), torch.empty_like(c), torch.zeros_like(d)
        lib = _lib.load()
        with torch.cuda.device(a.device):
            _lib.check(lib.n3ds_compose_mode_backward(ctx.mode, _lib.ptr(ga), _lib.ptr(gcs), _lib.ptr(gdp),
                                                      _lib.ptr(gd), _lib.ptr(gc), _lib.ptr(a), _lib.ptr(c),
                                                      _lib.ptr(d), a.shape[0], S, C, _lib.stream_ptr()))
        return ga.reshape(*ctx.pre, S), gcs.reshape(*ctx.pre, S, C), gdp, None


def compose_strokes(alphas, colors, density_params, composition_type: str):
    """Composite strokes (reference strokes.py:376-419): 'over' through the drop-in
    _strokelib operators, the other modes through their own kernels."""
    if composition_type == "over":
        return _ComposeFn.apply(alphas, colors, density_params)
    if composition_type in _COMPOSE_MODES:
        if not alphas.is_cuda:
            raise RuntimeError("alphas must be a CUDA tensor")
        return _ComposeModeFn.apply(alphas, colors, density_params, _COMPOSE_MODES[composition_type])
    raise ValueError(f"Unknown composition type {composition_type}")
