"""Drop-in replacement of the reference native module ``_strokelib``.

The reference binds four functions with pybind11 (source/strokelib/src/bindings.cpp:6-11)
and its Python layer imports ``_strokelib`` before falling back to a JIT build
(source/strokelib/strokes.py:7-10). This module exposes the same four functions with
the same argument order, meaning and error behaviour:

- inputs must be CUDA, contiguous, float32 (CHECK_FLOAT_INPUT, common.h:10-23),
  otherwise ``RuntimeError``;
- outputs are caller-allocated; gradient outputs are accumulated into (the reference
  Python layer passes zeroed tensors, strokes.py:212-216, 365-367);
- a numel-0 tensor means "absent" (sdf_output, grad_sdf, grad_x, grad_density,
  grad_color);
- launches go to the current torch stream, asynchronously.

Each call forwards to the C ABI of ``libn3ds.so`` (include/n3ds.h). Gradient mode:
``exact`` (default; the exact adjoint of the forward) or ``compat`` (the reference's
hand-written formulas), selected by ``set_grad_mode`` or the ``N3DS_GRAD_MODE``
environment variable.
"""
import os

import torch

from . import _lib

_MODES = {"exact": _lib.N3DS_GRAD_EXACT, "compat": _lib.N3DS_GRAD_COMPAT}
_grad_mode = _MODES[os.environ.get("N3DS_GRAD_MODE", "exact")]


def set_grad_mode(mode: str):
    """Select 'exact' or 'compat' backward formulas for this process."""
    global _grad_mode
    if mode not in _MODES:
        raise ValueError(f"grad mode must be one of {sorted(_MODES)}")
    _grad_mode = _MODES[mode]


def get_grad_mode() -> str:
    return {v: k for k, v in _MODES.items()}[_grad_mode]


def _check_float_input(t, name):
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be a contiguous tensor")
    if t.dtype != torch.float32:
        raise RuntimeError(f"{name} must be a float32 tensor")


def _need(cond, msg):
    if not cond:
        raise RuntimeError(msg)


def stroke_forward(alpha_output, color_output, sdf_output, texcoord_output, x, radius, viewdir,
                   shape_params, color_params, sdf_id, color_id, sdf_delta, use_laplace_transform,
                   inv_scale_radius):
    """strokes_forward.cu:170-225: alpha [P,S], color [P,S,3] (+ sdf [P,S])."""
    names = ["alpha_output", "color_output", "sdf_output", "texcoord_output", "x", "radius", "viewdir",
             "shape_params", "color_params"]
    ts = [alpha_output, color_output, sdf_output, texcoord_output, x, radius, viewdir, shape_params,
          color_params]
    for n, t in zip(names, ts):
        _check_float_input(t, n)
    P, S = x.size(0), shape_params.size(0)
    _need(x.dim() == 2 and x.size(1) == 3, "x must be [P, 3]")
    _need(radius.numel() >= P, "radius must hold one value per point")
    _need(alpha_output.numel() >= P * S and color_output.numel() >= P * S * 3,
          "alpha_output / color_output are too small")
    _need(sdf_output.numel() == 0 or sdf_output.numel() >= P * S, "sdf_output is too small")
    lib = _lib.load()
    with torch.cuda.device(x.device):
        ws_bytes = lib.n3ds_stroke_workspace_bytes(S)
        ws = _lib.workspace(ws_bytes, x.device)
        rc = lib.n3ds_stroke_forward(
            _lib.ptr(alpha_output), _lib.ptr(color_output), _lib.ptr(sdf_output), _lib.ptr(texcoord_output),
            texcoord_output.numel(),
            _lib.ptr(x), _lib.ptr(radius), _lib.ptr(viewdir), _lib.ptr(shape_params), _lib.ptr(color_params),
            P, viewdir.size(0), S, shape_params.size(1) if shape_params.dim() == 2 else 0,
            color_params.size(1) if color_params.dim() == 2 else 0, int(sdf_id), int(color_id),
            float(sdf_delta), int(bool(use_laplace_transform)), int(bool(inv_scale_radius)),
            _lib.ptr(ws), ws_bytes, _lib.stream_ptr())
    _lib.check(rc)


def stroke_backward(grad_shape_params, grad_color_params, grad_x, grad_alpha, grad_color, grad_sdf, x,
                    radius, viewdir, alpha, shape_params, color_params, sdf_id, color_id, sdf_delta,
                    use_laplace_transform, inv_scale_radius):
    """strokes_backward.cu:224-287: accumulates grad_shape_params, grad_color_params, grad_x."""
    names = ["grad_shape_params", "grad_color_params", "grad_x", "grad_alpha", "grad_color", "grad_sdf",
             "x", "radius", "viewdir", "shape_params", "color_params"]
    ts = [grad_shape_params, grad_color_params, grad_x, grad_alpha, grad_color, grad_sdf, x, radius, viewdir,
          shape_params, color_params]
    for n, t in zip(names, ts):
        _check_float_input(t, n)
    P, S = x.size(0), shape_params.size(0)
    _need(grad_alpha.numel() >= P * S and grad_color.numel() >= P * S * 3 and alpha.numel() >= P * S,
          "grad_alpha / grad_color / alpha are too small")
    _need(grad_x.numel() == 0 or grad_x.numel() >= P * 3, "grad_x is too small")
    _need(grad_sdf.numel() == 0 or grad_sdf.numel() >= P * S, "grad_sdf is too small")
    _need(grad_shape_params.shape == shape_params.shape and grad_color_params.shape == color_params.shape,
          "gradient buffers must match the parameter shapes")
    lib = _lib.load()
    with torch.cuda.device(x.device):
        ws_bytes = lib.n3ds_stroke_workspace_bytes(S)
        ws = _lib.workspace(ws_bytes, x.device)
        rc = lib.n3ds_stroke_backward(
            _lib.ptr(grad_shape_params), _lib.ptr(grad_color_params), _lib.ptr(grad_x), _lib.ptr(grad_alpha),
            _lib.ptr(grad_color), _lib.ptr(grad_sdf), _lib.ptr(x), _lib.ptr(radius), _lib.ptr(viewdir),
            _lib.ptr(alpha), _lib.ptr(shape_params), _lib.ptr(color_params), P, viewdir.size(0), S,
            shape_params.size(1), color_params.size(1), int(sdf_id), int(color_id), float(sdf_delta),
            int(bool(use_laplace_transform)), int(bool(inv_scale_radius)), _grad_mode, _lib.ptr(ws), ws_bytes,
            _lib.stream_ptr())
    _lib.check(rc)


def compose_forward(density_output, color_output, alphas, colors, density_params):
    """compositing.cu:159-204: 'over' compositing, last stroke on top."""
    for n, t in zip(["density_output", "color_output", "alphas", "colors", "density_params"],
                    [density_output, color_output, alphas, colors, density_params]):
        _check_float_input(t, n)
    P, S = alphas.size(0), alphas.size(1)
    C = colors.size(2)
    _need(colors.numel() == P * S * C and density_params.numel() >= S, "colors / density_params shape mismatch")
    _need(density_output.numel() >= P and color_output.numel() >= P * C, "outputs are too small")
    lib = _lib.load()
    with torch.cuda.device(alphas.device):
        rc = lib.n3ds_compose_forward(_lib.ptr(density_output), _lib.ptr(color_output), _lib.ptr(alphas),
                                      _lib.ptr(colors), _lib.ptr(density_params), P, S, C, _lib.stream_ptr())
    _lib.check(rc)


def compose_backward(grad_alphas, grad_colors, grad_density_params, grad_density_output, grad_color_output,
                     alphas, colors, density_params):
    """compositing.cu:206-262: accumulates grad_alphas, grad_colors, grad_density_params."""
    for n, t in zip(["grad_alphas", "grad_colors", "grad_density_params", "grad_density_output",
                     "grad_color_output", "alphas", "colors", "density_params"],
                    [grad_alphas, grad_colors, grad_density_params, grad_density_output, grad_color_output,
                     alphas, colors, density_params]):
        _check_float_input(t, n)
    P, S = alphas.size(0), alphas.size(1)
    C = colors.size(2)
    _need(grad_alphas.numel() >= P * S and grad_colors.numel() >= P * S * C and
          grad_density_params.numel() >= S, "gradient buffers are too small")
    _need(grad_density_output.numel() in (0, P) and grad_color_output.numel() in (0, P * C),
          "upstream gradient shape mismatch")
    lib = _lib.load()
    with torch.cuda.device(alphas.device):
        ws_bytes = lib.n3ds_compose_workspace_bytes(P, S, _grad_mode)
        ws = _lib.workspace(ws_bytes, alphas.device) if ws_bytes else None
        rc = lib.n3ds_compose_backward(
            _lib.ptr(grad_alphas), _lib.ptr(grad_colors), _lib.ptr(grad_density_params),
            _lib.ptr(grad_density_output), _lib.ptr(grad_color_output), _lib.ptr(alphas), _lib.ptr(colors),
            _lib.ptr(density_params), P, S, C, _grad_mode, _lib.ptr(ws), ws_bytes, _lib.stream_ptr())
    _lib.check(rc)
