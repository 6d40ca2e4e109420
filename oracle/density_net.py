"""Float64 restatement of the proposal / error fields' density network, TEST
INFRASTRUCTURE ONLY: imported by tests, never by the product package.

It follows source/models.py:
  _warp_coords (:19-33) and coord.contract (source/utils/coord.py:5-11) in float32,
  with the rounding torch's CUDA ops give (a division by a Python scalar is a
  multiplication by its float32 reciprocal; the sum of three squares reduced as
  (x0^2 + x2^2) + x1^2; correctly rounded sqrt and division; no fused multiply-adds),
  the order measured on torch 2.11's CUDA kernels (tests/test_density_net_gpu.py
  checks it against them);
  GridEncoder.forward's (x + bound) / (2 bound) (source/gridencoder/grid.py:158-160)
  in float32;
  the grid encoding in float64 at the kernel's float32 cells (oracle.gridencoder);
  density_layer (:342-346) Linear(L*C, 64), ReLU, Linear(64, 1) and
  softplus(raw + density_bias) (:430-431) in float64.
The backward is float64 autograd through the layers and oracle.gridencoder's table
adjoint for the features.
"""
import numpy as np
import torch
import torch.nn.functional as F

from . import gridencoder as og

WARP_SCALE, WARP_CONTRACT, WARP_NONE = 0, 1, 2


def _r32(t):
    return t.to(torch.float32)


def warp_to_unit(coords, warp, bbox_size=2.0, bound=1.0):
    """(warped coordinates, grid inputs in [0, 1]) as float32 [B, 3], each step rounded
    as torch's CUDA ops round it: float64 arithmetic rounded to float32 after every
    operation (exact emulation of one correctly rounded float32 operation), the sum of
    squares in the order torch's CUDA reduction uses for three values, (x0^2 + x2^2) +
    x1^2, and a division by a Python scalar as a multiplication by its float32
    reciprocal."""
    x = coords.detach().to(torch.float32).cpu().reshape(-1, 3)
    d = x.to(torch.float64)
    if warp == WARP_SCALE:
        r = float(np.float32(1.0) / np.float32(bbox_size / 2))
        w = _r32(d * r)
    elif warp == WARP_CONTRACT:
        eps = float(torch.finfo(torch.float32).eps)
        sq = [_r32(d[:, i] * d[:, i]).double() for i in range(3)]
        m = _r32(_r32(sq[0] + sq[2]).double() + sq[1]).double().clamp_min(eps)[:, None]
        s = _r32(torch.sqrt(m)).double()
        k = _r32(_r32(2 * s - 1).double() / m).double()
        w = _r32(torch.where(m <= 1, d, _r32(k * d).double()) * 0.5)
    else:
        w = x.clone()
    inv = float(np.float32(1.0) / np.float32(2 * bound))
    u = _r32(_r32(w.double() + float(np.float32(bound))).double() * inv)
    return w, u


def features(u, table, offsets, S, H, gridtype=0, align_corners=False):
    """[B, L * C] float64, level-major as GridEncoder.forward returns them."""
    out, _ = og.grid_encode_forward(u, table.detach().cpu(), offsets.cpu(), S, H, gridtype=gridtype,
                                    align_corners=align_corners)
    L, B, C = out.shape
    return out.permute(1, 0, 2).reshape(B, L * C)


def _layers(feat, w1, b1, w2, b2, density_bias, raw_output):
    pre = feat @ w1.T + b1
    h = torch.relu(pre)
    raw = (h @ w2.reshape(1, -1).T).reshape(-1) + b2.reshape(())
    return raw if raw_output else F.softplus(raw + density_bias)


def forward(coords, table, offsets, S, H, w1, b1, w2, b2, density_bias=-1.0, warp=WARP_SCALE, bbox_size=2.0,
            bound=1.0, raw_output=False, gridtype=0, align_corners=False):
    """(density [B] float64, warped coords [B, 3] float32, features [B, L*C] float64)."""
    w, u = warp_to_unit(coords, warp, bbox_size, bound)
    feat = features(u, table, offsets, S, H, gridtype, align_corners)
    d = lambda t: t.detach().cpu().to(torch.float64)
    with torch.no_grad():
        dens = _layers(feat, d(w1), d(b1), d(w2), d(b2), density_bias, raw_output)
    return dens, w, feat


def backward(grad_density, coords, table, offsets, S, H, w1, b1, w2, b2, density_bias=-1.0, warp=WARP_SCALE,
             bbox_size=2.0, bound=1.0, raw_output=False, gridtype=0, align_corners=False):
    """Gradients (table, w1, b1, w2, b2) in float64 for upstream grad_density [B]."""
    _, u = warp_to_unit(coords, warp, bbox_size, bound)
    feat = features(u, table, offsets, S, H, gridtype, align_corners).requires_grad_(True)
    params = [t.detach().cpu().to(torch.float64).requires_grad_(True) for t in (w1, b1, w2, b2)]
    with torch.enable_grad():
        dens = _layers(feat, *params, density_bias, raw_output)
        grads = torch.autograd.grad(dens, [feat] + params, grad_density.detach().cpu().to(torch.float64))
    dfeat = grads[0]
    L = len(offsets) - 1
    C = table.shape[1]
    gtab, _ = og.grid_encode_backward(dfeat.reshape(-1, L, C).permute(1, 0, 2), u, table.detach().cpu(),
                                      offsets.cpu(), S, H, gridtype=gridtype, align_corners=align_corners)
    return (gtab,) + tuple(grads[1:])


def level_mean_sq(table, offsets, all_channels=False):
    """models.py:472-488 in float64: [L, C] means of squares per level (channel 0
    only, others 0, for the scatter_reduce_ fallback)."""
    t = table.detach().cpu().to(torch.float64)
    offs = [int(o) for o in offsets]
    L, C = len(offs) - 1, t.shape[1]
    out = torch.zeros(L, C, dtype=torch.float64)
    for lv in range(L):
        rows = t[offs[lv]:offs[lv + 1]]
        m = (rows * rows).mean(0)
        out[lv] = m if all_channels else torch.cat([m[:1], torch.zeros(C - 1, dtype=torch.float64)])
    return out
