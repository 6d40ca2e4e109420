"""Torch restatement of the reference's multi-resolution grid encoder
(source/gridencoder/src/gridencoder.cu, source/gridencoder/grid.py), TEST
INFRASTRUCTURE ONLY: imported by tests, never by the product package.

Cell selection follows the kernel's float32 steps exactly, so that the oracle and
the CUDA code pick the same corners:
  scale      = fma(exp2(level * S), H, -1)                  (gridencoder.cu:127)
  resolution = ceil(scale) + 1                              (gridencoder.cu:128)
  pos        = fma(x, scale, align_corners ? 0 : 0.5)       (gridencoder.cu:137)
  cell       = floor(pos), frac = pos - cell                (gridencoder.cu:138-139)
Corner indices use the kernel's uint32 arithmetic (wrapping multiplies, the
early-exit stride loop and the coherent prime hash, gridencoder.cu:48-82), done in
int64 with masks. Everything after the fractions (smoothstep, corner weights, the
sums) runs in float64, so the oracle is the exact value of the interpolant at the
kernel's cells.

Layouts are the reference's: inputs [B, D] in [0, 1]; embeddings [sO, C];
offsets [L + 1] int32; outputs [L, B, C]; dy_dx [B, L * D * C] ordered (l, d, c);
grad [L, B, C].
"""
import math

import numpy as np
import torch

M32 = 0xFFFFFFFF
PRIMES = (1, 2654435761, 805459861, 3674653429, 2097192037, 1434869437, 2165219737)


def _f32(v):
    return np.float32(v)


def level_constants(level, S, H):
    """(scale, resolution) of one level with float32 rounding (gridencoder.cu:127-128)."""
    e = np.float32(2.0 ** float(np.float32(np.float32(level) * np.float32(S))))
    scale = np.float32(float(e) * float(H) - 1.0)          # one rounding: fma
    return scale, int(math.ceil(float(scale))) + 1


def level_offsets(input_dim=3, num_levels=16, level_dim=2, per_level_scale=2, base_resolution=16,
                  log2_hashmap_size=19, desired_resolution=None, align_corners=False):
    """Parameter layout of GridEncoder.__init__ (grid.py:98-130): returns
    (offsets int32 [L + 1], resolutions [L], per_level_scale)."""
    if desired_resolution is not None:
        per_level_scale = np.exp2(np.log2(desired_resolution / base_resolution) / (num_levels - 1))
    max_params = 2 ** log2_hashmap_size
    offsets, resolutions, offset = [], [], 0
    for i in range(num_levels):
        res = int(np.ceil(base_resolution * per_level_scale ** i))
        res = res if align_corners else res + 1
        n = min(max_params, res ** input_dim)
        n = int(np.ceil(n / 8) * 8)
        resolutions.append(res)
        offsets.append(offset)
        offset += n
    offsets.append(offset)
    return np.array(offsets, dtype=np.int32), resolutions, per_level_scale


def grid_index(cells, gridtype, align_corners, hashmap_size, resolution):
    """Row of the embedding table for integer cells [..., D] (get_grid_index,
    gridencoder.cu:65-82), uint32 arithmetic in int64."""
    D = cells.shape[-1]
    stride = 1
    index = torch.zeros(cells.shape[:-1], dtype=torch.int64, device=cells.device)
    mult = resolution if align_corners else resolution + 1
    for d in range(D):
        if stride > hashmap_size:
            break
        index = (index + cells[..., d] * stride) & M32
        stride = (stride * mult) & M32
    if gridtype == 0 and stride > hashmap_size:
        h = torch.zeros_like(index)
        for d in range(D):
            h = h ^ ((cells[..., d] * PRIMES[d]) & M32)
        index = h
    return index % hashmap_size


def _positions(inputs, scale, align_corners):
    """float32 fma(x, scale, off), its floor and fraction (exact float32 emulation:
    the float64 product of two float32 values plus 0.5 is exact)."""
    x = inputs.to(torch.float64)
    off = 0.0 if align_corners else 0.5
    pos = (x * float(scale) + off).to(torch.float32).to(torch.float64)
    cell = torch.floor(pos)
    return cell.to(torch.int64), pos - cell


def _in_range(inputs):
    return ((inputs >= 0) & (inputs <= 1)).all(-1)


def grid_encode_forward(inputs, embeddings, offsets, S, H, calc_dy_dx=False, gridtype=0, align_corners=False,
                        interp=0):
    """kernel_grid (gridencoder.cu:86-244): returns (outputs [L, B, C] float64,
    dy_dx [B, L*D*C] float64 or None)."""
    B, D = inputs.shape
    C = embeddings.shape[1]
    offs = [int(o) for o in offsets]
    L = len(offs) - 1
    emb = embeddings.to(torch.float64)
    ok = _in_range(inputs)
    out = torch.zeros(L, B, C, dtype=torch.float64)
    dydx = torch.zeros(B, L, D, C, dtype=torch.float64) if calc_dy_dx else None
    for lv in range(L):
        hsize = offs[lv + 1] - offs[lv]
        scale, res = level_constants(lv, S, H)
        table = emb[offs[lv]:offs[lv + 1]]
        cell, frac = _positions(inputs, scale, align_corners)
        if interp == 1:
            deriv = 6 * frac * (1 - frac)
            frac = frac * frac * (3 - 2 * frac)
        else:
            deriv = torch.ones_like(frac)
        for corner in range(1 << D):
            w = torch.ones(B, dtype=torch.float64)
            cc = cell.clone()
            for d in range(D):
                if corner >> d & 1:
                    w = w * frac[:, d]
                    cc[:, d] += 1
                else:
                    w = w * (1 - frac[:, d])
            idx = grid_index(cc, gridtype, align_corners, hsize, res)
            out[lv] += w[:, None] * table[idx]
        if calc_dy_dx:
            for gd in range(D):
                acc = torch.zeros(B, C, dtype=torch.float64)
                others = [d for d in range(D) if d != gd]
                for corner in range(1 << (D - 1)):
                    w = torch.full((B,), float(scale), dtype=torch.float64)
                    cc = cell.clone()
                    for k, d in enumerate(others):
                        if corner >> k & 1:
                            w = w * frac[:, d]
                            cc[:, d] += 1
                        else:
                            w = w * (1 - frac[:, d])
                    left = table[grid_index(cc, gridtype, align_corners, hsize, res)]
                    cc[:, gd] += 1
                    right = table[grid_index(cc, gridtype, align_corners, hsize, res)]
                    acc += (w * deriv[:, gd])[:, None] * (right - left)
                dydx[:, lv, gd] = acc
    out[:, ~ok] = 0
    if calc_dy_dx:
        dydx[~ok] = 0
        dydx = dydx.reshape(B, L * D * C)
    return out, dydx


def grid_encode_backward(grad, inputs, embeddings, offsets, S, H, dy_dx=None, gridtype=0, align_corners=False,
                         interp=0):
    """kernel_grid_backward + kernel_input_backward (gridencoder.cu:247-365):
    returns (grad_embeddings [sO, C] float64, grad_inputs [B, D] float64 or None).
    Out-of-range points contribute nothing to the table gradient."""
    B, D = inputs.shape
    C = embeddings.shape[1]
    offs = [int(o) for o in offsets]
    L = len(offs) - 1
    g = grad.to(torch.float64)
    ok = _in_range(inputs)
    gemb = torch.zeros(embeddings.shape, dtype=torch.float64)
    for lv in range(L):
        hsize = offs[lv + 1] - offs[lv]
        scale, res = level_constants(lv, S, H)
        cell, frac = _positions(inputs, scale, align_corners)
        if interp == 1:
            frac = frac * frac * (3 - 2 * frac)
        for corner in range(1 << D):
            w = torch.ones(B, dtype=torch.float64)
            cc = cell.clone()
            for d in range(D):
                if corner >> d & 1:
                    w = w * frac[:, d]
                    cc[:, d] += 1
                else:
                    w = w * (1 - frac[:, d])
            idx = grid_index(cc, gridtype, align_corners, hsize, res)
            contrib = (w[:, None] * g[lv]) * ok[:, None]
            gemb.index_add_(0, idx[ok] + offs[lv], contrib[ok])
    gin = None
    if dy_dx is not None:
        dd = dy_dx.to(torch.float64).reshape(B, L, D, C)
        gin = torch.einsum("lbc,bldc->bd", g, dd)
    return gemb, gin


def grad_total_variation(inputs, embeddings, grad, offsets, weight, S, H, gridtype=0, align_corners=False):
    """kernel_grad_tv (gridencoder.cu:453-559): adds to ``grad`` (in place, float64
    copy returned) w * sum_n(e - e_n) / sqrt(sum_n (e - e_n)^2 + 1e-9) at the cell of
    each in-range point, w = weight / (2 D), over the face neighbours inside
    [0, resolution]."""
    B, D = inputs.shape
    offs = [int(o) for o in offsets]
    L = len(offs) - 1
    emb = embeddings.to(torch.float64)
    out = grad.to(torch.float64).clone()
    ok = _in_range(inputs)
    w = float(np.float32(weight)) / (2 * D)
    for lv in range(L):
        hsize = offs[lv + 1] - offs[lv]
        scale, res = level_constants(lv, S, H)
        cell, _ = _positions(inputs.to(torch.float32), scale, align_corners)
        table = emb[offs[lv]:offs[lv + 1]]
        idx = grid_index(cell, gridtype, align_corners, hsize, res)
        e = table[idx]
        s = torch.zeros_like(e)
        sq = torch.zeros_like(e)
        for d in range(D):
            for step, keep in ((1, cell[:, d] < res), (-1, cell[:, d] > 0)):
                nb = cell.clone()
                nb[:, d] += step
                diff = (e - table[grid_index(nb, gridtype, align_corners, hsize, res)]) * keep[:, None]
                s += diff
                sq += diff * diff
        val = w * s / torch.sqrt(sq + 1e-9)
        out.index_add_(0, idx[ok] + offs[lv], val[ok])
    return out
