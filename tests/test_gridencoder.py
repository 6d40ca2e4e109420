"""Grid encoder on the CPU: the oracle (oracle/gridencoder.py) and the host-side
parameter layout (neural3dstrokes_b200.gridencoder.GridEncoder) against what the
reference produced (tests/golden/grid_layouts.json from source/gridencoder/grid.py;
tests/golden/grid_golden.npz from its CUDA kernels), plus known answers:

- a tiled grid whose rows hold their own cell coordinates interpolates to the
  continuous position x * scale + 1/2 (multilinear interpolation of a linear field
  is exact), with dy/dx = scale;
- the uint32 index arithmetic against Python integers;
- the table gradient is the adjoint of the (table-linear) forward, dy_dx matches
  float64 central differences, and a constant table has zero total variation.
"""
import json
import os

import numpy as np
import pytest
import torch

from neural3dstrokes_b200.gridencoder import GridEncoder
from oracle import gridencoder as og

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def layouts():
    with open(os.path.join(GOLDEN, "grid_layouts.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name", list(layouts()))
def test_layout_matches_reference(name):
    ref = layouts()[name]
    enc = GridEncoder(**ref["kwargs"])
    assert enc.offsets.tolist() == ref["offsets"]
    assert enc.grid_sizes.tolist() == ref["grid_sizes"]
    assert torch.bincount(enc.idx, minlength=enc.num_levels).tolist() == ref["idx_counts"]
    assert int(enc.n_params) == ref["n_params"] and enc.output_dim == ref["output_dim"]
    assert list(enc.embeddings.shape) == ref["embeddings_shape"]
    assert repr(enc) == ref["repr"]
    assert abs(float(enc.per_level_scale) - ref["per_level_scale"]) == 0
    kw = {k: v for k, v in ref["kwargs"].items() if k not in ("gridtype", "interpolation")}
    offs, res, _ = og.level_offsets(**kw)
    assert offs.tolist() == ref["offsets"] and res == ref["grid_sizes"]


def test_embeddings_init_range():
    torch.manual_seed(0)
    enc = GridEncoder(num_levels=3, level_dim=2, log2_hashmap_size=10, init_std=1e-3)
    e = enc.embeddings.detach()
    assert e.abs().max() <= 1e-3 and e.abs().max() > 5e-4


def _linear_table(D, L, S, H, align):
    """Tiled table whose row at cell c holds c (first D channels of C = 4 or 8)."""
    C = 4 if D <= 4 else 8
    offsets, tables = [0], []
    for lv in range(L):
        scale, res = og.level_constants(lv, S, H)
        n = res if align else res + 1
        cells = torch.stack(torch.meshgrid(*[torch.arange(n)] * D, indexing="ij"), -1).reshape(-1, D)
        row = og.grid_index(cells, 1, align, n ** D, res)
        t = torch.zeros(n ** D, C, dtype=torch.float64)
        t[row, :D] = cells.double()
        pad = (-t.shape[0]) % 8
        tables.append(torch.cat([t, torch.zeros(pad, C, dtype=torch.float64)]))
        offsets.append(offsets[-1] + tables[-1].shape[0])
    return torch.cat(tables), torch.tensor(offsets, dtype=torch.int32), C


@pytest.mark.parametrize("D,align", [(2, False), (3, True), (3, False), (4, False)])
def test_tiled_linear_field_is_reproduced(D, align):
    L, S, H = 3, 0.5, 3
    table, offsets, C = _linear_table(D, L, S, H, align)
    g = torch.Generator().manual_seed(D)
    x = torch.rand(200, D, generator=g)
    out, dydx = og.grid_encode_forward(x, table, offsets, S, H, calc_dy_dx=True, gridtype=1,
                                       align_corners=align)
    dydx = dydx.reshape(200, L, D, C)
    for lv in range(L):
        scale, _ = og.level_constants(lv, S, H)
        pos = (x.double() * float(scale) + (0.0 if align else 0.5)).float().double()
        assert torch.allclose(out[lv, :, :D], pos, atol=1e-9)
        assert torch.allclose(dydx[:, lv, :, :D], float(scale) * torch.eye(D, dtype=torch.float64).expand(200, D, D),
                              atol=1e-9)


def test_out_of_range_points_give_zero():
    table, offsets, C = _linear_table(3, 2, 1.0, 4, False)
    x = torch.tensor([[-0.01, 0.5, 0.5], [0.5, 1.01, 0.5], [0.2, 0.3, 0.4]])
    out, dydx = og.grid_encode_forward(x, table + 1, offsets, 1.0, 4, calc_dy_dx=True, gridtype=1)
    assert (out[:, :2] == 0).all() and (dydx[:2] == 0).all() and (out[:, 2] != 0).all()
    gemb, _ = og.grid_encode_backward(torch.ones(2, 2, C), x[:2], table, offsets, 1.0, 4, gridtype=1)
    assert (gemb == 0).all()


def test_index_arithmetic_matches_python_integers():
    rng = np.random.default_rng(3)
    for D in (2, 3, 5):
        cells = rng.integers(0, 9000, size=(300, D))
        for hsize, res, gridtype, align in [(2 ** 19, 8191, 0, False), (4096, 20, 0, True), (1000, 200, 1, False),
                                            (2 ** 21, 40, 0, False)]:
            got = og.grid_index(torch.from_numpy(cells), gridtype, align, hsize, res).numpy()
            mult = res if align else res + 1
            for c, v in zip(cells.tolist(), got.tolist()):
                stride, index = 1, 0
                for d in range(D):
                    if stride > hsize:
                        break
                    index = (index + c[d] * stride) % 2 ** 32
                    stride = (stride * mult) % 2 ** 32
                if gridtype == 0 and stride > hsize:
                    index = 0
                    for d in range(D):
                        index ^= (c[d] * og.PRIMES[d]) % 2 ** 32
                assert v == index % hsize


def _case(D=3, C=4, L=4, S=0.7, H=5, log2_rows=9, gridtype=0, align=False, B=64, seed=0):
    g = torch.Generator().manual_seed(seed)
    offsets = [0]
    for lv in range(L):
        _, res = og.level_constants(lv, S, H)
        dense = (res if align else res + 1) ** D
        offsets.append(offsets[-1] + int(np.ceil(min(2 ** log2_rows, dense) / 8) * 8))
    x = torch.rand(B, D, generator=g) * 0.98 + 0.01
    table = torch.rand(offsets[-1], C, generator=g, dtype=torch.float64) * 2 - 1
    return x, table, torch.tensor(offsets, dtype=torch.int32)


@pytest.mark.parametrize("interp", [0, 1])
@pytest.mark.parametrize("gridtype,align", [(0, False), (1, True)])
def test_table_gradient_is_the_adjoint(interp, gridtype, align):
    x, table, offsets = _case(gridtype=gridtype, align=align)
    t = table.clone().requires_grad_(True)
    out, _ = og.grid_encode_forward(x, t, offsets, 0.7, 5, gridtype=gridtype, align_corners=align, interp=interp)
    grad = torch.randn(out.shape, generator=torch.Generator().manual_seed(1), dtype=torch.float64)
    (out * grad).sum().backward()
    gemb, _ = og.grid_encode_backward(grad, x, table, offsets, 0.7, 5, gridtype=gridtype, align_corners=align,
                                      interp=interp)
    assert torch.allclose(gemb, t.grad, rtol=0, atol=1e-12)


@pytest.mark.parametrize("interp", [0, 1])
def test_dy_dx_matches_central_differences(interp):
    x, table, offsets = _case(L=3, S=0.5, H=3, log2_rows=12)
    out, dydx = og.grid_encode_forward(x, table, offsets, 0.5, 3, calc_dy_dx=True, interp=interp)
    dydx = dydx.reshape(x.shape[0], 3, 3, 4)
    h = 1e-4
    for d in range(3):
        e = torch.zeros(3)
        e[d] = h
        op, _ = og.grid_encode_forward(x + e, table, offsets, 0.5, 3, interp=interp)
        om, _ = og.grid_encode_forward(x - e, table, offsets, 0.5, 3, interp=interp)
        fd = ((op - om) / (2 * h)).permute(1, 0, 2)      # [B, L, C]
        # points whose +-h step crosses a cell face (float32 positions) are skipped
        same = torch.ones(x.shape[0], dtype=torch.bool)
        for lv in range(3):
            scale, _ = og.level_constants(lv, 0.5, 3)
            cp, _ = og._positions(x + e, scale, False)
            cm, _ = og._positions(x - e, scale, False)
            same &= (cp == cm).all(-1)
        assert same.sum() > x.shape[0] // 2
        err = (fd[same] - dydx[same, :, d]).abs().max() / dydx[same, :, d].abs().max()
        assert err < 2e-3, err          # float32 positions limit the difference quotient


def test_total_variation_of_constant_table_is_zero():
    x, table, offsets = _case(gridtype=1, align=False, log2_rows=14)
    const = torch.full_like(table, 0.3)
    out = og.grad_total_variation(x, const, torch.zeros_like(const), offsets, 1.0, 0.7, 5, gridtype=1)
    assert (out == 0).all()
    out = og.grad_total_variation(x, table, torch.zeros_like(table), offsets, 1.0, 0.7, 5, gridtype=1)
    assert out.abs().max() > 0


def golden_cases():
    path = os.path.join(GOLDEN, "grid_golden.npz")
    if not os.path.exists(path):
        return None, []
    z = np.load(path)
    return z, sorted({k.split("/")[0] for k in z.files})


@pytest.mark.parametrize("tag", golden_cases()[1])
def test_oracle_matches_reference_kernels(tag):
    """The oracle against the reference's own CUDA kernels (outputs recorded on a B200)."""
    z, _ = golden_cases()
    D, C, L, S, H, gt, al, it = z[f"{tag}/meta"].tolist()
    D, C, L, H, gt, al, it = int(D), int(C), int(L), int(H), int(gt), bool(al), int(it)
    x = torch.from_numpy(z[f"{tag}/inputs"])
    emb = torch.from_numpy(z[f"{tag}/embeddings"])
    offs = torch.from_numpy(z[f"{tag}/offsets"])
    grad = torch.from_numpy(z[f"{tag}/grad"])
    half = emb.dtype == torch.float16
    # 1e-5: at levels with a fractional exponent the kernels take the scale from
    # CUDA's exp2f (within 2 ulp of 2^x) and the oracle from the rounded power, which
    # moves positions by about 1e-6 relative; the float16 kernel rounds every partial
    # sum to half (4e-3 forward, 2e-2 for its atomically accumulated gradients)
    tol, gtol = (4e-3, 2e-2) if half else (1e-5, 1e-5)
    out, dydx = og.grid_encode_forward(x, emb, offs, S, H, calc_dy_dx=True, gridtype=gt, align_corners=al, interp=it)
    assert rel(out, z[f"{tag}/outputs"]) < tol
    assert rel(dydx, z[f"{tag}/dy_dx"]) < tol
    gemb, gin = og.grid_encode_backward(grad, x, emb, offs, S, H, torch.from_numpy(z[f"{tag}/dy_dx"]), gridtype=gt,
                                        align_corners=al, interp=it)
    assert rel(gemb, z[f"{tag}/grad_embeddings"]) < gtol
    assert rel(gin, z[f"{tag}/grad_inputs"]) < gtol
    if not half:
        tv = og.grad_total_variation(x.to(emb.dtype), emb, torch.zeros_like(emb), offs, 1e-3, S, H, gridtype=gt,
                                     align_corners=al)
        assert rel(tv, z[f"{tag}/tv"]) < tol


def rel(a, b):
    a = torch.as_tensor(a).double()
    b = torch.as_tensor(b).double()
    return float((a - b).abs().max() / max(float(b.abs().max()), 1e-30))


SHIM = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "neural3dstrokes_b200", "shim")


def _with_shim(fn):
    import sys
    sys.path.insert(0, SHIM)
    saved = sys.modules.pop("_gridencoder", None)
    try:
        return fn()
    finally:
        sys.path.remove(SHIM)
        sys.modules.pop("_gridencoder", None)
        if saved is not None:
            sys.modules["_gridencoder"] = saved


def test_shim_exposes_the_backend_functions():
    from neural3dstrokes_b200 import gridencoder as ge

    def check():
        import _gridencoder
        assert _gridencoder.grid_encode_forward is ge.grid_encode_forward
        assert _gridencoder.grid_encode_backward is ge.grid_encode_backward
        assert _gridencoder.grad_total_variation is ge.grad_total_variation
    _with_shim(check)
