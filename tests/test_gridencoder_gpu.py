"""Grid encoder kernels (n3ds_grid_*) on the GPU against the oracle
(oracle/gridencoder.py), against the reference's own kernels (their recorded outputs
in tests/golden/grid_golden.npz, and the reference extension itself when
oracle/_ref/grid holds a build of it), and through the GridEncoder module and the
``_gridencoder`` shim.

Tolerances (normwise relative error, max |a - b| / max |b|) against the oracle:
1e-5 for float32 and float64 outputs, dy_dx and gradients (at levels with a
fractional exponent the kernel's scale comes from CUDA's exp2f, within 2 ulp of
2^x, the oracle's from the rounded power: positions move by about 1e-6 relative;
gradients also see the atomic accumulation order); float64 tables with integer
exponents 1e-6 (positions and corner weights are float32 for every table type, as
in the reference); float16 4e-3 forward / 2e-2 gradients (half rounding). Against the
reference's kernels, which take the same float32 steps: 1e-6 forward (bit-equal at
the proposal size), 1e-5 gradients.
"""
import glob
import importlib.machinery
import importlib.util
import os
import sys

import numpy as np
import pytest
import torch

from neural3dstrokes_b200 import gridencoder as ge
from oracle import gridencoder as og

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel(a, b):
    a = torch.as_tensor(a).detach().double().cpu()
    b = torch.as_tensor(b).detach().double().cpu()
    return float((a - b).abs().max() / max(float(b.abs().max()), 1e-30))


def make_case(D, C, L, S, H, log2_rows, align, B, seed, dtype=torch.float32, outside=True):
    g = torch.Generator().manual_seed(seed)
    offsets = [0]
    for lv in range(L):
        _, res = og.level_constants(lv, S, H)
        dense = (res if align else res + 1) ** D
        offsets.append(offsets[-1] + int(np.ceil(min(2 ** log2_rows, dense) / 8) * 8))
    x = torch.rand(B, D, generator=g)
    if outside:
        x[:B // 16] = x[:B // 16] * 1.4 - 0.2
    emb = (torch.rand(offsets[-1], C, generator=g, dtype=torch.float64) * 2 - 1).to(dtype)
    grad = torch.randn(L, B, C, generator=g, dtype=torch.float64).to(dtype)
    return x, emb, torch.tensor(offsets, dtype=torch.int32), grad


def run_ours(x, emb, offs, grad, S, H, gt, al, it, dev, tv_weight=1e-3):
    B, D = x.shape
    L, C = offs.numel() - 1, emb.shape[1]
    xd, ed, od = x.to(dev), emb.to(dev), offs.to(dev)
    out = torch.empty(L, B, C, device=dev, dtype=emb.dtype)
    dydx = torch.empty(B, L * D * C, device=dev, dtype=emb.dtype)
    ge.grid_encode_forward(xd, ed, od, out, B, D, C, L, S, H, dydx, gt, al, it)
    gemb = torch.zeros_like(ed)
    gin = torch.zeros(B, D, device=dev, dtype=emb.dtype)
    ge.grid_encode_backward(grad.to(dev), xd, ed, od, gemb, B, D, C, L, S, H, dydx, gin, gt, al, it)
    tv = torch.zeros_like(ed)
    ge.grad_total_variation(xd.to(emb.dtype), ed, tv, od, tv_weight, B, D, C, L, S, H, gt, al)
    torch.cuda.synchronize(dev)
    return out, dydx, gemb, gin, tv


CASES = [  # D, C, L, S, H, log2 rows, gridtype, align, interp
    (3, 4, 5, 1.0, 4, 10, 0, False, 0),
    (3, 2, 4, 0.6, 5, 9, 0, False, 1),
    (3, 1, 4, 0.5, 3, 11, 1, True, 0),
    (3, 8, 3, 0.9, 6, 12, 0, True, 1),
    (2, 8, 6, 0.75, 4, 8, 0, False, 0),
    (2, 4, 3, 1.0, 6, 12, 1, True, 1),
    (4, 2, 3, 0.5, 3, 12, 0, False, 0),
    (5, 1, 2, 0.5, 2, 12, 1, False, 1),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "D{}C{}L{}_g{}a{}i{}".format(c[0], c[1], c[2], *c[6:]))
def test_kernels_match_oracle(cuda, case):
    D, C, L, S, H, lr, gt, al, it = case
    x, emb, offs, grad = make_case(D, C, L, S, H, lr, al, 700, seed=sum(case[:3]))
    out, dydx, gemb, gin, tv = run_ours(x, emb, offs, grad, S, H, gt, al, it, cuda)
    o_out, o_dydx = og.grid_encode_forward(x, emb, offs, S, H, True, gt, al, it)
    assert rel(out, o_out) < 1e-5
    assert rel(dydx, o_dydx) < 1e-5
    o_gemb, o_gin = og.grid_encode_backward(grad, x, emb, offs, S, H, o_dydx, gt, al, it)
    assert rel(gemb, o_gemb) < 1e-5
    assert rel(gin, o_gin) < 1e-5
    o_tv = og.grad_total_variation(x, emb, torch.zeros_like(emb), offs, 1e-3, S, H, gt, al)
    assert rel(tv, o_tv) < 1e-5


@pytest.mark.parametrize("dtype", [torch.float64, torch.float16])
def test_other_dtypes_match_oracle(cuda, dtype):
    # the kernels, as the reference's, form positions and corner weights in float32
    # for every table type, so float64 tables agree with the oracle to ~1e-7
    D, C, L, S, H, lr, gt, al, it = 3, 4, 4, 1.0, 4, 10, 0, False, 0
    x, emb, offs, grad = make_case(D, C, L, S, H, lr, al, 500, seed=5, dtype=dtype)
    out, dydx, gemb, gin, tv = run_ours(x, emb, offs, grad, S, H, gt, al, it, cuda)
    o_out, o_dydx = og.grid_encode_forward(x, emb, offs, S, H, True, gt, al, it)
    o_gemb, o_gin = og.grid_encode_backward(grad, x, emb, offs, S, H, o_dydx, gt, al, it)
    if dtype == torch.float64:
        for a, b in ((out, o_out), (dydx, o_dydx), (gemb, o_gemb), (gin, o_gin)):
            assert rel(a, b) < 1e-6
    else:
        assert rel(out, o_out) < 4e-3 and rel(dydx, o_dydx) < 4e-3
        assert rel(gemb, o_gemb) < 2e-2 and rel(gin, o_gin) < 2e-2


def golden():
    path = os.path.join(ROOT, "tests", "golden", "grid_golden.npz")
    if not os.path.exists(path):
        return None, []
    z = np.load(path)
    return z, sorted({k.split("/")[0] for k in z.files})


@pytest.mark.parametrize("tag", golden()[1])
def test_kernels_match_reference_golden(cuda, tag):
    z, _ = golden()
    D, C, L, S, H, gt, al, it = z[f"{tag}/meta"].tolist()
    D, C, L, H, gt, al, it = int(D), int(C), int(L), int(H), int(gt), bool(al), int(it)
    x = torch.from_numpy(z[f"{tag}/inputs"])
    emb = torch.from_numpy(z[f"{tag}/embeddings"])
    offs = torch.from_numpy(z[f"{tag}/offsets"])
    grad = torch.from_numpy(z[f"{tag}/grad"])
    out, dydx, gemb, gin, tv = run_ours(x, emb, offs, grad, S, H, gt, al, it, cuda)
    if emb.dtype == torch.float16:
        ftol, gtol = 4e-3, 2e-2
    elif emb.dtype == torch.float64:
        ftol, gtol = 1e-12, 1e-12
    else:
        ftol, gtol = 1e-6, 1e-5
    assert rel(out, z[f"{tag}/outputs"]) < ftol
    assert rel(dydx, z[f"{tag}/dy_dx"]) < max(ftol, 1e-6) * 4
    assert rel(gemb, z[f"{tag}/grad_embeddings"]) < gtol
    assert rel(gin, z[f"{tag}/grad_inputs"]) < gtol
    if emb.dtype != torch.float16:
        assert rel(tv, z[f"{tag}/tv"]) < max(gtol, 1e-6)


def reference_module():
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "grid", "_gridencoder*.so"))
    if not hits:
        return None
    loader = importlib.machinery.ExtensionFileLoader("_gridencoder", hits[0])
    spec = importlib.util.spec_from_file_location("_gridencoder", hits[0], loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def test_kernels_match_reference_extension_at_proposal_size(cuda):
    """The proposal network's grid (L = 10, C = 4, 2^21 rows per fine level) on 2^18
    points, against the reference kernels built from their sources."""
    ref = reference_module()
    if ref is None:
        pytest.skip("reference grid encoder not built (oracle/build_ref.py --only grid)")
    enc = ge.GridEncoder(input_dim=3, num_levels=10, level_dim=4, base_resolution=16, desired_resolution=8192,
                         log2_hashmap_size=21).to(cuda)
    g = torch.Generator(device=cuda).manual_seed(3)
    with torch.no_grad():
        enc.embeddings.uniform_(-1, 1, generator=g)
    B, D, C, L = 1 << 18, 3, 4, 10
    S, H = float(np.log2(enc.per_level_scale)), 16
    x = torch.rand(B, D, device=cuda, generator=g)
    outs = []
    for mod in (ref, ge):
        out = torch.empty(L, B, C, device=cuda)
        dydx = torch.empty(B, L * D * C, device=cuda)
        mod.grid_encode_forward(x, enc.embeddings.data, enc.offsets, out, B, D, C, L, S, H, dydx, 0, False, 0)
        grad = torch.randn(L, B, C, device=cuda, generator=torch.Generator(device=cuda).manual_seed(4))
        gemb = torch.zeros_like(enc.embeddings.data)
        gin = torch.zeros(B, D, device=cuda)
        mod.grid_encode_backward(grad, x, enc.embeddings.data, enc.offsets, gemb, B, D, C, L, S, H, dydx, gin, 0,
                                 False, 0)
        outs.append((out, dydx, gemb, gin))
    torch.cuda.synchronize(cuda)
    (r_out, r_dd, r_ge, r_gi), (o_out, o_dd, o_ge, o_gi) = outs
    assert torch.equal(o_out, r_out)          # same float32 steps in the same order
    assert rel(o_dd, r_dd) < 1e-6
    assert rel(o_ge, r_ge) < 1e-5
    assert rel(o_gi, r_gi) < 1e-5


def test_module_autograd_matches_oracle(cuda):
    torch.manual_seed(0)
    enc = ge.GridEncoder(input_dim=3, num_levels=4, level_dim=2, per_level_scale=1.7, base_resolution=5,
                         log2_hashmap_size=10, init_std=0.5).to(cuda)
    pts = (torch.rand(300, 3, device=cuda) * 2 - 1) * 0.99
    pts.requires_grad_(True)
    y = enc(pts, bound=1)
    assert y.shape == (300, 8)
    up = torch.randn_like(y)
    (y * up).sum().backward()
    xin = ((pts.detach() + 1) / 2).cpu()
    S = float(np.log2(1.7))
    o_out, o_dd = og.grid_encode_forward(xin, enc.embeddings.detach().cpu(), enc.offsets.cpu(), S, 5, True)
    assert rel(y, o_out.permute(1, 0, 2).reshape(300, 8)) < 1e-5
    g = up.view(300, 4, 2).permute(1, 0, 2).cpu()
    o_ge, o_gi = og.grid_encode_backward(g, xin, enc.embeddings.detach().cpu(), enc.offsets.cpu(), S, 5, o_dd)
    assert rel(enc.embeddings.grad, o_ge) < 1e-5
    assert rel(pts.grad, o_gi / 2) < 1e-5        # d inputs / d pts = 1 / (2 bound)


def test_module_under_autocast_uses_half_tables(cuda):
    torch.manual_seed(1)
    enc = ge.GridEncoder(num_levels=4, level_dim=4, log2_hashmap_size=12, init_std=0.5).to(cuda)
    pts = torch.rand(1000, 3, device=cuda) * 2 - 1
    y32 = enc(pts)
    with torch.autocast("cuda", dtype=torch.float16):
        y16 = enc(pts)
    assert y16.dtype == torch.float16
    assert rel(y16, y32) < 4e-3
    y16.float().sum().backward()
    assert enc.embeddings.grad.dtype == torch.float32 and enc.embeddings.grad.abs().sum() > 0


def test_total_variation_method(cuda):
    torch.manual_seed(2)
    enc = ge.GridEncoder(num_levels=3, level_dim=2, log2_hashmap_size=11, init_std=0.5).to(cuda)
    pts = torch.rand(400, 3, device=cuda) * 2 - 1
    with pytest.raises(ValueError):
        enc.grad_total_variation(1e-2, pts)
    enc(pts).sum().backward()
    before = enc.embeddings.grad.clone()
    enc.grad_total_variation(1e-2, pts)
    o = og.grad_total_variation(((pts + 1) / 2).cpu(), enc.embeddings.detach().cpu(), before.cpu(), enc.offsets.cpu(),
                                1e-2, 1.0, 16)
    assert rel(enc.embeddings.grad, o) < 1e-5
    enc.grad_total_variation(1e-2, B=4096)      # random points: runs and changes the gradient
    assert not torch.equal(enc.embeddings.grad, before)


def test_shim_module_binds_these_kernels(cuda):
    shim = os.path.join(ROOT, "neural3dstrokes_b200", "shim")
    sys.path.insert(0, shim)
    try:
        sys.modules.pop("_gridencoder", None)
        import _gridencoder
        assert _gridencoder.grid_encode_forward is ge.grid_encode_forward
        assert _gridencoder.grid_encode_backward is ge.grid_encode_backward
        assert _gridencoder.grad_total_variation is ge.grad_total_variation
    finally:
        sys.path.remove(shim)
        sys.modules.pop("_gridencoder", None)


def test_misaligned_table_and_outputs(cuda):
    D, C, L, S, H, lr = 3, 4, 3, 1.0, 4, 10
    x, emb, offs, grad = make_case(D, C, L, S, H, lr, False, 300, seed=9)
    B = x.shape[0]
    flat = torch.empty(emb.numel() + 1, device=cuda)
    e_mis = flat[1:].view(emb.shape)
    e_mis.copy_(emb.to(cuda))
    assert e_mis.data_ptr() % 16 != 0
    oflat = torch.empty(L * B * C + 1, device=cuda)
    out = oflat[1:].view(L, B, C)
    xd, od = x.to(cuda), offs.to(cuda)
    ge.grid_encode_forward(xd, e_mis, od, out, B, D, C, L, S, H, None, 0, False, 0)
    gflat = torch.zeros(emb.numel() + 1, device=cuda)
    g_mis = gflat[1:].view(emb.shape)
    ge.grid_encode_backward(grad.to(cuda), xd, e_mis, od, g_mis, B, D, C, L, S, H, None, None, 0, False, 0)
    o_out, _ = og.grid_encode_forward(x, emb, offs, S, H)
    o_ge, _ = og.grid_encode_backward(grad, x, emb, offs, S, H)
    assert rel(out, o_out) < 1e-5 and rel(g_mis, o_ge) < 1e-5


def test_errors_raise(cuda):
    x, emb, offs, grad = make_case(3, 4, 2, 1.0, 4, 8, False, 64, seed=1)
    xd, ed, od = x.to(cuda), emb.to(cuda), offs.to(cuda)
    out = torch.empty(2, 64, 4, device=cuda)
    with pytest.raises(RuntimeError, match="C must be"):
        ge.grid_encode_forward(xd, ed[:, :3].contiguous(), od, out, 64, 3, 3, 2, 1.0, 4)
    with pytest.raises(RuntimeError, match="CUDA"):
        ge.grid_encode_forward(x, ed, od, out, 64, 3, 4, 2, 1.0, 4)
    with pytest.raises(RuntimeError, match="contiguous"):
        ge.grid_encode_forward(xd.t(), ed, od, out, 64, 3, 4, 2, 1.0, 4)
    with pytest.raises(RuntimeError, match="int"):
        ge.grid_encode_forward(xd, ed, od.long(), out, 64, 3, 4, 2, 1.0, 4)
    with pytest.raises(RuntimeError, match="outputs"):
        ge.grid_encode_forward(xd, ed, od, out[:1], 64, 3, 4, 2, 1.0, 4)
    bad = od.clone()
    bad[-1] = emb.shape[0] + 8
    with pytest.raises(RuntimeError, match="offsets"):
        ge.grid_encode_forward(xd, ed, bad, out, 64, 3, 4, 2, 1.0, 4)
    with pytest.raises(RuntimeError, match="D must be"):
        ge.grid_encode_forward(xd, ed, od, out, 64, 6, 4, 2, 1.0, 4)


def test_full_size_level_sums(cuda):
    """Proposal-network grid at 2^21 points: every in-range point's corner weights sum
    to one, so each level's table-gradient sum equals that level's grad sum over the
    in-range points; a 4096-point subset matches the oracle."""
    enc = ge.GridEncoder(input_dim=3, num_levels=10, level_dim=4, base_resolution=16, desired_resolution=8192,
                         log2_hashmap_size=21).to(cuda)
    g = torch.Generator(device=cuda).manual_seed(7)
    with torch.no_grad():
        enc.embeddings.uniform_(-1, 1, generator=g)
    B, D, C, L = 1 << 21, 3, 4, 10
    S, H = float(np.log2(enc.per_level_scale)), 16
    x = torch.rand(B, D, device=cuda, generator=g) * 1.02 - 0.01
    out = torch.empty(L, B, C, device=cuda)
    ge.grid_encode_forward(x, enc.embeddings.data, enc.offsets, out, B, D, C, L, S, H)
    grad = torch.randn(L, B, C, device=cuda, generator=g)
    gemb = torch.zeros_like(enc.embeddings.data)
    ge.grid_encode_backward(grad, x, enc.embeddings.data, enc.offsets, gemb, B, D, C, L, S, H)
    ok = ((x >= 0) & (x <= 1)).all(-1)
    offs = enc.offsets.tolist()
    for lv in range(L):
        want = grad[lv][ok].double().sum(0)
        got = gemb[offs[lv]:offs[lv + 1]].double().sum(0)
        assert (got - want).abs().max() < 1e-3 * grad[lv][ok].abs().sum(0).max() ** 0.5
    sub = torch.randperm(B, device=cuda, generator=g)[:4096]
    o_out, _ = og.grid_encode_forward(x[sub].cpu(), enc.embeddings.detach().cpu(), enc.offsets.cpu(), S, H)
    assert rel(out[:, sub], o_out) < 1e-5


def ray_points(R, N, seed, spread=0.2):
    """R rays of N samples each, ray-ordered as a sampler emits them: neighbours share
    cells at the coarse levels."""
    g = torch.Generator().manual_seed(seed)
    o = torch.rand(R, 1, 3, generator=g) * 0.6 + 0.2
    d = torch.nn.functional.normalize(torch.randn(R, 1, 3, generator=g), dim=-1)
    t = torch.linspace(-spread, spread, N)[None, :, None]
    return (o + d * t).reshape(R * N, 3).contiguous()


def offsets_for(D, L, S, H, log2_rows, align=False):
    offsets = [0]
    for lv in range(L):
        _, res = og.level_constants(lv, S, H)
        dense = (res if align else res + 1) ** D
        offsets.append(offsets[-1] + int(np.ceil(min(2 ** log2_rows, dense) / 8) * 8))
    return torch.tensor(offsets, dtype=torch.int32)


@pytest.mark.parametrize("C,dtype", [(1, torch.float32), (2, torch.float32), (4, torch.float32), (8, torch.float32),
                                     (4, torch.float64), (4, torch.float16)])
def test_backward_runs_of_shared_cells(cuda, C, dtype):
    """Ray-ordered points (the warp-run aggregation of the backward), out-of-range points
    inside runs, a partial last warp (B = 1073)."""
    x = ray_points(37, 29, seed=C)
    x[::17] = 1.3
    S, H, L = 1.0, 4, 6
    offs = offsets_for(3, L, S, H, 12)
    g = torch.Generator().manual_seed(40 + C)
    emb = (torch.rand(int(offs[-1]), C, generator=g, dtype=torch.float64) * 2 - 1).to(dtype)
    grad = torch.randn(L, x.shape[0], C, generator=g, dtype=torch.float64).to(dtype)
    out, dydx, gemb, gin, _ = run_ours(x, emb, offs, grad, S, H, 0, False, 0, cuda)
    o_out, o_dd = og.grid_encode_forward(x, emb, offs, S, H, True)
    o_ge, o_gi = og.grid_encode_backward(grad, x, emb, offs, S, H, o_dd)
    ftol, gtol = (4e-3, 2e-2) if dtype == torch.float16 else (1e-5, 1e-5)
    assert rel(out, o_out) < ftol
    assert rel(gemb, o_ge) < gtol
    assert rel(gin, o_gi) < gtol


@pytest.mark.parametrize("C,dtype", [(4, torch.float32), (2, torch.float32), (1, torch.float32),
                                     (2, torch.float16), (4, torch.float16)])
def test_odd_level_offsets(cuda, C, dtype):
    """Offsets the C ABI accepts but GridEncoder never builds: odd level starts and
    odd row counts, on levels large enough (>= 2^19 rows) for the paired row loads,
    which must fall back to single rows at an odd start or at a level's last row;
    and small odd levels."""
    offs = torch.tensor([0, 524289, 1048582, 1572870, 1572883, 1572910], dtype=torch.int32)
    g = torch.Generator().manual_seed(C)
    x = torch.cat([torch.rand(3000, 3, generator=g), ray_points(20, 50, seed=3), torch.ones(4, 3)])
    emb = (torch.rand(int(offs[-1]), C, generator=g, dtype=torch.float64) * 2 - 1).to(dtype)
    grad = torch.randn(5, x.shape[0], C, generator=g, dtype=torch.float64).to(dtype)
    for gt, S, H in ((0, 1.0, 64), (1, 1.0, 3)):
        out, dydx, gemb, gin, tv = run_ours(x, emb, offs, grad, S, H, gt, False, 0, cuda)
        o_out, o_dd = og.grid_encode_forward(x, emb, offs, S, H, True, gt)
        o_ge, _ = og.grid_encode_backward(grad, x, emb, offs, S, H, None, gt)
        ftol, gtol = (4e-3, 2e-2) if dtype == torch.float16 else (1e-5, 1e-5)
        assert rel(out, o_out) < ftol and rel(dydx, o_dd) < ftol
        assert rel(gemb, o_ge) < gtol
