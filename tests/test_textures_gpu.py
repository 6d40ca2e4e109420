"""ImageTexture on CUDA (n3ds_texture_forward / _backward) against the float64 oracle
(F.grid_sample, textures.py:58-83). Tolerances: forward 1e-5, gradients 1e-5
(normwise relative)."""
import pytest
import torch

from helpers import rel
from oracle import strokefield as orr
from neural3dstrokes_b200 import textures

pytestmark = pytest.mark.gpu


def make(C, P=300, S=7, H=17, W=23, seed=0, lo=-0.15, hi=1.15):
    g = torch.Generator().manual_seed(seed)
    tc = lo + (hi - lo) * torch.rand(P, S, 2, generator=g)
    tc[0, :, 0] = 0.0  # exact edges
    tc[1, :, 1] = 1.0
    col = torch.rand(P, S, 3, generator=g)
    al = torch.rand(P, S, generator=g)
    img = torch.rand(1, C, H, W, generator=g) * 255
    return tc, col, al, img


@pytest.mark.parametrize("C", [3, 1])
@pytest.mark.parametrize("tint_ratio,modulate", [(1.0, False), (0.6, True), (0.0, True)])
def test_texture_matches_oracle(cuda, C, tint_ratio, modulate):
    tc, col, al, img = make(C)
    tex = textures.ImageTexture(img[0].permute(1, 2, 0).numpy(), img.shape[2:], tint_ratio=tint_ratio,
                                modulate_alpha=modulate)
    colc, alc = col.to(cuda).requires_grad_(True), al.to(cuda).requires_grad_(True)
    out_c, out_a = tex(tc.to(cuda), colc, alc)
    g = torch.Generator().manual_seed(5)
    gc, ga = torch.randn(out_c.shape, generator=g), torch.randn(out_a.shape, generator=g)
    ((out_c * gc.to(cuda)).sum() + (out_a * ga.to(cuda)).sum()).backward()

    img64 = tex.image_texture[0].double()
    col64, al64 = col.double().requires_grad_(True), al.double().requires_grad_(True)
    ref_c, ref_a = orr.image_texture(tc.double().reshape(-1, 2), col64.reshape(-1, 3), al64.reshape(-1), img64,
                                     tint_ratio, modulate)
    ((ref_c * gc.double().reshape(-1, 3)).sum() + (ref_a * ga.double().reshape(-1)).sum()).backward()
    assert rel(out_c.reshape(-1, 3), ref_c) < 1e-5
    assert rel(out_a.reshape(-1), ref_a) < 1e-5
    assert rel(colc.grad, col64.grad) < 1e-5
    assert rel(alc.grad, al64.grad) < 1e-5


def test_texture_empty_and_nonfinite(cuda):
    tex = textures.ImageTexture(torch.rand(8, 8, 3).numpy() * 255, (8, 8))
    c, a = tex(torch.zeros(0, 2, device=cuda), torch.zeros(0, 3, device=cuda), torch.zeros(0, device=cuda))
    assert c.shape == (0, 3) and a.shape == (0,)
    tc = torch.tensor([[float("nan"), 0.5], [0.5, float("inf")], [1e30, -1e30]], device=cuda)
    c, a = tex(tc, torch.ones(3, 3, device=cuda), torch.ones(3, device=cuda))
    assert torch.all(c == 0)  # no pixel read: zero tint
    assert torch.all(a == 1)  # alphas untouched without modulate_alpha


def test_texture_in_stroke_pipeline(cuda):
    """stroke_fn with texcoords -> ImageTexture -> compose_strokes, as models.py:681-709."""
    from neural3dstrokes_b200 import strokes
    stroke_fn, *_ = strokes.get_stroke("sphere", "constant_rgb", "random")
    g = torch.Generator().manual_seed(2)
    S, P = 6, 400
    shape = torch.cat([torch.rand(S, 1, generator=g) * 0.3 + 0.2, torch.rand(S, 3, generator=g) - 0.5], 1)
    color = torch.rand(S, 3, generator=g)
    x = torch.rand(P, 3, generator=g) * 1.4 - 0.7
    radius = torch.full((P,), 0.01)
    tex = textures.ImageTexture(torch.rand(32, 32, 3, generator=g).numpy() * 255, (16, 16), modulate_alpha=True)
    out = stroke_fn(x.to(cuda), radius.to(cuda), torch.zeros(P, 3, device=cuda), shape.to(cuda), color.to(cuda),
                    0.02, True, True, True, True)
    alphas, colors, texcoords = out[0], out[1], out[-1]
    assert texcoords.shape == (P, S, 2)
    c2, a2 = tex(texcoords, colors, alphas)
    dens, rgb = strokes.compose_strokes(a2, c2, torch.full((S,), 10.0, device=cuda), "over")
    ref_c, ref_a = orr.image_texture(texcoords.double().reshape(-1, 2).cpu(), colors.double().reshape(-1, 3).cpu(),
                                     alphas.double().reshape(-1).cpu(), tex.image_texture[0].double(), 1.0, True)
    assert rel(c2.reshape(-1, 3), ref_c) < 1e-5 and rel(a2.reshape(-1), ref_a) < 1e-5
    assert torch.isfinite(rgb).all() and torch.isfinite(dens).all()


@pytest.mark.parametrize("C,modulate", [(3, True), (1, True), (3, False)])
def test_packed_texture_equals_planar(cuda, C, modulate):
    """n3ds_texture_forward/backward_packed (float4 texels, what ImageTexture runs) give
    the planar entry points' results to a few ulps (the compiler contracts the two
    four-term sums into FMAs differently), outside and non-finite coordinates
    included."""
    from neural3dstrokes_b200 import _lib
    g = torch.Generator().manual_seed(C)
    H, W, n = 37, 53, 5000
    img = torch.rand(C, H, W, generator=g).to(cuda)
    tc = (torch.rand(n, 2, generator=g) * 1.4 - 0.2).to(cuda)
    tc[:5, 0] = float("nan")
    tc[5:10, 1] = float("inf")
    col = torch.rand(n, 3, generator=g).to(cuda)
    al = torch.rand(n, generator=g).to(cuda)
    gco, gal = torch.randn(n, 3, generator=g).to(cuda), torch.randn(n, generator=g).to(cuda)
    packed = torch.empty(H, W, 4, device=cuda)
    lib, st = _lib.load(), _lib.stream_ptr()
    P = _lib.ptr
    _lib.check(lib.n3ds_texture_pack(P(packed), P(img), C, H, W, st))
    outs = []
    for fwd, bwd, im in ((lib.n3ds_texture_forward, lib.n3ds_texture_backward, img),
                         (lib.n3ds_texture_forward_packed, lib.n3ds_texture_backward_packed, packed)):
        co, ao = torch.empty_like(col), torch.empty_like(al)
        gc, ga = torch.empty_like(col), torch.empty_like(al)
        _lib.check(fwd(P(co), P(ao), P(tc), P(col), P(al), n, P(im), C, H, W, 0.7, int(modulate), st))
        _lib.check(bwd(P(gc), P(ga), P(gco), P(gal), P(tc), n, P(im), C, H, W, 0.7, int(modulate), st))
        outs.append((co, ao, gc, ga))
    torch.cuda.synchronize(cuda)
    for a, b in zip(*outs):
        assert rel(a, b) < 1e-6


@pytest.mark.parametrize("P,offset", [(301, 0), (300, 1)])
@pytest.mark.parametrize("modulate", [False, True])
def test_texture_tail_and_unaligned_arrays(cuda, P, offset, modulate):
    """The kernels take four pairs per thread on 16-byte-aligned arrays and the rest
    one by one: a pair count that is not a multiple of four and colours one float into
    a buffer (the whole call on the scalar path) give the oracle's values too."""
    tc, col, al, img = make(3, P=P, seed=3)
    tex = textures.ImageTexture(img[0].permute(1, 2, 0).numpy(), img.shape[2:], tint_ratio=0.7,
                                modulate_alpha=modulate)
    buf = torch.empty(col.numel() + offset, device=cuda)
    buf[offset:] = col.reshape(-1).to(cuda)
    colc = buf[offset:].view(col.shape).detach().requires_grad_(True)
    alc = al.to(cuda).requires_grad_(True)
    out_c, out_a = tex(tc.to(cuda), colc, alc)
    if not modulate:
        assert out_a is alc  # the reference returns its alphas unchanged
    g = torch.Generator().manual_seed(6)
    gc = torch.randn(out_c.shape, generator=g)
    (out_c * gc.to(cuda)).sum().backward()
    img64 = tex.image_texture[0].double()
    col64 = col.double().requires_grad_(True)
    ref_c, ref_a = orr.image_texture(tc.double().reshape(-1, 2), col64.reshape(-1, 3), al.double().reshape(-1), img64,
                                     0.7, modulate)
    (ref_c * gc.double().reshape(-1, 3)).sum().backward()
    assert rel(out_c.reshape(-1, 3), ref_c) < 1e-5 and rel(out_a.reshape(-1), ref_a) < 1e-5
    assert rel(colc.grad, col64.grad) < 1e-5
