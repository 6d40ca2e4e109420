"""Colour fields of the drop-in stroke operators (gradient rgb, SH2, SH3): colours
against the float64 oracle (1e-5), exact gradients against float64 autograd of the
oracle (1e-4; includes the gradient rgb's dependence on the sample position, which
the reference drops), compat gradients against the reference op itself (1e-4)."""
import pytest
import torch

from helpers import FWD_TOL, GRAD_TOL, rel
from neural3dstrokes_b200 import scenes
from neural3dstrokes_b200 import strokelib as sl
from oracle import cpu_port
from oracle import strokefield as sf

pytestmark = pytest.mark.gpu

KINDS = ["sphere", "obb", "capsule", "cubic_bezier", "tetrahedron"]
NPC = {1: 12, 2: 12, 3: 27}


def case(kind, cid, seed=0, n_strokes=20, n_rays=40, n_samples=16):
    g = torch.Generator().manual_seed(seed + 31 * cid)
    sc = scenes.make_strokes([kind] * n_strokes, g)
    rays = scenes.make_rays(n_rays, n_samples, g)
    sid = scenes.SDF_ID[kind]
    ps = sc.shape_params[:, :sf.num_shape_params(sid)].contiguous()
    if cid == 1:
        cp = torch.cat([torch.rand(n_strokes, 6, generator=g) * 2 - 1, torch.rand(n_strokes, 6, generator=g)], -1)
    else:
        cp = torch.randn(n_strokes, NPC[cid], generator=g)
    x = rays.x.reshape(-1, 3).contiguous()
    r = rays.radius.reshape(-1).contiguous()
    vd = (rays.dirs / rays.dirs.norm(dim=-1, keepdim=True)).contiguous()
    return sid, ps, cp, x, r, vd


def fwd(sid, cid, ps, cp, x, r, vd, dev):
    P, S = x.shape[0], ps.shape[0]
    a = torch.empty(P, S, device=dev)
    c = torch.empty(P, S, 3, device=dev)
    sl.stroke_forward(a, c, torch.empty(0, device=dev), torch.empty(0, device=dev), x.to(dev), r.to(dev),
                      vd.to(dev), ps.to(dev), cp.to(dev), sid, cid, 0.02, True, True)
    return a, c


@pytest.mark.parametrize("cid", [1, 2, 3])
@pytest.mark.parametrize("kind", KINDS)
def test_color_field_forward(cuda, kind, cid):
    sid, ps, cp, x, r, vd = case(kind, cid)
    a, c = fwd(sid, cid, ps, cp, x, r, vd, cuda)
    a_r, c_r = sf.stroke_forward(x.double(), r.double(), ps.double(), cp.double(), sid, 0.02, True, True,
                                 color_id=cid, viewdir=vd.double())
    assert rel(c, c_r) < FWD_TOL and rel(a, a_r) < FWD_TOL


@pytest.mark.parametrize("cid", [1, 2, 3])
@pytest.mark.parametrize("kind", KINDS)
def test_color_field_exact_backward(cuda, kind, cid):
    sid, ps, cp, x, r, vd = case(kind, cid, seed=5)
    P, S = x.shape[0], ps.shape[0]
    g = torch.Generator().manual_seed(9)
    ga, gc = torch.randn(P, S, generator=g), torch.randn(P, S, 3, generator=g)
    a, _ = fwd(sid, cid, ps, cp, x, r, vd, cuda)
    gps, gcp, gx = (torch.zeros_like(ps, device=cuda), torch.zeros_like(cp, device=cuda),
                    torch.zeros(P, 3, device=cuda))
    sl.set_grad_mode("exact")
    sl.stroke_backward(gps, gcp, gx, ga.to(cuda), gc.to(cuda), torch.empty(0, device=cuda), x.to(cuda), r.to(cuda),
                       vd.to(cuda), a, ps.to(cuda), cp.to(cuda), sid, cid, 0.02, True, True)
    xd, pd, cd = (t.double().requires_grad_(True) for t in (x, ps, cp))
    a_r, c_r = sf.stroke_forward(xd, r.double(), pd, cd, sid, 0.02, True, True, color_id=cid, viewdir=vd.double())
    ((a_r * ga.double()).sum() + (c_r * gc.double()).sum()).backward()
    assert rel(gcp, cd.grad) < GRAD_TOL, rel(gcp, cd.grad)
    assert rel(gps, pd.grad) < GRAD_TOL, rel(gps, pd.grad)
    assert rel(gx, xd.grad) < GRAD_TOL, rel(gx, xd.grad)


@pytest.mark.parametrize("cid", [1, 2, 3])
@pytest.mark.parametrize("kind", ["sphere", "obb", "cubic_bezier"])
def test_color_field_compat_matches_reference_op(cuda, kind, cid):
    ref = cpu_port.reference_extension()
    if ref is None:
        pytest.skip("reference extension not built (oracle/_ref)")
    sid, ps, cp, x, r, vd = case(kind, cid, seed=11)
    P, S = x.shape[0], ps.shape[0]
    g = torch.Generator().manual_seed(3)
    ga, gc = torch.randn(P, S, generator=g).to(cuda), torch.randn(P, S, 3, generator=g).to(cuda)
    a_r = torch.empty(P, S, device=cuda)
    c_r = torch.empty(P, S, 3, device=cuda)
    ref.stroke_forward(a_r, c_r, torch.empty(0, device=cuda), torch.empty(0, device=cuda), x.to(cuda), r.to(cuda),
                       vd.to(cuda), ps.to(cuda), cp.to(cuda), sid, cid, 0.02, True, True)
    a, c = fwd(sid, cid, ps, cp, x, r, vd, cuda)
    assert rel(c, c_r) < FWD_TOL
    outs = []
    for impl in (sl, ref):
        gps, gcp, gx = (torch.zeros_like(ps, device=cuda), torch.zeros_like(cp, device=cuda),
                        torch.zeros(P, 3, device=cuda))
        sl.set_grad_mode("compat")
        try:
            impl.stroke_backward(gps, gcp, gx, ga, gc, torch.empty(0, device=cuda), x.to(cuda), r.to(cuda),
                                 vd.to(cuda), a_r, ps.to(cuda), cp.to(cuda), sid, cid, 0.02, True, True)
        finally:
            sl.set_grad_mode("exact")
        outs.append((gps, gcp, gx))
    for m, rr in zip(*outs):
        assert rel(m, rr) < GRAD_TOL, rel(m, rr)


@pytest.mark.parametrize("kind", ["sphere", "ellipsoid", "cube", "aabb", "roundbox", "capsule", "scapsule", "line",
                                  "octahedron", "cubic_bezier"])
def test_texcoord_matches_oracle(cuda, kind):
    g = torch.Generator().manual_seed(41)
    sc = scenes.make_strokes([kind] * 10, g)
    rays = scenes.make_rays(30, 12, g)
    sid = scenes.SDF_ID[kind]
    ps = sc.shape_params[:, :sf.num_shape_params(sid)].contiguous()
    x = rays.x.reshape(-1, 3).contiguous()
    r = rays.radius.reshape(-1).contiguous()
    P, S = x.shape[0], ps.shape[0]
    a = torch.empty(P, S, device=cuda)
    c = torch.empty(P, S, 3, device=cuda)
    tex = torch.empty(P, S, 2, device=cuda)
    sl.stroke_forward(a, c, torch.empty(0, device=cuda), tex, x.to(cuda), r.to(cuda), rays.dirs.to(cuda), ps.to(cuda),
                      sc.color_params.to(cuda), sid, 0, 0.02, True, True)
    *_, tex_r = sf.stroke_forward(x.double(), r.double(), ps.double(), sc.color_params.double(), sid, 0.02, True, True,
                                  return_texcoord=True)
    d = (tex.cpu().double() - tex_r).abs()
    d = torch.minimum(d, (1.0 - d).abs())
    assert float(d.max()) < 1e-5, float(d.max())
