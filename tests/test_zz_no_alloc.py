"""n3ds_stroke_forward_static (static device scratch, no workspace, no allocation)
against n3ds_stroke_forward with a caller workspace, both through the C ABI.

Collected last (file name) so that it also runs after every other GPU test has used
the device; it passes alone in a fresh process too. Tolerance: forward 1e-5
(helpers.FWD_TOL, normwise relative).
"""
import pytest
import torch

from helpers import FWD_TOL, rel
from neural3dstrokes_b200 import _lib, scenes
from oracle import strokefield as sf

pytestmark = pytest.mark.gpu

MAX_STROKES = 4096  # N3DS_STATIC_MAX_STROKES


def _inputs(kind, n_strokes, n_rays, seed):
    g = torch.Generator().manual_seed(seed)
    sc = scenes.make_strokes([kind] * n_strokes, g)
    rays = scenes.make_rays(n_rays, 32, g)
    sid = scenes.SDF_ID[kind]
    dev = torch.device("cuda:0")
    ps = sc.shape_params[:, :sf.num_shape_params(sid)].contiguous().to(dev)
    col = sc.color_params.contiguous().to(dev)
    x = rays.x.reshape(-1, 3).contiguous().to(dev)
    r = rays.radius.reshape(-1).contiguous().to(dev)
    vd = rays.dirs.contiguous().to(dev)
    return sid, ps, col, x, r, vd


def _outputs(P, S, dev):
    return torch.full((P, S), float("nan"), device=dev), torch.full((P, S, 3), float("nan"), device=dev), \
        torch.full((P, S), float("nan"), device=dev)


def _call(lib, fn, outs, sid, ps, col, x, r, vd, delta, lap, inv, ws=None, color_id=0, tex=None):
    a, c, d = outs
    P, S = x.shape[0], ps.shape[0]
    args = [_lib.ptr(a), _lib.ptr(c), _lib.ptr(d), _lib.ptr(tex), 0 if tex is None else tex.numel(), _lib.ptr(x),
            _lib.ptr(r), _lib.ptr(vd), _lib.ptr(ps), _lib.ptr(col), P, vd.shape[0], S, ps.shape[1], col.shape[1], sid,
            color_id, delta, int(lap), int(inv)]
    if ws is not None:
        args += [_lib.ptr(ws), ws.numel()]
    rc = fn(*args, _lib.stream_ptr())
    if rc:
        raise RuntimeError(lib.n3ds_last_error().decode())


@pytest.mark.parametrize("kind,n_strokes,lap,inv", [("sphere", 300, True, True), ("cube", 96, True, False),
                                                    ("capsule", 50, False, True), ("quadratic_bezier", 64, True, True),
                                                    ("cubic_bezier", 40, True, True)])
def test_static_scratch_matches_workspace_entry_point(kind, n_strokes, lap, inv):
    lib = _lib.load()
    dev = torch.device("cuda:0")
    sid, ps, col, x, r, vd = _inputs(kind, n_strokes, 64, seed=7 + n_strokes)
    P, S = x.shape[0], ps.shape[0]
    delta = 0.02 if lap else 0.5
    want = _outputs(P, S, dev)
    ws = _lib.workspace(lib.n3ds_stroke_workspace_bytes(S), dev)
    _call(lib, lib.n3ds_stroke_forward, want, sid, ps, col, x, r, vd, delta, lap, inv, ws)
    for _ in range(2):  # two calls in a row on the same scratch
        got = _outputs(P, S, dev)
        _call(lib, lib.n3ds_stroke_forward_static, got, sid, ps, col, x, r, vd, delta, lap, inv)
        torch.cuda.synchronize()
        for g_, w_ in zip(got, want):
            assert torch.isfinite(g_).all()
            assert rel(g_, w_) < FWD_TOL


def test_static_scratch_rejects_too_many_strokes():
    lib = _lib.load()
    dev = torch.device("cuda:0")
    sid, ps, col, x, r, vd = _inputs("sphere", 4, 2, seed=3)
    S = MAX_STROKES + 1
    ps_big = ps[:1].expand(S, ps.shape[1]).contiguous()
    col_big = col[:1].expand(S, 3).contiguous()
    outs = _outputs(x.shape[0], S, dev)
    with pytest.raises(RuntimeError, match="exceeds the static scratch"):
        _call(lib, lib.n3ds_stroke_forward_static, outs, sid, ps_big, col_big, x, r, vd, 0.02, True, True)
    # the entry point is still usable afterwards
    _call(lib, lib.n3ds_stroke_forward_static, _outputs(x.shape[0], 4, dev), sid, ps, col, x, r, vd, 0.02, True,
          True)
    torch.cuda.synchronize()


@pytest.mark.parametrize("kind,color_id,n_color", [("sphere", 3, 27), ("capsule", 2, 12), ("cube", 1, 12)])
def test_static_scratch_colour_fields_and_texcoords(kind, color_id, n_color):
    """The colour-field branches (gradient rgb, SH2, SH3: per-sample colour from the
    view direction and the local point) and the texture-coordinate output read the
    same prepared records: the static entry point gives the workspace entry point's
    alpha, colour, SDF and texcoords, on two calls in a row, and allocates nothing
    (neither torch's allocator nor the device's free memory moves across the calls)."""
    lib = _lib.load()
    dev = torch.device("cuda:0")
    sid, ps, _, x, r, vd = _inputs(kind, 70, 48, seed=21 + color_id)
    P, S = x.shape[0], ps.shape[0]
    col = torch.randn(S, n_color, generator=torch.Generator().manual_seed(5)).to(dev).contiguous()
    want = _outputs(P, S, dev)
    want_tex = torch.full((P, S, 2), float("nan"), device=dev)
    ws = _lib.workspace(lib.n3ds_stroke_workspace_bytes(S), dev)
    _call(lib, lib.n3ds_stroke_forward, want, sid, ps, col, x, r, vd, 0.02, True, True, ws, color_id, want_tex)
    got = [_outputs(P, S, dev) for _ in range(2)]
    got_tex = [torch.full((P, S, 2), float("nan"), device=dev) for _ in range(2)]
    _call(lib, lib.n3ds_stroke_forward_static, got[0], sid, ps, col, x, r, vd, 0.02, True, True, None, color_id,
          got_tex[0])
    torch.cuda.synchronize()
    alloc0, free0 = torch.cuda.memory_allocated(dev), torch.cuda.mem_get_info(dev)[0]
    _call(lib, lib.n3ds_stroke_forward_static, got[1], sid, ps, col, x, r, vd, 0.02, True, True, None, color_id,
          got_tex[1])
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated(dev) == alloc0 and torch.cuda.mem_get_info(dev)[0] == free0
    for outs, tex in zip(got, got_tex):
        for g_, w_ in zip(list(outs) + [tex], list(want) + [want_tex]):
            assert torch.isfinite(g_).all()
            assert rel(g_, w_) < FWD_TOL
