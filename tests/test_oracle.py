"""CPU checks of the oracle itself, before it is trusted as the parity reference.

- layouts: sdf_ids, parameter counts and clamp ranges agree with what the reference
  get_stroke produces (tests/golden/layouts.json, written from the reference's own
  strokes.py by tests/golden/make_golden.py);
- volume rendering: the restatement reproduces the reference render.py outputs
  (tests/golden/render_golden.npz, float64) to 1e-12;
- strokelib: the float32 port reproduces the reference CUDA op's outputs
  (tests/golden/strokelib_golden.npz, recorded on a B200 from oracle/_ref) to 1e-5
  forward and 1e-4 for the compat backward;
- autograd of the float64 oracle agrees with central finite differences;
- the known divergences of the reference backward are present in the compat
  restatement (and absent in the exact adjoint).
"""
import json
import math
import os

import numpy as np
import pytest
import torch

from neural3dstrokes_b200 import scenes
from oracle import render as orr
from oracle import strokefield as sf

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    a, b = torch.as_tensor(a).double(), torch.as_tensor(b).double()
    return float((a - b).abs().max() / max(float(b.abs().max()), 1e-30))


def test_layouts_match_reference_get_stroke():
    lay = json.load(open(os.path.join(GOLDEN, "layouts.json")))
    for name, sid in scenes.SDF_ID.items():
        assert lay[name]["sdf_id"] == sid, name
        assert lay[name]["dim_shape"] == scenes.N_PARAMS[name] == sf.num_shape_params(sid), name
        lo, hi = scenes.param_ranges(name)
        for j, (a, b) in enumerate(lay[name]["shape_ranges"]):
            assert (a if a is not None else -math.inf) == pytest.approx(lo[j]), (name, j)
            assert (b if b is not None else math.inf) == pytest.approx(hi[j]), (name, j)
    for name, v in lay.items():  # every reference shape type, implemented or not
        assert sf.num_shape_params(v["sdf_id"]) == v["dim_shape"], name
        assert v["dim_color"] == 3


def test_render_restatement_matches_reference_render():
    z = np.load(os.path.join(GOLDEN, "render_golden.npz"))
    t = {k: torch.from_numpy(z[k]) for k in z.files}
    w, a, tr = orr.compute_alpha_weights(t["density"], t["tdist"], t["dirs"])
    assert rel(w, t["weights"]) < 1e-12 and rel(a, t["alpha"]) < 1e-12 and rel(tr, t["trans"]) < 1e-12
    wo, _, _ = orr.compute_alpha_weights(t["density"], t["tdist"], t["dirs"], opaque_background=True)
    assert rel(wo, t["weights_opaque"]) < 1e-12
    rgb, depth, acc = orr.volumetric_rendering(t["rgbs"], w, t["tdist"], t["bg"])
    assert rel(rgb, t["rgb"]) < 1e-12 and rel(depth, t["depth"]) < 1e-12 and rel(acc, t["acc"]) < 1e-12
    rgb, depth, acc = orr.volumetric_rendering(t["rgbs"], wo, t["tdist"], 1.0)
    assert rel(rgb, t["rgb_opaque"]) < 1e-12 and rel(depth, t["depth_opaque"]) < 1e-12


STROKELIB = os.path.join(GOLDEN, "strokelib_golden.npz")
KINDS = scenes.EVERY_KIND  # every shape type of the reference get_stroke


@pytest.mark.skipif(not os.path.exists(STROKELIB), reason="strokelib golden not recorded yet")
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("mode", ["11", "00"])
def test_port_matches_reference_strokelib(kind, mode):
    z = np.load(STROKELIB)
    tag = f"{kind}_{mode}"
    g = lambda k: torch.from_numpy(z[f"{tag}/{k}"])
    lap, inv = mode[0] == "1", mode[1] == "1"
    sid = int(z[f"{tag}/sdf_id"])
    delta = float(z[f"{tag}/delta"]) if f"{tag}/delta" in z.files else 0.02
    # Bezier tubes: the float32 closest-point solve differs in rounding between the
    # CPU port and the CUDA op (and from float64) at rare near-tie / near-degenerate
    # samples; the linear soft step (slope 0.5 / (delta r) = 25) amplifies that, so
    # their alpha and SDF values are held to 1e-4
    tol = 1e-4 if kind in ("quadratic_bezier", "cubic_bezier", "catmull_rom") else 1e-5
    a, c, sdf = sf.stroke_forward(g("x"), g("radius"), g("shape"), g("color"), sid, delta, lap, inv, return_sdf=True)
    assert rel(a, g("alpha")) < tol and rel(c, g("colors")) == 0.0 and rel(sdf, g("sdf")) < tol
    a64, _, sdf64 = sf.stroke_forward(g("x").double(), g("radius").double(), g("shape").double(),
                                      g("color").double(), sid, delta, lap, inv, return_sdf=True)
    assert rel(g("alpha"), a64) < tol and rel(g("sdf"), sdf64) < tol
    if kind == "quadratic_bezier":
        return  # the reference quadratic-Bezier adjoint is not restated (known divergence)
    gs, gc, gx = sf.stroke_backward_compat(g("g_alpha").double(), g("g_color").double(), g("x").double(),
                                           g("radius").double(), g("alpha").double(), g("shape").double(),
                                           g("color").double(), sid, delta, lap, inv)
    assert rel(gs, g("grad_shape")) < 1e-4, rel(gs, g("grad_shape"))
    assert rel(gc, g("grad_color")) < 1e-5
    assert rel(gx, g("grad_x")) < 1e-4, rel(gx, g("grad_x"))


@pytest.mark.skipif(not os.path.exists(STROKELIB), reason="strokelib golden not recorded yet")
def test_compose_matches_reference_strokelib():
    z = np.load(STROKELIB)
    g = lambda k: torch.from_numpy(z[f"compose/{k}"])
    d, c = sf.compose_forward(g("alphas"), g("colors"), g("density_params"))
    assert rel(d, g("density")) < 1e-6 and rel(c, g("color")) < 1e-6
    ga, gc, gd = sf.compose_backward_compat(g("g_density").double(), g("g_color").double(), g("alphas").double(),
                                            g("colors").double(), g("density_params").double())
    assert rel(ga, g("grad_alphas")) < 1e-4 and rel(gc, g("grad_colors")) < 1e-5
    assert rel(gd, g("grad_density_params")) < 1e-5


def _fd_check(fn, inputs, idx, eps=1e-6, n=6, seed=0):
    """Central differences of scalar fn at n random coordinates of inputs[idx]."""
    g = torch.Generator().manual_seed(seed)
    x = inputs[idx]
    xs = [t.detach().clone() for t in inputs]
    xs[idx] = x.detach().clone().requires_grad_(True)
    grad, = torch.autograd.grad(fn(*xs), [xs[idx]])
    flat = torch.randperm(x.numel(), generator=g)[:n]
    for k in flat.tolist():
        p = [t.detach().clone().contiguous() for t in inputs]
        m = [t.detach().clone().contiguous() for t in inputs]
        p[idx].view(-1)[k] += eps
        m[idx].view(-1)[k] -= eps
        fd = (fn(*p) - fn(*m)) / (2 * eps)
        gk = float(grad.reshape(-1)[k])
        assert abs(float(fd) - gk) <= 1e-5 * max(1.0, abs(float(fd))), (k, float(fd), gk)


@pytest.mark.parametrize("kind", KINDS)
def test_oracle_autograd_matches_finite_differences(kind):
    g = torch.Generator().manual_seed(21)
    sc = scenes.make_strokes([kind] * 6, g)
    rays = scenes.make_rays(12, 24, g)
    sid = scenes.SDF_ID[kind]
    gr = torch.randn(12, 3, generator=g, dtype=torch.float64)
    # depth = D / acc is ill-conditioned on rays that barely touch a stroke: weight it
    # only where the ray is at least 5% opaque
    _, acc0, _ = orr.render_strokes(rays.x.double(), rays.radius.double(), rays.tdist.double(),
                                    rays.dirs.double(), sc.shape_params.double(), sc.sdf_ids,
                                    sc.color_params.double(), sc.density.double(), 0.05)
    dmask = (acc0 > 0.05).double()

    def f(x, sp, col, den):
        rgb, acc, depth = orr.render_strokes(x, rays.radius.double(), rays.tdist.double(), rays.dirs.double(), sp,
                                             sc.sdf_ids, col, den, 0.05)
        return (rgb * gr).sum() + acc.sum() + 0.1 * (depth * dmask).sum()

    inputs = [rays.x.double(), sc.shape_params[:, :16].double(), sc.color_params.double(), sc.density.double()]
    _fd_check(f, inputs, 0)
    _fd_check(f, inputs, 2)
    _fd_check(f, inputs, 3)
    # only the slots the primitive uses
    npar = sf.num_shape_params(sid)

    def fs(part):
        sp = torch.cat([part, inputs[1][:, npar:]], 1)
        return f(inputs[0], sp, inputs[2], inputs[3])
    _fd_check(lambda p: fs(p), [inputs[1][:, :npar].contiguous()], 0, n=10)


def test_known_divergences_of_reference_backward():
    """Divergences of the reference adjoint (exact = float64 autograd):
    cube exterior 2*max(q,0); scale gradient missing the soft-step-width term under
    inv_scale_radius; cubic Bezier gradient scaled by 2 dL/dSDF |v|; compose colour
    -> alpha gradient exact only for one non-zero stroke."""
    g = torch.Generator().manual_seed(3)

    def compare(kind, inv):
        sc = scenes.make_strokes([kind] * 8, g)
        rays = scenes.make_rays(40, 16, g)
        sid = scenes.SDF_ID[kind]
        ps = sc.shape_params[:, :sf.num_shape_params(sid)].double()
        x = rays.x.reshape(-1, 3).double()
        r = rays.radius.reshape(-1).double()
        ga = torch.randn(x.shape[0], 8, generator=g, dtype=torch.float64)
        xg, pg = x.clone().requires_grad_(True), ps.clone().requires_grad_(True)
        a, _ = sf.stroke_forward(xg, r, pg, sc.color_params.double(), sid, 0.05, True, inv)
        gx, gp = torch.autograd.grad((a * ga).sum(), [xg, pg])
        cp, _, cx = sf.stroke_backward_compat(ga, torch.zeros(x.shape[0], 8, 3, dtype=torch.float64), x, r,
                                              a.detach(), ps, sc.color_params.double(), sid, 0.05, True, inv)
        return rel(cp, gp), rel(cx, gx)

    assert max(compare("sphere", False)) < 1e-9          # reference exact here
    assert max(compare("octahedron", False)) < 1e-9
    assert compare("sphere", True)[0] > 1e-3             # scale through the soft-step width
    assert compare("cube", False)[1] > 1e-3              # 2*max(q,0) exterior
    assert compare("cubic_bezier", False)[1] > 1e-3      # 2 dL/dSDF |v| scaling
    al = torch.rand(50, 6, generator=g, dtype=torch.float64) * 0.9
    co = torch.rand(50, 6, 3, generator=g, dtype=torch.float64)
    dp = torch.rand(6, generator=g, dtype=torch.float64)
    gc = torch.randn(50, 3, generator=g, dtype=torch.float64)
    ga_ref, _, _ = sf.compose_backward_compat(torch.zeros(50, dtype=torch.float64), gc, al, co, dp)
    alg = al.clone().requires_grad_(True)
    _, c = sf.compose_forward(alg, co, dp)
    ga_ex, = torch.autograd.grad((c * gc).sum(), [alg])
    assert rel(ga_ref, ga_ex) > 1e-3                     # colour -> alpha approximation


def test_compose_modes_restatement_matches_reference_torch():
    """oracle.compose_mode against the reference's own torch compositing modes
    (strokes.py:390-417), run in float64 by tests/golden/make_golden.py --compose."""
    z = np.load(os.path.join(GOLDEN, "compose_modes_golden.npz"))
    for C in (1, 3):
        t = {k: torch.from_numpy(z[f"c{C}/{k}"]) for k in ("alphas", "colors", "density_params", "g_density",
                                                         "g_color")}
        for mode in ("max", "max_density_weighted", "softmax", "softmax_density_weighted"):
            a, c, d = (t[k].clone().requires_grad_(True) for k in ("alphas", "colors", "density_params"))
            dens, col = sf.compose_mode(a, c, d, mode)
            ((dens * t["g_density"]).sum() + (col * t["g_color"]).sum()).backward()
            ref = lambda k: torch.from_numpy(z[f"c{C}/{mode}/{k}"])
            assert rel(dens, ref("density")) < 1e-12 and rel(col, ref("color")) < 1e-12, mode
            assert rel(a.grad, ref("grad_alphas")) < 1e-12 and rel(c.grad, ref("grad_colors")) < 1e-12, mode
            assert rel(d.grad, ref("grad_density_params")) < 1e-12, mode


@pytest.mark.skipif(not os.path.exists(STROKELIB), reason="strokelib golden not recorded yet")
@pytest.mark.parametrize("kind", ["sphere", "obb", "capsule", "cubic_bezier"])
@pytest.mark.parametrize("cid", [1, 2, 3])
def test_color_fields_match_reference_strokelib(kind, cid):
    """Colour fields (gradient rgb, SH2, SH3) of the restatement against the reference op:
    colours and the colour-parameter gradients (the reference formulas)."""
    z = np.load(STROKELIB)
    tag = f"{kind}_c{cid}"
    if f"{tag}/alpha" not in z.files:
        pytest.skip("colour-field golden vectors not recorded")
    g = lambda k: torch.from_numpy(z[f"{tag}/{k}"]).double()
    sid = int(z[f"{tag}/sdf_id"])
    a, c = sf.stroke_forward(g("x"), g("radius"), g("shape"), g("color"), sid, 0.02, True, True, color_id=cid,
                             viewdir=g("viewdir"))
    assert rel(c, g("colors")) < 1e-5 and rel(a, g("alpha")) < 1e-4
    gs, gc, gx = sf.stroke_backward_compat(g("g_alpha"), g("g_color"), g("x"), g("radius"), g("alpha"), g("shape"),
                                           g("color"), sid, 0.02, True, True, color_id=cid, viewdir=g("viewdir"))
    assert rel(gc, g("grad_color")) < 1e-5, rel(gc, g("grad_color"))
    assert rel(gs, g("grad_shape")) < 1e-4 and rel(gx, g("grad_x")) < 1e-4


@pytest.mark.skipif(not os.path.exists(STROKELIB), reason="strokelib golden not recorded yet")
@pytest.mark.parametrize("kind", ["sphere", "ellipsoid", "cube", "aabb", "roundbox", "capsule", "scapsule", "line",
                                  "octahedron"])
def test_texcoord_matches_reference_strokelib(kind):
    """Texture coordinates of the restatement against the reference op (away from the
    v seam, where atan2 jumps between 0 and 1)."""
    z = np.load(STROKELIB)
    tag = f"{kind}_tex"
    if f"{tag}/texcoord" not in z.files:
        pytest.skip("texcoord golden vectors not recorded")
    g = lambda k: torch.from_numpy(z[f"{tag}/{k}"]).double()
    sid = int(z[f"{tag}/sdf_id"])
    *_, tex = sf.stroke_forward(g("x"), g("radius"), g("shape"), g("color"), sid, 0.02, True, True,
                                return_texcoord=True)
    ref = g("texcoord")
    d = (tex - ref).abs()
    d = torch.minimum(d, (1.0 - d).abs())  # the seam of v
    assert float(d.max()) < 1e-5, float(d.max())


def test_cast_rays_restatement_matches_reference_cast_rays():
    """oracle.render.cast_rays against the reference cast_rays' float32 outputs
    (tests/golden/cast_golden.npz, render.py:5-26): bit for bit."""
    z = np.load(os.path.join(GOLDEN, "cast_golden.npz"))
    t = lambda k: torch.from_numpy(z[k])
    coords, radius, tm = orr.cast_rays(t("tdist"), t("origins"), t("directions"), t("radii"))
    assert torch.equal(coords, t("coords")) and torch.equal(radius, t("radius")) and torch.equal(tm, t("t"))
