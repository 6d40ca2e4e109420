"""CPU checks of the config-scale accuracy harness (oracle/accuracy.py) itself.

The harness runs a field over a whole workload with upstream gradients on a ray
subset only and compares the subset against the float64 oracle. Here the "field" is
a stand-in that computes every output and gradient with the float64 oracle and
stores them in float32, as the CUDA field's buffers are: the harness must then
report errors at float32 rounding level, find no position gradient outside the
subset, and detect a planted mistake (one stroke's gradient row perturbed).
"""

import torch

from neural3dstrokes_b200 import scenes
from neural3dstrokes_b200.field import FieldOptions
from oracle import accuracy
from oracle import render as orr

class OracleField:
    """The BatchedField interface the harness uses, computed by the oracle."""

    def __init__(self, w, plant=None):
        self.w = w
        self.device = torch.device("cpu")
        self.options = FieldOptions()
        self.c_opt = None
        self.bg_value = 1.0
        self.plant = plant
        R = sum(r.n_rays for r in w.rays)
        S = sum(s.n_strokes for s in w.scenes)
        N = w.rays[0].n_samples
        self.rgb, self.acc, self.depth = torch.zeros(R, 3), torch.zeros(R), torch.zeros(R)
        self.g_rgb, self.g_acc, self.g_depth = torch.zeros(R, 3), torch.zeros(R), torch.zeros(R)
        self.grad_x = torch.zeros(R, N, 3)
        self.grad_shape = torch.zeros(S, scenes.PARAM_STRIDE)
        self.grad_color, self.grad_density, self.grad_delta = torch.zeros(S, 3), torch.zeros(S), torch.zeros(S)

    def _each(self, fn):
        r0 = s0 = 0
        for sc, rays in zip(self.w.scenes, self.w.rays):
            fn(sc, rays, r0, r0 + rays.n_rays, s0, s0 + sc.n_strokes)
            r0 += rays.n_rays
            s0 += sc.n_strokes

    def forward(self):
        def one(sc, rays, a, b, c, d):
            d64 = lambda t: t.double()
            rgb, acc, depth = orr.render_strokes(d64(rays.x), d64(rays.radius), d64(rays.tdist), d64(rays.dirs),
                                                 d64(sc.shape_params), sc.sdf_ids, d64(sc.color_params),
                                                 d64(sc.density), self.w.sdf_delta)
            self.rgb[a:b], self.acc[a:b], self.depth[a:b] = rgb.float(), acc.float(), depth.float()
        self._each(one)

    def backward(self):
        def one(sc, rays, a, b, c, d):
            o, _ = accuracy.oracle_scene(sc, rays, self.g_rgb[a:b], self.g_acc[a:b], self.g_depth[a:b],
                                         self.w.sdf_delta, True, True)
            self.grad_x[a:b] = o["x"].float()
            self.grad_shape[c:d] = o["shape"].float()
            self.grad_color[c:d], self.grad_density[c:d] = o["color"].float(), o["density"].float()
            self.grad_delta[c:d] = o["delta"].float()
        self._each(one)
        if self.plant is not None:
            self.grad_shape[self.plant] *= 1.01

    def status(self):
        return 0, 0

def workload():
    g = torch.Generator().manual_seed(3)
    sc = [scenes.make_strokes([scenes.MIXED_PRIMS[i % 6] for i in range(n)], g) for n in (12, 7, 20)]
    rays = [scenes.make_rays(r, 16, g) for r in (40, 25, 33)]
    return scenes.Workload("three small scenes", sc, rays)

def test_subset_indices():
    idx = accuracy.ray_subset(100, 7)
    assert idx[0] == 0 and idx[-1] == 99 and idx.numel() == 7
    assert accuracy.ray_subset(5, 32).tolist() == [0, 1, 2, 3, 4]

def test_harness_reports_float32_rounding_for_an_exact_field():
    w = workload()
    res = accuracy.subset_accuracy(OracleField(w), w, rays_per_scene=6)
    assert res["ok"], res
    assert res["grad_x_nonzero_outside_subset"] == 0
    assert max(res["vs_fp64_oracle"].values()) < 1e-6, res

def test_harness_detects_a_planted_gradient_error():
    w = workload()
    # the planted error sits in the oracle-backed stand-in, never in the product
    fld = OracleField(w, plant=(13, 0))  # stroke 1 of scene 1, its scale slot, 1 % off
    res = accuracy.subset_accuracy(fld, w, rays_per_scene=6)
    assert not res["ok"] and res["vs_fp64_oracle"]["grad_shape"] > 1e-4, res

class PortRef:
    """A stand-in for the reference extension with its four operators' signatures
    (bindings.cpp:6-11), computed by the oracle's float32 port on the host."""

    def stroke_forward(self, a, c, sdf, tex, x, r, vd, ps, cp, sid, cid, delta, lap, inv):
        from oracle import strokefield as sf
        aa, cc = sf.stroke_forward(x, r, ps, cp, sid, delta, lap, inv)
        a.copy_(aa)
        c.copy_(cc)

    def compose_forward(self, dens, col, alphas, colors, dp):
        from oracle import strokefield as sf
        d, c = sf.compose_forward(alphas, colors, dp)
        dens.copy_(d)
        col.copy_(c)

    def compose_backward(self, ga, gc, gdp, gd, gcol, alphas, colors, dp):
        from oracle import strokefield as sf
        a, c, p = sf.compose_backward_compat(gd, gcol, alphas, colors, dp)
        ga += a
        gc += c
        gdp += p

    def stroke_backward(self, gs, gcol, gx, ga, gc, gsdf, x, r, vd, a, ps, cp, sid, cid, delta, lap, inv):
        from oracle import strokefield as sf
        s_, c_, x_ = sf.stroke_backward_compat(ga, gc, x, r, a, ps, cp, sid, delta, lap, inv)
        gs += s_
        gcol += c_
        gx += x_

def test_harness_reference_op_branch_runs_on_host():
    """The reference-op comparison's plumbing (ray chunks, per-group calls, grad_x
    layout) with the port standing in for the extension: its forward agrees with the
    exact stand-in field to float32 rounding."""
    w = workload()
    res = accuracy.subset_accuracy(OracleField(w), w, rays_per_scene=5, ref=PortRef())
    vr = res["vs_reference_op"]
    assert isinstance(vr, dict) and set(vr["compat_gradients"]) >= {"grad_shape", "grad_color", "grad_x"}
    assert max(vr["forward"].values()) < 1e-5, vr
    cmp = accuracy.plain_op_compare(OracleField(w), w, PortRef())
    assert cmp["calls"] == 3 and max(v for k, v in cmp["compat_errors"].items() if not k.startswith("grad")) < 1e-5
