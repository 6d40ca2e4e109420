"""The Model's ray-sampling loop over the fused kernels (neural3dstrokes_b200/sampler.py:
two proposal levels, PropMLP at the default desired resolutions 512 and 2048, then the
stroke level with the samples cast in its kernels) against the float64 oracle.

The loop is checked level by level on its own inputs: each level's resampling against
the oracle's (oracle/stepfun.py, in float32 like the reference) of the previous level's
posts and weights as the kernels produced them, with the slope-scaled bound of the
resampling tests; the proposal density against the oracle network at the level's cast
samples (1e-5); the weights against compute_alpha_weights in float64 (1e-5); and the
stroke level's rgb / opacity / depth against the oracle's render of the final intervals
at the kernels' float32 sample positions (1e-5). End to end the chain amplifies
rounding (a post moved by one float32 ulp moves the next level's fine-grid density),
so the levels are not compared through the whole chain at once."""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

from helpers import FWD_TOL, rel
from neural3dstrokes_b200 import mlp, sampler, scenes, stepfun
from neural3dstrokes_b200.field import render_rays
from oracle import density_net as odn
from oracle import render as orr
from oracle import stepfun as ost
from test_stepfun_gpu import check_posts

pytestmark = pytest.mark.gpu

N_PROP, N_NERF = 64, 32
DIL_BIAS, DIL_MULT = 0.0025, 0.5


def prop_nets(cuda, seed=0):
    nets = []
    for i, res in enumerate((512, 2048)):
        torch.manual_seed(seed + i)
        net = mlp.PropMLP(grid_disired_resolution=res, warp_fn=None, bbox_size=3.0).to(cuda)
        g = torch.Generator(device=cuda).manual_seed(seed + 10 + i)
        with torch.no_grad():
            net.encoder.embeddings.uniform_(-1, 1, generator=g)
            net.density_layer[0].weight.mul_(3.0)
        nets.append(net)
    return nets


def rays(cuda, R, seed=3):
    g = torch.Generator().manual_seed(seed)
    o = F.normalize(torch.randn(R, 3, generator=g), dim=-1) * 1.4
    d = F.normalize(-o + 0.3 * torch.randn(R, 3, generator=g), dim=-1)
    radii = torch.full((R,), 0.5)
    near, far = torch.full((R,), 0.2), torch.full((R,), 3.0)
    return [t.to(cuda) for t in (o, d, radii, near, far)]


def oracle_density(net, coords):
    enc, lay = net.encoder, net.density_layer
    dens, _, _ = odn.forward(coords, enc.embeddings, enc.offsets, float(np.log2(enc.per_level_scale)),
                             enc.base_resolution, lay[0].weight, lay[0].bias, lay[2].weight, lay[2].bias,
                             density_bias=net.density_bias, warp=odn.WARP_SCALE, bbox_size=net.bbox_size)
    return dens


def check_level(s_prev, w_prev, s, t, n, dilation, near, far, jitter):
    """One level's resampling against the oracle's, in float32, on the same inputs."""
    sp, wp = s_prev.detach().cpu().float(), w_prev.detach().cpu().float()
    nr, fr = near.cpu()[:, None], far.cpu()[:, None]
    ref_s, _ = ost.resample_level(sp, wp, n, jitter, True, dilation, 0.0, (0.0, 1.0), nr, fr)
    if dilation > 0:
        sd, wd = ost.max_dilate_weights(sp, wp, dilation, (0.0, 1.0), True)
        sd, wd = sd[..., 1:-1], wd[..., 1:-1]
    else:
        sd, wd = sp, wp
    logits = torch.where(sd[..., 1:] > sd[..., :-1], torch.log(wd), torch.full_like(wd, float("-inf")))
    check_posts(s, ref_s, sd, logits)
    assert torch.allclose(t, s * far[:, None] + (1 - s) * near[:, None], rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("rand", [False, True])
def test_sampling_loop_level_by_level(cuda, rand, monkeypatch):
    R = 256
    o, d, radii, near, far = rays(cuda, R)
    nets = prop_nets(cuda)
    jitter = None
    with monkeypatch.context() as m:
        if rand:  # the same single-jitter draw for every level, fed to both sides
            jitter = torch.rand(R, 1, generator=torch.Generator().manual_seed(5))
            jit_d = jitter.to(cuda)
            m.setattr(stepfun.torch, "rand", lambda *a, **k: jit_d.clone())
        out = sampler.sample_rays(o, d, radii, near, far, nets, N_PROP, N_NERF, DIL_BIAS, DIL_MULT, rand=rand)
    assert len(out.levels) == 2
    assert out.sdist.shape == (R, N_NERF + 1) and out.tdist.shape == (R, N_NERF + 1)

    s_prev = torch.tensor([[0.0, 1.0]], device=cuda).expand(R, 2)
    w_prev = torch.ones(R, 1, device=cuda)
    prod = 1
    for i, lv in enumerate(out.levels + [dict(sdist=out.sdist, tdist=out.tdist)]):
        n = N_PROP if i < 2 else N_NERF
        dilation = (DIL_BIAS + DIL_MULT / prod) if i > 0 else 0.0
        prod *= n
        check_level(s_prev, w_prev, lv["sdist"], lv["tdist"], n, dilation, near, far, jitter)
        if i == 2:
            break
        x, _, _ = orr.cast_rays(lv["tdist"], o, d, radii[:, None])
        dens_ref = oracle_density(nets[i], x.reshape(-1, 3)).reshape(R, n)
        assert rel(lv["density"], dens_ref) < FWD_TOL, (i, rel(lv["density"], dens_ref))
        w_ref = orr.compute_alpha_weights(lv["density"].detach().double().cpu(), lv["tdist"].double().cpu(),
                                          d.double().cpu())[0]
        assert rel(lv["weights"], w_ref) < FWD_TOL
        s_prev, w_prev = lv["sdist"], lv["weights"]

    # the stroke level on the final intervals, samples cast inside the kernels
    g = torch.Generator().manual_seed(9)
    kinds = [scenes.MIXED_PRIMS[int(k)] for k in torch.randint(0, 6, (40,), generator=g)]
    sc = scenes.make_strokes(kinds, g)
    rgb, acc, depth = render_rays(o, d, radii, out.tdist, sc.shape_params.to(cuda), sc.sdf_ids.to(cuda),
                                  sc.color_params.to(cuda), sc.density.to(cuda), 0.02)
    # the oracle at the kernels' own sample positions: cast in float32 in the kernels'
    # operation order (t = (t0 + t1) / 2, x = d t + o, radius = radii t)
    t = (out.tdist[:, :-1] + out.tdist[:, 1:]) / 2
    x = d[:, None, :] * t[..., None]
    x = x + o[:, None, :]
    r = radii[:, None] * t
    td = out.tdist.double().cpu()
    ref = orr.render_strokes(x.double().cpu(), r.double().cpu(), td, d.double().cpu(), sc.shape_params.double(),
                             sc.sdf_ids, sc.color_params.double(), sc.density.double(), 0.02)
    assert rel(rgb, ref[0]) < FWD_TOL and rel(acc, ref[1]) < FWD_TOL
    assert rel(acc * depth, ref[1] * ref[2]) < FWD_TOL


def test_proposal_weights_are_differentiable(cuda):
    """Each proposal level's weights carry the gradient of its own network (the
    interlevel loss trains the proposal networks); the intervals carry none."""
    R = 64
    o, d, radii, near, far = rays(cuda, R)
    nets = prop_nets(cuda)
    out = sampler.sample_rays(o, d, radii, near, far, nets, N_PROP, N_NERF, DIL_BIAS, DIL_MULT)
    assert not out.tdist.requires_grad and not out.levels[1]["sdist"].requires_grad
    loss = out.levels[0]["weights"].square().sum() + out.levels[1]["weights"].square().sum()
    loss.backward()
    for net in nets:
        assert net.encoder.embeddings.grad is not None and float(net.encoder.embeddings.grad.abs().sum()) > 0
        assert float(net.density_layer[0].weight.grad.abs().sum()) > 0


def test_rejects_mismatched_rays(cuda):
    o, d, radii, near, far = rays(cuda, 16)
    nets = prop_nets(cuda)
    with pytest.raises(ValueError):
        sampler.sample_rays(o[:8], d, radii, near, far, nets)
    with pytest.raises(ValueError):
        sampler.sample_rays(o, d, radii[:8], near, far, nets)


def test_without_proposal_samples_the_last_level_samples_the_whole_ray(cuda):
    """num_prop_samples = 0 skips the proposal levels (models.py:137-138): the last
    level dilates (i_level > 0) and resamples the initial single interval, i.e. centred
    samples over [near, far]."""
    R = 8
    o, d, radii, near, far = rays(cuda, R)
    out = sampler.sample_rays(o, d, radii, near, far, prop_nets(cuda), num_prop_samples=0, num_nerf_samples=N_NERF)
    assert out.levels == []
    ref_s, _ = ost.resample_level(torch.tensor([[0.0, 1.0]]).expand(R, 2), torch.ones(R, 1), N_NERF, None, True,
                                  DIL_BIAS + DIL_MULT, 0.0, (0.0, 1.0), near.cpu()[:, None], far.cpu()[:, None])
    assert torch.allclose(out.sdist.cpu(), ref_s, atol=1e-6)
