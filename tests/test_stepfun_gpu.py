"""Proposal-resampling kernels (n3ds_max_dilate_weights / n3ds_sample_intervals /
n3ds_resample_intervals) against the reference's own outputs (stepfun golden
vectors) and, at other sizes, against the oracle run in float32 like the reference
(its eps = finfo(float32).eps enters the pdf of zero-width bins).

Tolerances. Dilated posts exact, dilated weights 1e-5 relative. Fence posts: the
inverse CDF turns a CDF difference dc into dc * width / weight of the bin it lands
in, so float32 cumulative sums summed in another order (about 1e-6 here) move a post
by up to dc times the steepest slope of its ray: each ray gets 2e-6 + 4e-6 * max over
its weighted bins of width / weight, and 99% of all posts must also be within 5e-6."""
import os

import numpy as np
import pytest
import torch

from helpers import rel
from oracle import stepfun as ost
from neural3dstrokes_b200 import stepfun

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "stepfun_golden.npz")


@pytest.fixture(scope="module")
def gold():
    d = np.load(GOLD)
    return {k: torch.from_numpy(np.asarray(d[k])) for k in d.files}


def check_posts(s, s_ref, t, logits):
    """Per-ray slope-scaled bound (see the module docstring)."""
    s, s_ref, t = s.cpu().double(), s_ref.cpu().double(), t.cpu().double()
    w = torch.softmax(logits.cpu().double(), -1)
    width = t[..., 1:] - t[..., :-1]
    slope = torch.where(w > 0, width / w.clamp_min(1e-300), torch.zeros_like(w)).amax(-1, keepdim=True)
    err = (s - s_ref).abs()
    assert torch.all(err <= 2e-6 + 4e-6 * slope), float((err - 4e-6 * slope).max())
    assert float((err <= 5e-6).double().mean()) >= 0.99


def test_dilation_matches_reference(cuda, gold):
    td, wd = stepfun.max_dilate_weights(gold["t"].to(cuda), gold["w"].to(cuda), float(gold["dilation"]),
                                        domain=(0.0, 1.0), renormalize=True)
    assert torch.equal(td.cpu(), gold["t_dilate"])
    assert rel(wd, gold["w_dilate"]) < 1e-5


@pytest.mark.parametrize("name,single", [("det", True), ("single", True), ("multi", False)])
def test_sampling_matches_reference(cuda, gold, name, single, monkeypatch):
    sd = gold["t_dilate"][..., 1:-1].to(cuda)
    if name != "det":  # feed the reference's recorded draws through the module's torch.rand
        jit = gold["jit_" + name].to(cuda)
        monkeypatch.setattr(stepfun.torch, "rand", lambda *a, **k: jit.clone())
    s = stepfun.sample_intervals(name != "det", sd, gold["logits"].to(cuda), 32, single_jitter=single,
                                 domain=(0.0, 1.0))
    check_posts(s, gold["s_" + name], sd, gold["logits"])


def test_fused_level_matches_reference(cuda, gold, monkeypatch):
    s, t = stepfun.resample_intervals(gold["t"].to(cuda), gold["w"].to(cuda), 32, rand=False,
                                      dilation=float(gold["dilation"]))
    assert t is None
    check_posts(s, gold["s_det"], gold["t_dilate"][..., 1:-1], gold["logits"])
    jit = gold["jit_level0"].to(cuda)
    monkeypatch.setattr(stepfun.torch, "rand", lambda *a, **k: jit.clone())
    R = jit.shape[0]
    s0 = torch.tensor([0.0, 1.0], device=cuda).expand(R, 2).contiguous()
    s1, t1 = stepfun.resample_intervals(s0, torch.ones(R, 1, device=cuda), 64, rand=True, single_jitter=True,
                                        near=gold["near"].to(cuda), far=gold["far"].to(cuda))
    assert (s1.cpu() - gold["s_level0"]).abs().max() < 5e-6
    assert rel(t1, gold["t_level0"]) < 1e-6


def _case(R, M, seed, zero_frac=0.2, dup_frac=0.05):
    """float32 step functions on [0, 1]: some zero-width bins (dup_frac) and zero
    weights (zero_frac), weights renormalised."""
    g = torch.Generator().manual_seed(seed)
    steps = torch.rand(R, M, generator=g) + 0.02
    if M > 2:
        steps[torch.rand(R, M, generator=g) < dup_frac] = 0.0
    steps[:, 0] += 0.1
    t = torch.cat([torch.zeros(R, 1), torch.cumsum(steps, -1)], -1)
    t = t / t[:, -1:]
    w = torch.rand(R, M, generator=g) ** 2 + 0.02
    w[torch.rand(R, M, generator=g) < zero_frac] = 0.0
    w[:, 0] += 1e-3
    return t, w / w.sum(-1, keepdim=True)


@pytest.mark.parametrize("R,M,N,dilation,padding,single", [
    (37, 1, 2, 0.0, 0.0, True), (64, 5, 33, 0.0, 0.01, False), (200, 64, 64, 0.0103, 0.0, True),
    (96, 130, 128, 0.004, 0.0, False), (33, 64, 32, 0.3, 0.0, True)])
def test_fused_level_matches_oracle(cuda, R, M, N, dilation, padding, single, monkeypatch):
    t, w = _case(R, M, seed=R + M)
    g = torch.Generator().manual_seed(N)
    jit = torch.rand(R, 1 if single else N, generator=g)
    near = 1.0 + torch.rand(R, 1, generator=g)
    far = near + 2.0
    ref_s, _ = ost.resample_level(t, w, N, jit, single, dilation, padding, (0.0, 1.0), near, far)
    jit_d = jit.to(cuda)
    monkeypatch.setattr(stepfun.torch, "rand", lambda *a, **k: jit_d.clone())
    s, tt = stepfun.resample_intervals(t.to(cuda), w.to(cuda), N, rand=True, single_jitter=single,
                                       dilation=dilation, resample_padding=padding, near=near.to(cuda),
                                       far=far.to(cuda))
    if dilation > 0:
        sd, wd = ost.max_dilate_weights(t, w, dilation, (0.0, 1.0), True)
        sd, wd = sd[..., 1:-1], wd[..., 1:-1]
    else:
        sd, wd = t, w
    logits = torch.where(sd[..., 1:] > sd[..., :-1], torch.log(wd + padding), torch.full_like(wd, float("-inf")))
    check_posts(s, ref_s, sd, logits)
    # tdist = s_to_t(s) of the kernel's own posts (the identity warp, coord.py:96-99)
    nd, fd = near.to(cuda), far.to(cuda)
    assert torch.allclose(tt, s * fd + (1 - s) * nd, rtol=1e-6, atol=1e-6)
    assert torch.all(s[..., 1:] >= s[..., :-1])


def test_batched_shapes_and_dilation_sizes(cuda):
    t, w = _case(24, 16, seed=3)
    t4, w4 = t.reshape(2, 3, 4, 17).to(cuda), w.reshape(2, 3, 4, 16).to(cuda)
    td, wd = stepfun.max_dilate_weights(t4, w4, 0.01, domain=(0.0, 1.0), renormalize=True)
    assert td.shape == (2, 3, 4, 49) and wd.shape == (2, 3, 4, 48)
    rtd, rwd = ost.max_dilate_weights(t, w, 0.01, (0.0, 1.0), True)
    assert torch.equal(td.reshape(24, 49).cpu(), rtd)
    assert rel(wd.reshape(24, 48), rwd) < 1e-5
    s = stepfun.sample_intervals(False, t4, torch.log(w4), 9)
    assert s.shape == (2, 3, 4, 10)


def test_rejects_bad_arguments(cuda):
    t = torch.linspace(0, 1, 5, device=cuda)[None]
    with pytest.raises(ValueError):
        stepfun.sample_intervals(False, t, torch.zeros(1, 4, device=cuda), 1)
    with pytest.raises(ValueError):
        stepfun.max_dilate_weights(t, torch.zeros(1, 5, device=cuda), 0.1)
    with pytest.raises(RuntimeError):
        stepfun.max_dilate_weights(t.cpu(), torch.zeros(1, 4), 0.1)
    with pytest.raises(RuntimeError):  # beyond the kernel's bin limit: a clear library error
        stepfun.max_dilate_weights(torch.linspace(0, 1, 3000, device=cuda)[None], torch.ones(1, 2999, device=cuda),
                                   0.1)
