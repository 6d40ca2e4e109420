"""CPU checks of the ray-sampling loop's host logic (neural3dstrokes_b200/sampler.py):
compute_alpha_weights as render.py:29-48 states it (the float64 oracle's restatement),
and the loop's refusal of host tensors (its resampling and networks are CUDA kernels)."""
import pytest
import torch

from neural3dstrokes_b200 import mlp, sampler
from oracle import render as orr


@pytest.mark.parametrize("opaque", [False, True])
def test_compute_alpha_weights_is_the_references(opaque):
    g = torch.Generator().manual_seed(0)
    R, N = 16, 24
    tdist = torch.sort(torch.rand(R, N + 1, generator=g, dtype=torch.float64) * 4 + 2, -1).values
    dens = torch.rand(R, N, generator=g, dtype=torch.float64) * 3
    dirs = torch.randn(R, 3, generator=g, dtype=torch.float64)
    ours = sampler.compute_alpha_weights(dens, tdist, dirs, opaque)
    ref = orr.compute_alpha_weights(dens, tdist, dirs, opaque)
    for a, b in zip(ours, ref):
        assert torch.allclose(a, b, rtol=1e-14, atol=1e-15)


def test_host_tensors_raise():
    R = 4
    o, d = torch.zeros(R, 3), torch.ones(R, 3)
    with pytest.raises(RuntimeError, match="CUDA"):
        sampler.sample_rays(o, d, torch.ones(R), torch.ones(R), torch.ones(R) * 2,
                            [mlp.PropMLP(grid_disired_resolution=512)])
