"""HostPipeline: batches uploaded from pinned host memory on a copy stream, overlapped
with the compute of the neighbouring steps, give the same results as running each
step directly: rgb and grad_x bit-identical (per-sample arithmetic in a fixed order),
the stroke-parameter gradients within 1e-6 (their per-CTA partial sums meet in
floating-point atomics, whose order varies from run to run)."""
import pytest
import torch

from helpers import rel
from neural3dstrokes_b200 import scenes
from neural3dstrokes_b200.train import BatchedField, HostPipeline, capture

pytestmark = pytest.mark.gpu


def test_pipelined_steps_match_direct_steps(cuda):
    g = torch.Generator().manual_seed(31)
    sc = [scenes.make_strokes([scenes.ALL_KINDS[int(i)] for i in torch.randint(0, 8, (30,), generator=g)], g)]
    rays = [scenes.make_rays(300, 40, g)]
    field = BatchedField(sc, rays, device=cuda)
    field.g_rgb.normal_()
    ins = [field.x, field.g_rgb]
    outs = [field.rgb, field.grad_shape, field.grad_x]
    graph = capture(field.step, cuda)
    n = 4
    host_in = []
    for i in range(n):
        x = rays[0].x.reshape(-1, 40, 3) + 0.01 * i
        host_in.append([x.contiguous().pin_memory(), (field.g_rgb.cpu() * (1 + i)).pin_memory()])
    host_out = [[torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in outs] for _ in range(n)]
    pipe = HostPipeline(graph, ins, outs, cuda)
    pipe.upload(0, host_in[0])
    for i in range(n):
        if i + 1 < n:
            pipe.upload(i + 1, host_in[i + 1])
        pipe.run(i, host_out[i])
    pipe.synchronize()
    for i in range(n):
        for d, h in zip(ins, host_in[i]):
            d.copy_(h)
        graph.replay()
        torch.cuda.synchronize()
        rgb, gshape, gx = (t.cpu() for t in outs)
        assert torch.equal(host_out[i][0], rgb), i
        assert torch.equal(host_out[i][2], gx), i
        assert rel(host_out[i][1], gshape) < 1e-6, i
