"""Failure paths of the fused stroke field, each made without faulting the GPU:

- a NaN stroke parameter: every sample it may touch evaluates it (NaN culling bounds
  never exclude a stroke), so the rays come out NaN, as through the reference op; the
  status word stays 0 and both passes return;
- an unsupported sdf_id written into the device array after the host checks: the
  prep kernel sets ST_BAD_KIND (bit 1) and the stroke evaluates to NaN, never to a
  silently wrong value;
- the bounded wait of the stroke staging barrier: with the staging copies withheld
  (test_stall_staging, no copy left in flight) and a 50 us limit every wait runs out,
  the kernels report ST_WAIT_TIMEOUT (bit 2) and return, and the context stays usable
  for the next, normal call.
"""
import pytest
import torch

from helpers import FWD_TOL, oracle_forward, rel, small_workload
from neural3dstrokes_b200.field import FieldOptions
from neural3dstrokes_b200.train import BatchedField

pytestmark = pytest.mark.gpu

ST_BAD_KIND, ST_WAIT_TIMEOUT = 1, 2


def field_of(sc, rays, dev, options=None):
    f = BatchedField([sc], [rays], options=options, device=dev)
    g = torch.Generator().manual_seed(2)
    f.g_rgb.copy_(torch.randn(rays.n_rays, 3, generator=g))
    f.g_acc.copy_(torch.randn(rays.n_rays, generator=g))
    return f


def test_nan_parameter_gives_nan_rays_and_status_zero(cuda):
    sc, rays = small_workload("mixed", n_strokes=24, n_rays=64, n_samples=48, seed=1)
    sc.shape_params[5, 0] = float("nan")
    f = field_of(sc, rays, cuda)
    f.forward()
    f.backward()
    torch.cuda.synchronize()
    st, _ = f.status()
    assert st == 0
    assert bool(torch.isnan(f.rgb).all()) and bool(torch.isnan(f.acc).all())
    assert bool(torch.isnan(f.grad_shape).any())


def test_unsupported_sdf_id_in_device_memory_sets_bad_kind(cuda):
    sc, rays = small_workload("mixed", n_strokes=24, n_rays=64, n_samples=48, seed=2)
    f = field_of(sc, rays, cuda)
    good = f.sdf_ids[7].clone()
    f.sdf_ids[7] = 0xC5  # base 12: no such primitive
    f.forward()
    f.backward()
    torch.cuda.synchronize()
    st, _ = f.status()
    assert st & ST_BAD_KIND
    assert bool(torch.isnan(f.rgb).all())
    # restored: the next forward is clean and right
    f.sdf_ids[7] = good
    f.forward()
    torch.cuda.synchronize()
    st, _ = f.status()
    assert st == 0
    rgb_r, acc_r, _ = oracle_forward(sc, rays)
    assert rel(f.rgb, rgb_r) < FWD_TOL and rel(f.acc, acc_r) < FWD_TOL


@pytest.mark.parametrize("schedule", ["segments", "runs"])
def test_bounded_wait_runs_out_and_reports(cuda, schedule):
    sc, rays = small_workload("every", n_strokes=40, n_rays=96, n_samples=64, seed=3)
    stalled = field_of(sc, rays, cuda, FieldOptions(schedule=schedule, wait_limit_us=50, test_stall_staging=True))
    stalled.forward()
    torch.cuda.synchronize()
    st, _ = stalled.status()
    assert st & ST_WAIT_TIMEOUT
    stalled.forward()
    stalled.backward()
    torch.cuda.synchronize()
    st, _ = stalled.status()
    assert st & ST_WAIT_TIMEOUT
    # the context is fine: a normal call on the same device right after
    ok = field_of(sc, rays, cuda, FieldOptions(schedule=schedule))
    ok.forward()
    ok.backward()
    torch.cuda.synchronize()
    st, _ = ok.status()
    assert st == 0
    rgb_r, acc_r, _ = oracle_forward(sc, rays)
    assert rel(ok.rgb, rgb_r) < FWD_TOL and rel(ok.acc, acc_r) < FWD_TOL


def test_base_hint_that_leaves_out_a_present_base_is_reported(cuda):
    """The base hint is checked on the device: a stroke whose base the hint leaves out
    sets ST_BAD_KIND and evaluates to NaN (here a cubic Bezier under a hint of the
    common primitives, which also selects their specialised forward)."""
    sc, rays = small_workload("mixed", n_strokes=24, n_rays=64, n_samples=48, seed=4)
    assert "cubic_bezier" in sc.kinds
    f = field_of(sc, rays, cuda)
    common = sum(1 << b for b in (0, 1, 2, 4, 7, 8))
    f.c_strokes.base_mask = common
    f.forward()
    torch.cuda.synchronize()
    st, _ = f.status()
    assert st & ST_BAD_KIND
    assert bool(torch.isnan(f.rgb).any())
