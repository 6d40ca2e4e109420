"""Accuracy of the fused stroke field at every benchmark workload's own shape.

Each test builds the workload at full size (all rays, all strokes: several
shared-memory stages per scene, stroke-block masks, uneven scenes handed between
persistent CTAs, exactly as the bench runs it) and checks it with the harness of
oracle/accuracy.py:
- every output and gradient against the float64 oracle on a fixed subset of
  evenly spaced rays per scene (upstream gradients zero elsewhere, so the
  whole-workload gradients are the subset's), forward <= 1e-5 and gradients <= 1e-4
  (normwise, worst scene);
- the same subset through the reference CUDA op (oracle/_ref): forward within
  1e-5 of it (or no further from it than it is from float64), compat gradients
  within 1e-4 on workloads without quadratic Beziers;
- the 16-scene workload against 16 sequential reference-op calls over all rays;
- the spline workload's 32-ray x 8-stroke slice against float64 central finite
  differences.
"""
import pytest
import torch

from neural3dstrokes_b200 import scenes
from neural3dstrokes_b200.train import BatchedField
from oracle import accuracy, cpu_port

pytestmark = pytest.mark.gpu

# evenly spaced rays per scene for the float64 oracle (a few seconds of host work each)
SUBSET = {0: 64, 1: 48, 2: 16, 3: 12, 4: 6}


def make_field(w, dev):
    return BatchedField(w.scenes, w.rays, w.sdf_delta, w.use_laplace, w.inv_scale_radius, device=dev)


@pytest.mark.parametrize("cfg", [0, 1, 2, 3, 4])
def test_config_accuracy_at_full_size(cuda, cfg):
    w = scenes.config(cfg)
    field = make_field(w, cuda)
    res = accuracy.subset_accuracy(field, w, SUBSET[cfg], ref=cpu_port.reference_extension())
    print(cfg, res)
    assert res["status_word"] == 0
    assert res["grad_x_nonzero_outside_subset"] == 0
    assert res["ok"], res["vs_fp64_oracle"]
    if isinstance(res["vs_reference_op"], dict):
        assert res["vs_reference_op"]["ok"], res["vs_reference_op"]


def test_config3_matches_16_sequential_plain_op_calls(cuda):
    ref = cpu_port.reference_extension()
    if ref is None:
        pytest.skip("reference extension not built (oracle/_ref)")
    w = scenes.config(3)
    assert len(w.scenes) == 16
    field = make_field(w, cuda)
    res = accuracy.plain_op_compare(field, w, ref)
    print(res)
    assert res["ok"], res


def test_config2_gradients_match_fp64_finite_differences(cuda):
    w = scenes.config(2)
    res = accuracy.fd_slice(w.scenes[0], w.rays[0], n_rays=32, n_strokes=8, device=cuda)
    print(res)
    assert res["rays"] == 32 and res["strokes"] == 8
    assert set(res["stroke_kinds"]) == {"quadratic_bezier", "cubic_bezier"}
    # the oracle itself against its finite differences first, then the fused kernels
    assert max(res["oracle_autograd_vs_fd"].values()) < 1e-6, res
    assert res["ok"], res["fused_vs_fd"]
