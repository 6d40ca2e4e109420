"""The proposal-resampling oracle (oracle/stepfun.py) against the reference's own
outputs (tests/golden/stepfun_golden.npz, made by importing source/utils/stepfun.py).
CPU only; the CUDA kernels are checked in test_stepfun_gpu.py."""
import os

import numpy as np
import pytest
import torch

from oracle import stepfun as ost

GOLD = os.path.join(os.path.dirname(__file__), "golden", "stepfun_golden.npz")


@pytest.fixture(scope="module")
def gold():
    d = np.load(GOLD)
    return {k: torch.from_numpy(np.asarray(d[k])) for k in d.files}


def test_dilation_matches_reference(gold):
    td, wd = ost.max_dilate_weights(gold["t"], gold["w"], float(gold["dilation"]), domain=(0.0, 1.0),
                                    renormalize=True)
    assert torch.equal(td, gold["t_dilate"])
    assert torch.allclose(wd, gold["w_dilate"], rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("name,single", [("det", True), ("single", True), ("multi", False)])
def test_sampling_matches_reference(gold, name, single):
    sd = gold["t_dilate"][..., 1:-1]
    jit = None if name == "det" else gold["jit_" + name]
    s = ost.sample_intervals(jit, sd, gold["logits"], 32, single_jitter=single, domain=(0.0, 1.0))
    assert torch.allclose(s, gold["s_" + name], rtol=0, atol=2e-6)


def test_level_chain_matches_reference(gold):
    s, _ = ost.resample_level(gold["t"], gold["w"], 32, None, True, float(gold["dilation"]), 0.0, (0.0, 1.0))
    assert torch.allclose(s, gold["s_det"], rtol=0, atol=2e-6)
    s0 = torch.tensor([[0.0, 1.0]]).expand(gold["near"].shape[0], 2)
    s1, t1 = ost.resample_level(s0, torch.ones(s0.shape[0], 1), 64, gold["jit_level0"], True, 0.0, 0.0, (0.0, 1.0),
                                gold["near"], gold["far"])
    assert torch.allclose(s1, gold["s_level0"], rtol=0, atol=1e-6)
    assert torch.allclose(t1, gold["t_level0"], rtol=1e-6, atol=1e-6)


def test_sampled_intervals_are_sorted_and_in_domain(gold):
    s = gold["s_multi"]
    assert torch.all(s[..., 1:] >= s[..., :-1]) and s.min() >= 0 and s.max() <= 1
