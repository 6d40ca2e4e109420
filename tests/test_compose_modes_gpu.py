"""Non-'over' composition modes (CUDA kernels behind compose_strokes) against the
float64 restatement of the reference's torch code (oracle.strokefield.compose_mode):
outputs within 1e-5, gradients of alphas, colours and density parameters within 1e-4
(helpers tolerances), both colour dimensions, batched leading shape."""
import pytest
import torch

from helpers import FWD_TOL, GRAD_TOL, rel
from neural3dstrokes_b200.strokes import compose_strokes
from oracle import strokefield as sf

pytestmark = pytest.mark.gpu

MODES = ["max", "max_density_weighted", "softmax", "softmax_density_weighted"]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("C,S", [(3, 37), (1, 5), (3, 300)])
def test_compose_mode_matches_reference_torch(cuda, mode, C, S):
    g = torch.Generator().manual_seed(S + C)
    a = torch.rand(6, 50, S, generator=g) ** 2
    c = torch.rand(6, 50, S, C, generator=g)
    d = torch.rand(S, generator=g) * 10
    gd = torch.randn(6, 50, generator=g)
    gc = torch.randn(6, 50, C, generator=g)
    ta, tc, td = (t.to(cuda).requires_grad_(True) for t in (a, c, d))
    dens, col = compose_strokes(ta, tc, td, mode)
    ((dens * gd.to(cuda)).sum() + (col * gc.to(cuda)).sum()).backward()
    ra, rc, rd = (t.double().requires_grad_(True) for t in (a, c, d))
    dens_r, col_r = sf.compose_mode(ra, rc, rd, mode)
    ((dens_r * gd.double()).sum() + (col_r * gc.double()).sum()).backward()
    assert rel(dens, dens_r) < FWD_TOL and rel(col, col_r) < FWD_TOL
    assert rel(ta.grad, ra.grad) < GRAD_TOL, rel(ta.grad, ra.grad)
    assert rel(tc.grad, rc.grad) < GRAD_TOL
    assert rel(td.grad, rd.grad) < GRAD_TOL, rel(td.grad, rd.grad)


def test_max_picks_first_of_ties(cuda):
    a = torch.tensor([[0.5, 0.9, 0.9, 0.1]], device=cuda)
    c = torch.arange(12, dtype=torch.float32, device=cuda).reshape(1, 4, 3)
    d = torch.ones(4, device=cuda)
    dens, col = compose_strokes(a, c, d, "max")
    assert float(dens[0]) == pytest.approx(0.9) and col[0].tolist() == [3.0, 4.0, 5.0]


def test_unknown_mode_raises(cuda):
    with pytest.raises(ValueError):
        compose_strokes(torch.rand(2, 3, device=cuda), torch.rand(2, 3, 3, device=cuda), torch.rand(3, device=cuda),
                        "median")
