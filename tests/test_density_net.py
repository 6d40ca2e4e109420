"""CPU checks of the proposal / error networks (neural3dstrokes_b200/mlp.py) and of
their float64 oracle: the reference's module layout, the supported configurations,
the host checks, the oracle's gradients against central differences, and
hash_levelwise_mean against the reference's scatter_reduce_ fallback."""
import numpy as np
import pytest
import torch

from neural3dstrokes_b200 import mlp
from oracle import density_net as odn


def test_module_layout_is_the_references():
    """Parameter and buffer names of models.py:285-346 (PropMLP and ErrorMLP with
    disable_rgb), levels from the desired resolution as models.py:322-325."""
    p0 = mlp.PropMLP(grid_disired_resolution=512)
    p1 = mlp.PropMLP(grid_disired_resolution=2048)
    e = mlp.ErrorMLP(grid_disired_resolution=256, disable_rgb=True)
    for m, L, C in ((p0, 6, 1), (p1, 8, 1), (e, 5, 2)):
        assert [n for n, _ in m.named_parameters()] == ["encoder.embeddings", "density_layer.0.weight",
                                                        "density_layer.0.bias", "density_layer.2.weight",
                                                        "density_layer.2.bias"]
        assert [n for n, _ in m.named_buffers()] == ["encoder.offsets", "encoder.idx", "encoder.grid_sizes"]
        assert m.encoder.num_levels == L and m.encoder.level_dim == C
        assert m.density_layer[0].weight.shape == (64, L * C) and m.density_layer[2].weight.shape == (1, 64)
        assert m.density_bias == -1.0 and m.warp_fn == "contract"
    assert e.encoder.log2_hashmap_size == 20 and p0.encoder.log2_hashmap_size == 21


@pytest.mark.parametrize("kw", [dict(), dict(disable_rgb=True, use_grid_encoder=False),
                                dict(disable_rgb=True, disable_density_normals=False),
                                dict(disable_rgb=True, grid_level_dim=8),
                                dict(disable_rgb=True, grid_level_dim=4)])
def test_unsupported_configurations_raise(kw):
    # MLP's defaults (rgb head; 10 levels x 4 channels) are not the density-only net
    with pytest.raises(NotImplementedError):
        mlp.MLP(**kw)


def test_unknown_warp_raises():
    with pytest.raises(NotImplementedError):
        mlp.PropMLP(warp_fn="sphere")


def test_host_tensors_raise():
    net = mlp.PropMLP(grid_disired_resolution=512)
    with pytest.raises(RuntimeError, match="CUDA"):
        net(torch.zeros(4, 3), None)


def small_net(seed=0, level_dim=1, desired=64):
    torch.manual_seed(seed)
    net = mlp.MLP(disable_rgb=True, grid_level_dim=level_dim, grid_disired_resolution=desired,
                  grid_log2_hashmap_size=10, warp_fn=None, bbox_size=2.0)
    with torch.no_grad():
        net.encoder.embeddings.uniform_(-1, 1)
    return net


def oracle_args(net):
    enc, lay = net.encoder, net.density_layer
    return (enc.embeddings, enc.offsets, float(np.log2(enc.per_level_scale)), enc.base_resolution,
            lay[0].weight, lay[0].bias, lay[2].weight, lay[2].bias)


def test_oracle_gradients_match_central_differences():
    net = small_net(level_dim=2)
    x = torch.rand(40, 3) * 1.8 - 0.9
    g = torch.randn(40, dtype=torch.float64)
    args = list(oracle_args(net))
    grads = odn.backward(g, x, *args, warp=odn.WARP_SCALE, bbox_size=2.0)
    h = 1e-6
    rng = np.random.default_rng(0)
    for k, idx in ((0, None), (4, (3, 1)), (5, (7,)), (6, (0, 11)), (7, (0,))):
        base = args[k].detach().double()
        if idx is None:  # a table row that the points touch
            idx = tuple(int(i) for i in np.argwhere(grads[0].abs().numpy() > 0)[rng.integers(0, 10)])
        plus, minus = base.clone(), base.clone()
        plus[idx] += h
        minus[idx] -= h
        f = []
        for t in (plus, minus):
            a = list(args)
            a[k] = t
            d, _, _ = odn.forward(x, *a, warp=odn.WARP_SCALE, bbox_size=2.0)
            f.append(float((d * g).sum()))
        fd = (f[0] - f[1]) / (2 * h)
        assert abs(fd - float(grads[k if k == 0 else k - 3][idx])) < 1e-6 * max(1.0, abs(fd))


def test_oracle_contract_warp_is_coord_contract():
    """The float32 restatement of the contract map against coord.contract as torch
    ops (source/utils/coord.py:5-11) followed by / 2. On the CPU torch sums the squares
    in another order and its sqrt is not always correctly rounded, so the two agree to
    a few ulp here; the GPU tests pin the restatement bit for bit to torch's CUDA ops."""
    x = torch.randn(1000, 3) * 2
    w, u = odn.warp_to_unit(x, odn.WARP_CONTRACT)
    eps = torch.finfo(x.dtype).eps
    m = torch.sum(x ** 2, dim=-1, keepdim=True).clamp_min(eps)
    ref = torch.where(m <= 1, x, ((2 * torch.sqrt(m) - 1) / m) * x) / 2.0
    assert float((w - ref).abs().max()) <= 4 * eps
    assert torch.equal(u, (w + 1.0) / 2.0)


def test_level_mean_sq_oracle_is_the_scatter_reduce_fallback():
    """models.py:476-488 without torch_scatter: scatter_reduce_ with an index of one
    column reduces channel 0 only."""
    net = mlp.ErrorMLP(grid_disired_resolution=64, disable_rgb=True, grid_log2_hashmap_size=10)
    with torch.no_grad():
        net.encoder.embeddings.uniform_(-1, 1)
    emb = net.encoder.embeddings.detach()
    ref = torch.zeros(net.encoder.num_levels, emb.shape[-1]).scatter_reduce_(
        0, net.encoder.idx.unsqueeze(1), torch.square(emb), reduce="mean", include_self=False)
    ours = odn.level_mean_sq(emb, net.encoder.offsets)
    assert float((ours - ref.double()).abs().max()) < 1e-6
    assert bool((ours[:, 1:] == 0).all())
    all_ch = odn.level_mean_sq(emb, net.encoder.offsets, all_channels=True)
    assert float((all_ch[:, 0] - ours[:, 0]).abs().max()) == 0.0 and bool((all_ch[:, 1] > 0).all())


def _net(**kw):
    from neural3dstrokes_b200 import _lib
    n = _lib.DensityNet()
    fake = 0x10000  # never dereferenced: every case below fails its host checks first
    n.table = n.offsets = n.w1 = n.b1 = n.w2 = n.b2 = fake
    n.n_levels, n.level_dim = 8, 1
    n.log2_per_level_scale, n.base_resolution = 1.0, 16
    n.grid_bound = 1.0
    n.warp_scale = 1.0
    for k, v in kw.items():
        setattr(n, k, v)
    return n


@pytest.mark.parametrize("kw,code", [(dict(level_dim=8), 2), (dict(n_levels=16), 2), (dict(level_dim=4, n_levels=4), 2),
                                     (dict(n_levels=0), 2), (dict(warp=7), 1), (dict(grid_bound=0.0), 1),
                                     (dict(base_resolution=0), 1), (dict(table=None), 1)])
def test_density_net_host_checks(kw, code):
    """Descriptors outside the supported network fail with N3DS_ERR_UNSUPPORTED (2) or
    N3DS_ERR_INVALID (1) and a message, before anything reaches the device."""
    import ctypes
    from neural3dstrokes_b200 import _lib
    lib = _lib.load()
    rc = lib.n3ds_density_net_forward(ctypes.byref(_net(**kw)), ctypes.c_void_p(0x10000), 10,
                                      ctypes.c_void_p(0x10000), None, None, None)
    assert rc == code and lib.n3ds_last_error().decode()


def test_density_net_host_checks_of_buffers():
    import ctypes
    from neural3dstrokes_b200 import _lib
    lib = _lib.load()
    p = ctypes.c_void_p(0x10000)
    net = ctypes.byref(_net())
    assert lib.n3ds_density_net_forward(net, p, -1, p, None, None, None) == 1         # negative count
    assert lib.n3ds_density_net_forward(net, None, 10, p, None, None, None) == 1      # no coordinates
    assert lib.n3ds_density_net_forward(net, p, 10, p, ctypes.c_void_p(0x10004), None, None) == 1  # record misaligned
    assert lib.n3ds_density_net_backward(net, p, None, p, 10, p, p, p, p, p, None) == 1  # no record
    assert lib.n3ds_density_net_backward(net, p, p, p, 10, None, p, p, p, p, None) == 1  # no table gradient
    assert lib.n3ds_density_net_forward(net, p, 0, p, None, None, None) == 0          # nothing to do
    assert lib.n3ds_grid_level_mean_sq(p, p, 8, 8, 0, p, None) == 2                   # level_dim 8
    assert lib.n3ds_grid_level_mean_sq(p, p, 8, 1, 0, None, None) == 1                # no output
    assert lib.n3ds_density_net_feature_stride(6, 1) == 8 and lib.n3ds_density_net_feature_stride(5, 2) == 12
