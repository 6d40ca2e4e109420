"""The proposal and error fields' networks (source/models.py:285-523) on the fused
density kernels (include/n3ds.h: n3ds_density_net_*).

``MLP``, ``PropMLP`` and ``ErrorMLP`` keep the reference's class attributes, keyword
constructor (``setattr`` of every keyword, as models.py:317-320 does), submodules
and parameter names: ``encoder`` is a GridEncoder (neural3dstrokes_b200.gridencoder)
with the reference's buffers, ``density_layer`` is ``Sequential(Linear(L*C, 64),
ReLU, Linear(64, 1))``. A state_dict of the reference's PropMLP / ErrorMLP loads
unchanged, and with the same torch seed the initial parameters are the reference's
(same construction order).

What runs is not those layers: ``forward``, ``predict_density`` and
``ErrorMLP.sample_error`` call one CUDA kernel that warps, grid-encodes and applies
both layers and the activation (the first layer on the tensor cores, at float32
accuracy), and one backward kernel that returns the table and layer gradients.
Supported configuration: the density-only networks the stroke model builds
(disable_rgb, disable_density_normals, use_grid_encoder, level_dim 1, 2 or 4 with
L*C <= 15, density_noise 0 in training). Others raise at construction. Coordinates
get no gradient (the reference's proposal and error levels never ask for one:
models.py:175-186 detaches the distances); a coordinate tensor that requires grad
under autograd raises rather than returning a silently incomplete graph.

``hash_levelwise_mean`` (training mode, models.py:472-488) is one reduction kernel
over the table; by default it mirrors the reference's ``scatter_reduce_`` fallback
(channel 0 only), ``hash_decay_all_channels = True`` mirrors torch_scatter's
segment_coo (every channel).
"""
import ctypes

import numpy as np
import torch
import torch.nn as nn

from . import _lib
from .gridencoder import GridEncoder

WARP_SCALE, WARP_CONTRACT, WARP_NONE = 0, 1, 2
HIDDEN = 64


def _warp_mode(warp_fn, no_warp):
    if no_warp:
        return WARP_NONE
    if warp_fn is None:
        return WARP_SCALE
    if warp_fn == "contract":
        return WARP_CONTRACT
    raise NotImplementedError(f"Unknown warp function {warp_fn}")


def _check_cuda(t, name):
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor (the density network has no CPU path)")


def _net_struct(enc, w1, b1, w2, b2, density_bias, warp, bbox_size, raw_output, status=None, wait_limit_us=0,
                test_stall=0):
    C = enc.embeddings.shape[1]
    L = enc.offsets.shape[0] - 1
    n = _lib.DensityNet()
    n.table = _lib.ptr(enc.embeddings)
    n.offsets = _lib.ptr(enc.offsets)
    n.n_levels = L
    n.level_dim = C
    n.log2_per_level_scale = float(np.log2(enc.per_level_scale))
    n.base_resolution = int(enc.base_resolution)
    n.gridtype = int(enc.gridtype_id)
    n.align_corners = int(bool(enc.align_corners))
    n.w1, n.b1, n.w2, n.b2 = _lib.ptr(w1), _lib.ptr(b1), _lib.ptr(w2), _lib.ptr(b2)
    n.density_bias = float(density_bias)
    n.warp = warp
    # torch divides by a Python scalar as a multiplication by its float32 reciprocal
    n.warp_scale = float(np.float32(1.0) / np.float32(bbox_size / 2)) if warp == WARP_SCALE else 1.0
    n.grid_bound = 1.0
    n.raw_output = int(bool(raw_output))
    n.status = _lib.ptr(status)
    n.wait_limit_us = int(wait_limit_us)
    n.test_stall = int(test_stall)
    return n


class _DensityNetFn(torch.autograd.Function):
    """density = net(coords) with the table and the four layer tensors as inputs."""

    @staticmethod
    def forward(ctx, coords, embeddings, w1, b1, w2, b2, spec):
        enc, density_bias, warp, bbox_size, raw_output, opts = spec
        x = coords.reshape(-1, 3).contiguous()
        n = x.shape[0]
        lib = _lib.load()
        L, C = enc.offsets.shape[0] - 1, embeddings.shape[1]
        need = any(ctx.needs_input_grad[1:6])
        stride = lib.n3ds_density_net_feature_stride(L, C)
        dev = x.device
        density = torch.empty(n, device=dev, dtype=torch.float32)
        warped = torch.empty(n, 3, device=dev, dtype=torch.float32)
        feats = torch.empty(n, stride, device=dev, dtype=torch.float32) if need else None
        net = _net_struct(enc, w1, b1, w2, b2, density_bias, warp, bbox_size, raw_output, **opts)
        with torch.cuda.device(dev):
            _lib.check(lib.n3ds_density_net_forward(ctypes.byref(net), _lib.ptr(x), n, _lib.ptr(density),
                                                    _lib.ptr(feats), _lib.ptr(warped), _lib.stream_ptr()))
        ctx.mark_non_differentiable(warped)
        ctx.spec = spec
        ctx.shape = coords.shape[:-1]
        ctx.save_for_backward(x, feats, embeddings, w1, b1, w2, b2)
        return density.reshape(ctx.shape), warped.reshape(coords.shape)

    @staticmethod
    def backward(ctx, g_density, g_warped):
        x, feats, embeddings, w1, b1, w2, b2 = ctx.saved_tensors
        enc, density_bias, warp, bbox_size, raw_output, opts = ctx.spec
        g = g_density.reshape(-1).contiguous().to(torch.float32)
        grads = [torch.zeros_like(t) for t in (embeddings, w1, b1, w2, b2)]
        net = _net_struct(enc, w1, b1, w2, b2, density_bias, warp, bbox_size, raw_output, **opts)
        lib = _lib.load()
        with torch.cuda.device(x.device):
            _lib.check(lib.n3ds_density_net_backward(ctypes.byref(net), _lib.ptr(x), _lib.ptr(feats), _lib.ptr(g),
                                                     x.shape[0], *[_lib.ptr(t) for t in grads],
                                                     _lib.stream_ptr()))
        return (None,) + tuple(grads) + (None,)


def density_net(coords, encoder, density_layer, density_bias=-1.0, warp_fn=None, bbox_size=2.0, no_warp=False,
                raw_output=False, status=None, wait_limit_us=0, test_stall=False):
    """(density [...], warped coords [..., 3]) of the network at coords [..., 3]:
    softplus(density_layer(encoder(warp(coords), bound=1.0)) + density_bias), or the
    density_layer output itself with raw_output."""
    _check_cuda(coords, "coords")
    if coords.requires_grad and torch.is_grad_enabled():
        raise RuntimeError("the fused density network gives no coordinate gradient; pass detached coordinates "
                           "(the reference's proposal and error levels do)")
    w1, b1 = density_layer[0].weight, density_layer[0].bias
    w2, b2 = density_layer[2].weight, density_layer[2].bias
    for name, t in (("embeddings", encoder.embeddings), ("w1", w1), ("b1", b1), ("w2", w2), ("b2", b2)):
        _check_cuda(t, name)
        if t.dtype != torch.float32 or not t.is_contiguous():
            raise RuntimeError(f"{name} must be a contiguous float32 tensor")
    if coords.dtype != torch.float32:
        raise RuntimeError("coords must be float32")
    spec = (encoder, float(density_bias), _warp_mode(warp_fn, no_warp), float(bbox_size), bool(raw_output),
            {"status": status, "wait_limit_us": wait_limit_us, "test_stall": int(bool(test_stall))})
    return _DensityNetFn.apply(coords, encoder.embeddings, w1, b1, w2, b2, spec)


class _LevelMeanSqFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, embeddings, offsets, all_channels):
        L, C = offsets.shape[0] - 1, embeddings.shape[1]
        out = torch.empty(L, C, device=embeddings.device, dtype=torch.float32)
        with torch.cuda.device(embeddings.device):
            _lib.check(_lib.load().n3ds_grid_level_mean_sq(_lib.ptr(embeddings), _lib.ptr(offsets), L, C,
                                                           int(bool(all_channels)), _lib.ptr(out),
                                                           _lib.stream_ptr()))
        ctx.save_for_backward(embeddings, offsets)
        ctx.all_channels = all_channels
        return out

    @staticmethod
    def backward(ctx, g):
        embeddings, offsets = ctx.saved_tensors
        L, C = offsets.shape[0] - 1, embeddings.shape[1]
        grad = torch.zeros_like(embeddings)
        with torch.cuda.device(embeddings.device):
            _lib.check(_lib.load().n3ds_grid_level_mean_sq_backward(
                _lib.ptr(embeddings), _lib.ptr(offsets), L, C, int(bool(ctx.all_channels)),
                _lib.ptr(g.contiguous().to(torch.float32)), _lib.ptr(grad), _lib.stream_ptr()))
        return grad, None, None


def level_mean_sq(embeddings, offsets, all_channels=False):
    """[L, C] mean over each level's rows of embeddings^2 (models.py:472-488)."""
    _check_cuda(embeddings, "embeddings")
    if embeddings.dtype != torch.float32 or not embeddings.is_contiguous():
        raise RuntimeError("embeddings must be a contiguous float32 tensor")
    return _LevelMeanSqFn.apply(embeddings, offsets, all_channels)


class MLP(nn.Module):
    """models.py:285-499, the density-only configuration (see the module docstring)."""
    bottleneck_width: int = 256
    net_depth_viewdirs: int = 2
    net_width_viewdirs: int = 256
    skip_layer_dir: int = 0
    num_rgb_channels: int = 3
    deg_view: int = 4
    bottleneck_noise: float = 0.0
    density_bias: float = -1.
    density_noise: float = 0.
    rgb_premultiplier: float = 1.
    rgb_bias: float = 0.
    rgb_padding: float = 0.001
    disable_density_normals: bool = True
    disable_rgb: bool = False
    bbox_size: float = 4.
    warp_fn = 'contract'

    use_grid_encoder: bool = True
    grid_level_interval: int = 2
    grid_level_dim: int = 4
    grid_base_resolution: int = 16
    grid_disired_resolution: int = 8192
    grid_log2_hashmap_size: int = 21
    mlp_pe_freqs: int = 8
    mlp_num_layers: int = 4
    mlp_hidden_dim: int = 128

    # not in the reference: which hash_levelwise_mean to mirror (False: the
    # scatter_reduce_ fallback, channel 0; True: torch_scatter's segment_coo)
    hash_decay_all_channels: bool = False

    def __init__(self, **kwargs):
        super().__init__()
        for k, v in kwargs.items():
            setattr(self, k, v)
        if not self.use_grid_encoder:
            raise NotImplementedError("only the hash-grid encoder is built (use_grid_encoder=True)")
        if not self.disable_rgb:
            raise NotImplementedError("only the density-only network is built (disable_rgb=True, as PropMLP "
                                      "and the stroke model's ErrorMLP)")
        if not self.disable_density_normals:
            raise NotImplementedError("density normals need coordinate gradients, which the fused network "
                                      "does not give (disable_density_normals=True)")
        _warp_mode(self.warp_fn, False)
        self.grid_num_levels = int(
            np.log(self.grid_disired_resolution / self.grid_base_resolution) / np.log(self.grid_level_interval)) + 1
        if self.grid_level_dim not in (1, 2, 4) or self.grid_num_levels * self.grid_level_dim > 15:
            raise NotImplementedError("the fused network takes level_dim 1, 2 or 4 and at most 15 features "
                                      f"(got {self.grid_num_levels} levels x {self.grid_level_dim})")
        self.encoder = GridEncoder(input_dim=3, num_levels=self.grid_num_levels, level_dim=self.grid_level_dim,
                                   base_resolution=self.grid_base_resolution,
                                   desired_resolution=self.grid_disired_resolution,
                                   log2_hashmap_size=self.grid_log2_hashmap_size, gridtype='hash',
                                   align_corners=False)
        last_dim = self.encoder.output_dim
        self.density_layer = nn.Sequential(nn.Linear(last_dim, HIDDEN), nn.ReLU(), nn.Linear(HIDDEN, 1))
        self.status = None  # optional device int32 status word of the kernels' bounded waits

    def _run(self, coords, no_warp, raw_output):
        if self.training and self.density_noise > 0:
            raise NotImplementedError("density_noise > 0 in training is not built")
        return density_net(coords, self.encoder, self.density_layer, self.density_bias, self.warp_fn,
                           self.bbox_size, no_warp, raw_output, status=self.status)

    def predict_density(self, coords, no_warp=False):
        """models.py:362-372: (raw_density [...], x [..., 1], warped coords)."""
        raw, warped = self._run(coords, no_warp, True)
        return raw, raw[..., None], warped

    def forward(self, coords, radius, viewdirs=None, no_warp=False):
        """models.py:374-499 with disable_rgb: dict(coord, density, rgb (zeros),
        normals None, hash_levelwise_mean)."""
        density, warped = self._run(coords, no_warp, False)
        rgb = torch.zeros(density.shape + (3, ), device=density.device)
        hash_levelwise_mean = None
        if self.training:
            hash_levelwise_mean = level_mean_sq(self.encoder.embeddings, self.encoder.offsets,
                                                self.hash_decay_all_channels)
        return dict(coord=warped, density=density, rgb=rgb, normals=None, hash_levelwise_mean=hash_levelwise_mean)


class NerfMLP(MLP):
    pass


class PropMLP(MLP):
    disable_rgb: bool = True
    grid_level_dim: int = 1


class ErrorMLP(MLP):
    num_rgb_channels: int = 1
    grid_level_dim: int = 2
    grid_log2_hashmap_size: int = 20

    def sample_error(self, coords, no_warp=False):
        """models.py:513-523 with disable_rgb: the density at coords."""
        density, _ = self._run(coords, no_warp, False)
        return density
