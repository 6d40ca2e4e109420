"""Drop-in replacement of the reference's grid encoder (source/gridencoder/grid.py)
and of its native module ``_gridencoder``.

grid.py imports ``_gridencoder`` before JIT-building its own backend
(grid.py:9-12), so the module ``neural3dstrokes_b200/shim/_gridencoder.py`` on
``sys.path`` routes the reference's GridEncoder to these kernels with no edit. The
three functions below keep the reference's argument order and meaning
(gridencoder.h:7-14):

- tensors must be CUDA and contiguous, embeddings / grads floating (float32,
  float16 or float64) and offsets int32, else ``RuntimeError``;
- C must be 1, 2, 4 or 8 and D 2 to 5 (``RuntimeError``, as the reference's
  ``std::runtime_error``);
- outputs are caller-allocated; grad_embeddings and the total variation's grad are
  accumulated into; launches go to the current torch stream.

Beyond the reference, sizes are checked against the tensors before any launch
(the reference indexes with whatever B, L and offsets it is given), and the
offsets are checked once per offsets tensor against the table (one host read).

``GridEncoder`` and ``grid_encode`` restate grid.py:24-193 on these functions.
"""
import numpy as np
import torch
import torch.nn as nn

from . import _lib

_gridtype_to_id = {"hash": 0, "tiled": 1}
_interp_to_id = {"linear": 0, "smoothstep": 1}
_DTYPES = {torch.float32: 0, torch.float16: 1, torch.float64: 2}
_checked_offsets = {}


def _check(t, name, floating=True):
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be a contiguous tensor")
    if floating and t.dtype not in _DTYPES:
        raise RuntimeError(f"{name} must be a floating tensor")


def _need(cond, msg):
    if not cond:
        raise RuntimeError(msg)


def _geometry(D, C, L, B):
    _need(0 <= B < 2 ** 32, "B must be in [0, 2^32) (a uint32, as in the reference)")
    _need(C in (1, 2, 4, 8), "GridEncoding: C must be 1, 2, 4, or 8.")
    _need(D in (2, 3, 4, 5), "GridEncoding: D must be 2, 3, 4, or 5.")
    _need(L >= 1, "GridEncoding: L must be >= 1")


def _check_offsets(offsets, L, rows):
    _check(offsets, "offsets", floating=False)
    _need(offsets.dtype == torch.int32, "offsets must be an int tensor")
    _need(offsets.numel() >= L + 1, "offsets must hold L + 1 entries")
    key = (offsets.data_ptr(), offsets._version, offsets.numel(), rows)
    if key not in _checked_offsets:
        if len(_checked_offsets) > 4096:  # a bounded memo, not a registry
            _checked_offsets.clear()
        o = offsets[:L + 1].cpu().numpy().astype(np.int64)
        _need(o[0] >= 0 and (np.diff(o) > 0).all() and o[-1] <= rows,
              "offsets must increase strictly from >= 0 and end within the embedding table")
        _checked_offsets[key] = True


def _dtype(t):
    return _DTYPES[t.dtype]


def grid_encode_forward(inputs, embeddings, offsets, outputs, B, D, C, L, S, H, dy_dx=None, gridtype=0,
                        align_corners=False, interp=0):
    """gridencoder.cu:567-592: outputs [L, B, C] (and dy_dx [B, L*D*C]) of embeddings' dtype."""
    for n, t in (("inputs", inputs), ("embeddings", embeddings), ("outputs", outputs)):
        _check(t, n)
    _need(inputs.dtype == torch.float32, "inputs must be a float32 tensor")
    _geometry(D, C, L, B)
    _need(outputs.dtype == embeddings.dtype, "outputs must have the embeddings' dtype")
    _need(inputs.numel() >= B * D, "inputs must hold B * D values")
    _need(embeddings.dim() == 2 and embeddings.size(1) == C, "embeddings must be [rows, C]")
    _need(outputs.numel() >= L * B * C, "outputs must hold L * B * C values")
    if dy_dx is not None:
        _check(dy_dx, "dy_dx")
        _need(dy_dx.dtype == embeddings.dtype and dy_dx.numel() >= B * L * D * C, "dy_dx must be [B, L * D * C]")
    _check_offsets(offsets, L, embeddings.size(0))
    lib = _lib.load()
    with torch.cuda.device(inputs.device):
        _lib.check(lib.n3ds_grid_encode_forward(
            _lib.ptr(inputs), _lib.ptr(embeddings), _lib.ptr(offsets), _lib.ptr(outputs), B, D, C, L, float(S),
            int(H), _lib.ptr(dy_dx), int(gridtype), int(bool(align_corners)), int(interp), _dtype(embeddings),
            _lib.stream_ptr()))


def grid_encode_backward(grad, inputs, embeddings, offsets, grad_embeddings, B, D, C, L, S, H, dy_dx=None,
                         grad_inputs=None, gridtype=0, align_corners=False, interp=0):
    """gridencoder.cu:594-626: grad_embeddings += the table gradient; grad_inputs
    (with dy_dx) = sum over levels and channels of grad * dy_dx."""
    for n, t in (("grad", grad), ("inputs", inputs), ("embeddings", embeddings),
                 ("grad_embeddings", grad_embeddings)):
        _check(t, n)
    _need(inputs.dtype == torch.float32, "inputs must be a float32 tensor")
    _geometry(D, C, L, B)
    _need(grad.dtype == embeddings.dtype == grad_embeddings.dtype, "grad, embeddings and grad_embeddings "
          "must share a dtype")
    _need(inputs.numel() >= B * D and grad.numel() >= L * B * C, "inputs / grad are too small")
    _need(grad_embeddings.shape == embeddings.shape, "grad_embeddings must have the embeddings' shape")
    if dy_dx is not None:
        _check(dy_dx, "dy_dx")
        _need(dy_dx.dtype == grad.dtype and dy_dx.numel() >= B * L * D * C, "dy_dx must be [B, L * D * C]")
    if grad_inputs is not None:
        _check(grad_inputs, "grad_inputs")
        _need(grad_inputs.dtype == grad.dtype and grad_inputs.numel() >= B * D, "grad_inputs must be [B, D]")
    _check_offsets(offsets, L, embeddings.size(0))
    lib = _lib.load()
    with torch.cuda.device(inputs.device):
        _lib.check(lib.n3ds_grid_encode_backward(
            _lib.ptr(grad), _lib.ptr(inputs), _lib.ptr(embeddings), _lib.ptr(offsets), _lib.ptr(grad_embeddings),
            B, D, C, L, float(S), int(H), _lib.ptr(dy_dx), _lib.ptr(grad_inputs), int(gridtype),
            int(bool(align_corners)), int(interp), _dtype(grad), _lib.stream_ptr()))


def grad_total_variation(inputs, embeddings, grad, offsets, weight, B, D, C, L, S, H, gridtype=0,
                         align_corners=False):
    """gridencoder.cu:629-644: grad += the total-variation gradient at B points.
    inputs have the embeddings' dtype (the reference reads them as scalar_t)."""
    for n, t in (("inputs", inputs), ("embeddings", embeddings), ("grad", grad)):
        _check(t, n)
    _geometry(D, C, L, B)
    _need(inputs.dtype == embeddings.dtype == grad.dtype, "inputs, embeddings and grad must share a dtype")
    _need(inputs.numel() >= B * D, "inputs must hold B * D values")
    _need(grad.shape == embeddings.shape and embeddings.dim() == 2 and embeddings.size(1) == C,
          "grad and embeddings must be [rows, C]")
    _check_offsets(offsets, L, embeddings.size(0))
    lib = _lib.load()
    with torch.cuda.device(inputs.device):
        _lib.check(lib.n3ds_grid_total_variation(
            _lib.ptr(inputs), _lib.ptr(embeddings), _lib.ptr(grad), _lib.ptr(offsets), float(weight), B, D, C, L,
            float(S), int(H), int(gridtype), int(bool(align_corners)), _dtype(embeddings), _lib.stream_ptr()))


def _autocast_on():
    try:
        return torch.is_autocast_enabled("cuda")
    except TypeError:
        return torch.is_autocast_enabled()


class _grid_encode(torch.autograd.Function):
    """grid.py:24-88."""

    @staticmethod
    @torch.amp.custom_fwd(device_type="cuda")
    def forward(ctx, inputs, embeddings, offsets, per_level_scale, base_resolution, calc_grad_inputs=False,
                gridtype=0, align_corners=False, interpolation=0):
        inputs = inputs.contiguous()
        B, D = inputs.shape
        L = offsets.shape[0] - 1
        C = embeddings.shape[1]
        S = np.log2(per_level_scale)
        H = base_resolution
        # half-precision tables under autocast when C is even (grid.py:41-44)
        if _autocast_on() and C % 2 == 0:
            embeddings = embeddings.to(torch.half)
        outputs = torch.empty(L, B, C, device=inputs.device, dtype=embeddings.dtype)
        dy_dx = torch.empty(B, L * D * C, device=inputs.device, dtype=embeddings.dtype) if calc_grad_inputs else None
        grid_encode_forward(inputs, embeddings, offsets, outputs, B, D, C, L, S, H, dy_dx, gridtype, align_corners,
                            interpolation)
        outputs = outputs.permute(1, 0, 2).reshape(B, L * C)
        ctx.save_for_backward(inputs, embeddings, offsets, dy_dx)
        ctx.dims = [B, D, C, L, S, H, gridtype, interpolation]
        ctx.align_corners = align_corners
        return outputs

    @staticmethod
    @torch.amp.custom_bwd(device_type="cuda")
    def backward(ctx, grad):
        inputs, embeddings, offsets, dy_dx = ctx.saved_tensors
        B, D, C, L, S, H, gridtype, interpolation = ctx.dims
        grad = grad.view(B, L, C).permute(1, 0, 2).contiguous().to(embeddings.dtype)
        grad_embeddings = torch.zeros_like(embeddings)
        grad_inputs = torch.zeros_like(inputs, dtype=embeddings.dtype) if dy_dx is not None else None
        grid_encode_backward(grad, inputs, embeddings, offsets, grad_embeddings, B, D, C, L, S, H, dy_dx,
                             grad_inputs, gridtype, ctx.align_corners, interpolation)
        if grad_inputs is not None:
            grad_inputs = grad_inputs.to(inputs.dtype)
        return grad_inputs, grad_embeddings, None, None, None, None, None, None, None


grid_encode = _grid_encode.apply


class GridEncoder(nn.Module):
    """grid.py:94-193: same constructor, buffers (offsets, idx, grid_sizes),
    parameter (embeddings [rows, level_dim]) and methods."""

    def __init__(self, input_dim=3, num_levels=16, level_dim=2, per_level_scale=2, base_resolution=16,
                 log2_hashmap_size=19, desired_resolution=None, gridtype="hash", align_corners=False,
                 interpolation="linear", init_std=1e-4):
        super().__init__()
        if desired_resolution is not None:
            per_level_scale = np.exp2(np.log2(desired_resolution / base_resolution) / (num_levels - 1))
        self.input_dim = input_dim
        self.num_levels = num_levels
        self.level_dim = level_dim
        self.per_level_scale = per_level_scale
        self.log2_hashmap_size = log2_hashmap_size
        self.base_resolution = base_resolution
        self.output_dim = num_levels * level_dim
        self.gridtype = gridtype
        self.gridtype_id = _gridtype_to_id[gridtype]
        self.interpolation = interpolation
        self.interp_id = _interp_to_id[interpolation]
        self.align_corners = align_corners
        self.init_std = init_std

        resolutions, offsets, offset = [], [], 0
        self.max_params = 2 ** log2_hashmap_size
        for i in range(num_levels):
            resolution = int(np.ceil(base_resolution * per_level_scale ** i))
            resolution = resolution if align_corners else resolution + 1
            params_in_level = min(self.max_params, resolution ** input_dim)
            params_in_level = int(np.ceil(params_in_level / 8) * 8)
            resolutions.append(resolution)
            offsets.append(offset)
            offset += params_in_level
        offsets.append(offset)
        self.register_buffer("offsets", torch.from_numpy(np.array(offsets, dtype=np.int32)))
        idx = torch.empty(offset, dtype=torch.long)
        for i in range(num_levels):
            idx[offsets[i]:offsets[i + 1]] = i
        self.register_buffer("idx", idx)
        self.register_buffer("grid_sizes", torch.from_numpy(np.array(resolutions, dtype=np.int32)))
        self.n_params = offsets[-1] * level_dim
        self.embeddings = nn.Parameter(torch.empty(offset, level_dim))
        self.reset_parameters()

    def reset_parameters(self):
        std = self.init_std
        self.embeddings.data.uniform_(-std, std)

    def __repr__(self):
        return (f"GridEncoder: input_dim={self.input_dim} num_levels={self.num_levels} level_dim={self.level_dim} "
                f"resolution={self.base_resolution} -> "
                f"{int(round(self.base_resolution * self.per_level_scale ** (self.num_levels - 1)))} "
                f"per_level_scale={self.per_level_scale:.4f} params={tuple(self.embeddings.shape)} "
                f"gridtype={self.gridtype} align_corners={self.align_corners} interpolation={self.interpolation}")

    def forward(self, inputs, bound=1):
        inputs = (inputs + bound) / (2 * bound)
        prefix_shape = list(inputs.shape[:-1])
        inputs = inputs.view(-1, self.input_dim)
        outputs = grid_encode(inputs, self.embeddings, self.offsets, self.per_level_scale, self.base_resolution,
                              inputs.requires_grad, self.gridtype_id, self.align_corners, self.interp_id)
        return outputs.view(prefix_shape + [self.output_dim])

    @torch.amp.autocast("cuda", enabled=False)
    def grad_total_variation(self, weight=1e-7, inputs=None, bound=1, B=1000000):
        """grid.py:172-193: adds the TV gradient to embeddings.grad at B random (or
        the given) points."""
        D = self.input_dim
        C = self.embeddings.shape[1]
        L = self.offsets.shape[0] - 1
        S = np.log2(self.per_level_scale)
        H = self.base_resolution
        if inputs is None:
            inputs = torch.rand(B, self.input_dim, device=self.embeddings.device)
        else:
            inputs = (inputs + bound) / (2 * bound)
            inputs = inputs.view(-1, self.input_dim)
            B = inputs.shape[0]
        if self.embeddings.grad is None:
            raise ValueError("grad is None, should be called after loss.backward() and before optimizer.step()!")
        grad_total_variation(inputs, self.embeddings, self.embeddings.grad, self.offsets, weight, B, D, C, L, S, H,
                             self.gridtype_id, self.align_corners)
