"""Stroke textures: the reference's source/textures.py API over the B200 backend.

``get_stroke_texture(stroke_texture, texture_image_path, texture_image_size)`` and
``ImageTexture(tint_image, texture_size, modulate_alpha=..., tint_ratio=...)`` with
``forward(texcoords, colors, alphas) -> (colors, alphas)`` as in textures.py:10-83:
the texture is sampled bilinearly at each (sample, stroke) pair's texcoord
(grid_sample semantics: align_corners=True, zero outside the image) in one CUDA
kernel per direction (``n3ds_texture_forward`` / ``n3ds_texture_backward``).

Differences, all deliberate: the image may be given as an array or tensor as well as
a file path; the configuration is passed as arguments instead of through gin.
"""
from typing import Optional, Sequence, Union

import numpy as np
import torch
import torch.nn as nn
import torch.nn.functional as F
from torch.autograd.function import once_differentiable

from . import _lib


def _load_image(src) -> torch.Tensor:
    """An image file path (read as misc.load_img does: PIL, float32 0..255), a numpy
    array or a tensor [H, W] or [H, W, C] in 0..255 -> float32 [1, C, H, W] in 0..1."""
    if isinstance(src, (str, bytes)):
        from PIL import Image
        src = np.array(Image.open(src), dtype=np.float32)
    image = torch.as_tensor(np.asarray(src, dtype=np.float32) if not torch.is_tensor(src) else src).float()
    if image.ndim == 2:
        image = image.unsqueeze(-1)
    return (image / 255.).permute(2, 0, 1).unsqueeze(0)


class _TextureFn(torch.autograd.Function):
    """Tinted colours (and, with modulate_alpha, modulated alphas; else no alpha
    output: the caller passes its alphas through, as the reference does)."""

    @staticmethod
    def forward(ctx, texcoords, colors, alphas, image, tint_ratio, modulate_alpha):
        n = colors.numel() // 3
        tc = texcoords.contiguous().float().reshape(n, 2)
        col = colors.contiguous().float().reshape(n, 3)
        al = alphas.contiguous().float().reshape(n)
        img = image.contiguous().float()
        C, H, W = img.shape
        col_out = torch.empty_like(col)
        al_out = torch.empty_like(al) if modulate_alpha else None
        # texels interleaved as float4 (r, g, b, 0): one load per bilinear corner
        packed = torch.empty(H, W, 4, device=col.device)
        lib = _lib.load()
        with torch.cuda.device(col.device):
            st = _lib.stream_ptr()
            _lib.check(lib.n3ds_texture_pack(_lib.ptr(packed), _lib.ptr(img), C, H, W, st))
            _lib.check(lib.n3ds_texture_forward_packed(_lib.ptr(col_out), _lib.ptr(al_out), _lib.ptr(tc),
                                                       _lib.ptr(col), _lib.ptr(al), n, _lib.ptr(packed), C, H, W,
                                                       float(tint_ratio), int(bool(modulate_alpha)), st))
        ctx.save_for_backward(tc, packed)
        ctx.meta = (float(tint_ratio), bool(modulate_alpha), colors.shape, alphas.shape, C)
        if not modulate_alpha:
            return col_out.reshape(colors.shape)
        return col_out.reshape(colors.shape), al_out.reshape(alphas.shape)

    @staticmethod
    @once_differentiable
    def backward(ctx, g_col, g_al=None):
        tc, packed = ctx.saved_tensors
        tint_ratio, modulate, cshape, ashape, C = ctx.meta
        n = tc.shape[0]
        H, W = packed.shape[0], packed.shape[1]
        gc = None if g_col is None else g_col.contiguous().float().reshape(n, 3)
        ga = None if g_al is None else g_al.contiguous().float().reshape(n)
        gcol = torch.empty(n, 3, device=tc.device) if ctx.needs_input_grad[1] else None
        gal = torch.empty(n, device=tc.device) if (modulate and ctx.needs_input_grad[2]) else None
        lib = _lib.load()
        with torch.cuda.device(tc.device):
            _lib.check(lib.n3ds_texture_backward_packed(_lib.ptr(gcol), _lib.ptr(gal), _lib.ptr(gc), _lib.ptr(ga),
                                                        _lib.ptr(tc), n, _lib.ptr(packed), C, H, W, tint_ratio,
                                                        int(modulate), _lib.stream_ptr()))
        return (None, None if gcol is None else gcol.reshape(cshape), None if gal is None else gal.reshape(ashape),
                None, None, None)


class StrokeTexture(nn.Module):
    """A 3D stroke texture queried at UV texture coordinates (textures.py:19-33)."""

    def forward(self, texcoords: torch.Tensor, colors: torch.Tensor, alphas: torch.Tensor):
        raise NotImplementedError


class ImageTexture(StrokeTexture):
    """Tint stroke colours (and optionally alphas) by an image (textures.py:36-83)."""
    modulate_alpha: bool = False  # whether to modulate alpha with the texture
    tint_ratio: float = 1.0       # the amount of original colour to tint with

    def __init__(self, tint_image: Union[str, np.ndarray, torch.Tensor], texture_size: Sequence[int], **kwargs):
        super().__init__()
        for k, v in kwargs.items():
            setattr(self, k, v)
        image = _load_image(tint_image)
        image = F.interpolate(image, tuple(int(s) for s in texture_size), mode="area")
        self.register_buffer("image_texture", image, persistent=False)

    def forward(self, texcoords: torch.Tensor, colors: torch.Tensor, alphas: torch.Tensor):
        if colors.shape[-1] != 3:
            raise ValueError("Colors should be RGB for ImageTexture")
        C = self.image_texture.shape[1]
        if C not in (1, 3):
            raise ValueError("Texture should be RGB or grayscale")
        if colors.shape[:-1] != alphas.shape or texcoords.shape[:-1] != alphas.shape or texcoords.shape[-1] != 2:
            raise ValueError("expected texcoords [..., 2], colors [..., 3], alphas [...] of one shape")
        if not colors.is_cuda:
            raise RuntimeError("ImageTexture runs on CUDA tensors")
        image = self.image_texture[0].to(colors.device)
        if not self.modulate_alpha:  # alphas pass through unchanged (the same tensor, as in the reference)
            return _TextureFn.apply(texcoords.detach(), colors, alphas, image, float(self.tint_ratio), False), alphas
        return _TextureFn.apply(texcoords.detach(), colors, alphas, image, float(self.tint_ratio), True)


def get_stroke_texture(stroke_texture: str = "none", texture_image_path: Optional[str] = None,
                       texture_image_size: Sequence[int] = (256, 256), **kwargs):
    """textures.py:10-16: None for 'none', an ImageTexture for 'image'."""
    if stroke_texture == "none":
        return None
    if stroke_texture == "image":
        return ImageTexture(texture_image_path, texture_image_size, **kwargs)
    raise ValueError(f"Unknown stroke texture {stroke_texture}")
