"""ImageTexture (textures.py:36-83): the oracle's known answers and the host side of
the module (no GPU). GPU parity is in test_textures_gpu.py."""
import numpy as np
import pytest
import torch

from oracle import strokefield as orr
from neural3dstrokes_b200 import textures


def _img(C=3, H=4, W=5, seed=0):
    g = torch.Generator().manual_seed(seed)
    return torch.rand(C, H, W, generator=g, dtype=torch.float64)


def test_oracle_corners_centre_and_outside():
    img = _img()
    C, H, W = img.shape
    tc = torch.tensor([[0.0, 0.0], [1.0, 1.0], [1.0, 0.0], [-0.5, 0.5], [0.5, 1.7]], dtype=torch.float64)
    col = torch.ones(5, 3, dtype=torch.float64)
    out, _ = orr.image_texture(tc, col, torch.ones(5, dtype=torch.float64), img)
    assert torch.allclose(out[0], img[:, 0, 0])
    assert torch.allclose(out[1], img[:, H - 1, W - 1])
    assert torch.allclose(out[2], img[:, 0, W - 1])  # u indexes the width, v the height
    assert torch.all(out[3] == 0) and torch.all(out[4] == 0)  # zero padding outside


def test_oracle_bilinear_midpoint_tint_ratio_and_alpha():
    img = torch.tensor([[[0.0, 1.0], [2.0, 3.0]]], dtype=torch.float64)  # grayscale 2x2
    tc = torch.tensor([[0.5, 0.5]], dtype=torch.float64)
    col = torch.tensor([[0.2, 0.4, 0.6]], dtype=torch.float64)
    out, a = orr.image_texture(tc, col, torch.tensor([0.5], dtype=torch.float64), img, tint_ratio=0.5,
                               modulate_alpha=True)
    assert torch.allclose(out, (col * 0.5 + 0.5) * 1.5)
    assert torch.allclose(a, torch.tensor([0.75], dtype=torch.float64))


def test_image_texture_from_array_and_file(tmp_path):
    from PIL import Image
    rgb = (np.arange(8 * 6 * 3) % 251).astype(np.uint8).reshape(8, 6, 3)
    t = textures.ImageTexture(rgb, (4, 3))
    assert tuple(t.image_texture.shape) == (1, 3, 4, 3)
    # area resize of an exact 2x2 block average
    ref = torch.tensor(rgb, dtype=torch.float32).permute(2, 0, 1).reshape(3, 4, 2, 3, 2).mean((2, 4)) / 255
    assert torch.allclose(t.image_texture[0], ref, atol=1e-6)
    p = tmp_path / "tex.png"
    Image.fromarray(rgb).save(p)
    t2 = textures.ImageTexture(str(p), (8, 6), tint_ratio=0.3, modulate_alpha=True)
    assert torch.allclose(t2.image_texture[0], torch.tensor(rgb, dtype=torch.float32).permute(2, 0, 1) / 255)
    assert t2.tint_ratio == 0.3 and t2.modulate_alpha is True
    gray = textures.ImageTexture(rgb[..., 0], (8, 6))
    assert gray.image_texture.shape[1] == 1


def test_get_stroke_texture_and_errors():
    assert textures.get_stroke_texture("none") is None
    with pytest.raises(ValueError):
        textures.get_stroke_texture("noise")
    t = textures.ImageTexture(np.zeros((4, 4, 3), np.uint8), (4, 4))
    with pytest.raises(ValueError):
        t(torch.zeros(2, 2), torch.zeros(2, 4), torch.zeros(2))
    with pytest.raises(RuntimeError):  # CPU tensors: the op is CUDA only, no fallback
        t(torch.zeros(2, 2), torch.zeros(2, 3), torch.zeros(2))
