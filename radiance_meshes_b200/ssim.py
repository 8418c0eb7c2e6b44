"""Structural similarity map (Wang, Bovik, Sheikh and Simoncelli, 2004).

Gaussian-weighted local statistics (11x11 window, sigma 1.5, zero padding)
and the constants C1 = 0.01^2, C2 = 0.03^2 for images in [0, 1].  Returns the
per-pixel, per-channel SSIM map, which is what the reference's densification
statistics read (``render_err.py:121``: ``1 - ssim(render, gt).mean(dim=0)``).
"""
from __future__ import annotations

import math

import torch
import torch.nn.functional as F

__all__ = ["ssim_map"]


def _window(size: int, sigma: float, channels: int, device, dtype) -> torch.Tensor:
    x = torch.arange(size, dtype=torch.float64) - size // 2
    g = torch.exp(-(x * x) / (2.0 * sigma * sigma))
    g = g / g.sum()
    w = torch.outer(g, g).to(device=device, dtype=dtype)
    return w.expand(channels, 1, size, size).contiguous()


def ssim_map(img1: torch.Tensor, img2: torch.Tensor, window_size: int = 11, sigma: float = 1.5) -> torch.Tensor:
    """SSIM map of two [C,H,W] (or [N,C,H,W]) images, same shape as the input."""
    squeeze = img1.dim() == 3
    if squeeze:
        img1, img2 = img1.unsqueeze(0), img2.unsqueeze(0)
    c = img1.shape[1]
    w = _window(window_size, sigma, c, img1.device, img1.dtype)
    pad = window_size // 2

    def blur(x):
        return F.conv2d(x, w, padding=pad, groups=c)

    mu1, mu2 = blur(img1), blur(img2)
    s11 = blur(img1 * img1) - mu1 * mu1
    s22 = blur(img2 * img2) - mu2 * mu2
    s12 = blur(img1 * img2) - mu1 * mu2
    c1, c2 = 0.01 ** 2, 0.03 ** 2
    out = ((2 * mu1 * mu2 + c1) * (2 * s12 + c2)) / ((mu1 * mu1 + mu2 * mu2 + c1) * (s11 + s22 + c2))
    return out.squeeze(0) if squeeze else out
