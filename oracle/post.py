"""CPU restatement of the post passes — TEST INFRASTRUCTURE.

Only tests/ import this module, as the checker of hdr_upscale / hdr_denoise.
  upscale_nearest : UpscalePass (passes/upscale_pass.cpp:13-95)
  chroma_blur     : Denoiser::_applyChromaticityBlur (passes/denoiser.cpp:54-96),
                    what Denoiser::Run does without OIDN (:164-201), alpha kept
  rendered_size   : CameraFrame::RenderedWidth/Height (renderContext/camera_frame.h:34-76)
Pinned against the reference's own passes compiled in place (oracle/_ref,
tests/test_post_passes.py). Float32 arithmetic in the reference's order: numpy
float32 elementwise operations round each step like the reference's build
(-ffp-contract=off), and the 3x3 sums are accumulated in its loop order.
"""
from __future__ import annotations

import numpy as np


def rendered_size(window: int, level: int) -> int:
    divisor = 1 << min(max(level, 0), 4)
    return max(1, (window + divisor - 1) // divisor)


def upscale_nearest(src: np.ndarray, src_w: int, src_h: int, dst_w: int, dst_h: int) -> np.ndarray:
    """src: (src_h * src_w, comps) -> (dst_h * dst_w, comps)."""
    x = np.minimum(src_w - 1, np.arange(dst_w, dtype=np.int64) * src_w // dst_w)
    y = np.minimum(src_h - 1, np.arange(dst_h, dtype=np.int64) * src_h // dst_h)
    idx = (y[:, None] * src_w + x[None, :]).reshape(-1)
    return np.asarray(src)[idx].copy()


def chroma_blur(rgba: np.ndarray, width: int, height: int) -> np.ndarray:
    """rgba: (height * width, 4) float32 -> the blurred image, alpha kept."""
    f = np.float32
    img = np.asarray(rgba, np.float32).reshape(height, width, 4)
    r, g, b = img[..., 0], img[..., 1], img[..., 2]
    luma = f(0.25) * r + f(0.5) * g + f(0.25) * b
    sum_co = np.zeros((height, width), np.float32)
    sum_cg = np.zeros((height, width), np.float32)
    weight = np.zeros((height, width), np.float32)
    ys, xs = np.arange(height), np.arange(width)
    for dy in (-1, 0, 1):
        ny = np.clip(ys + dy, 0, height - 1)
        for dx in (-1, 0, 1):
            nx = np.clip(xs + dx, 0, width - 1)
            q = img[ny][:, nx]
            sum_co = sum_co + (f(0.50) * q[..., 0] - f(0.5) * q[..., 2])
            sum_cg = sum_cg + ((f(-0.25) * q[..., 0] + f(0.5) * q[..., 1]) - f(0.25) * q[..., 2])
            weight = weight + f(1.0)
    co = sum_co / weight
    cg = sum_cg / weight

    def max0(v):  # std::max(0.0f, v)
        return np.where(f(0.0) < v, v, f(0.0)).astype(np.float32)

    out = img.copy()
    out[..., 0] = max0((luma + co) - cg)
    out[..., 1] = max0(luma + cg)
    out[..., 2] = max0((luma - co) - cg)
    return out.reshape(-1, 4)
