"""CPU restatement of HdRestirRenderBuffer's _WriteOutput — TEST INFRASTRUCTURE.

Only tests/ import this module, as the checker of hdr_resolve. It restates
hydra/hd_restir_render_buffer.cpp:46-73 (the per-component conversion) as
CopyFromFrameBuffer (:113-148) applies it to a float frame buffer. Parity
unpinned: the reference's tests hold no render-buffer vectors and the Hydra
plugin needs OpenUSD, which is not built here; the known answers in
tests/test_render_buffer.py follow the source's arithmetic (float32 products,
std::clamp, truncating integer casts, GfHalf rounding to nearest even).
"""
from __future__ import annotations

import numpy as np

FLOAT32, FLOAT16, UNORM8, SNORM8, INT32 = 0, 1, 2, 3, 4


def _clamp(v: np.ndarray, lo: float, hi: float) -> np.ndarray:
    # std::clamp(v, lo, hi): (v < lo) ? lo : (hi < v) ? hi : v
    lo32, hi32 = np.float32(lo), np.float32(hi)
    return np.where(v < lo32, lo32, np.where(hi32 < v, hi32, v)).astype(np.float32)


def write_output(values: np.ndarray, component_format: int, dst_components: int) -> np.ndarray:
    """values: (pixels, source components) float32 -> (pixels, dst_components) in the format's
    dtype, component by component as _WriteOutput writes them (missing components are 0)."""
    values = np.asarray(values, np.float32)
    pixels, src = values.shape
    v = np.zeros((pixels, dst_components), np.float32)
    k = min(src, dst_components)
    v[:, :k] = values[:, :k]
    have = np.zeros(dst_components, bool)
    have[:k] = True
    with np.errstate(invalid="ignore", over="ignore"):
        if component_format == FLOAT32:
            out = v.copy()
        elif component_format == FLOAT16:
            out = v.astype(np.float16).view(np.uint16)
        elif component_format == UNORM8:
            out = np.trunc(_clamp(v * np.float32(255.0), 0.0, 255.0)).astype(np.uint8)
        elif component_format == SNORM8:
            out = np.trunc(_clamp(v * np.float32(127.0), -128.0, 127.0)).astype(np.int8)
        elif component_format == INT32:
            out = np.trunc(v).astype(np.int32)
        else:
            raise ValueError(f"unknown component format {component_format}")
    out[:, ~have] = 0
    return out
