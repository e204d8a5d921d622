"""CPU restatement of HdRestirRenderBuffer::CopyFromFrameBuffer and its
_WriteOutput — TEST INFRASTRUCTURE.

Only tests/ import this module, as the checker of hdr_resolve. It restates
hydra/hd_restir_render_buffer.cpp:46-73 (the per-component conversion) and
:113-148 (CopyFromFrameBuffer: a raw byte copy when the frame buffer's stride
equals the render buffer's, else the conversion). Pinned bit for bit to the
reference's own render buffer compiled in place against the HdFormat and GfHalf
stand-ins (tests/test_render_buffer.py).
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


_COMPONENT_BYTES = {FLOAT32: 4, FLOAT16: 2, UNORM8: 1, SNORM8: 1, INT32: 4}
_DTYPES = {FLOAT32: np.float32, FLOAT16: np.uint16, UNORM8: np.uint8, SNORM8: np.int8, INT32: np.int32}


def copy_from_frame_buffer(values: np.ndarray, component_format: int, dst_components: int) -> np.ndarray:
    """CopyFromFrameBuffer (hd_restir_render_buffer.cpp:113-148): when a pixel of the
    frame buffer (source components x 4 bytes) has the render buffer's size the
    bytes are copied as they are, otherwise each pixel goes through _WriteOutput."""
    values = np.ascontiguousarray(values, np.float32)
    pixels, src = values.shape
    if src * 4 == dst_components * _COMPONENT_BYTES[component_format]:
        return values.view(np.uint8).view(_DTYPES[component_format]).reshape(pixels, dst_components).copy()
    return write_output(values, component_format, dst_components)
