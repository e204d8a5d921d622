"""Render-buffer conversion (HdRestirRenderBuffer::_WriteOutput,
hydra/hd_restir_render_buffer.cpp:46-73): the CPU restatement pinned to the
reference's own render buffer compiled in place, its known answers, and
hdr_resolve on the GPU against it, bit for bit, to host and device memory."""
import numpy as np
import pytest

from oracle import refharness
from oracle import render_buffer as rb

_TYPES = {rb.FLOAT32: "float32", rb.FLOAT16: "float16", rb.UNORM8: "unorm8", rb.SNORM8: "snorm8", rb.INT32: "int32"}


def _edge_values(rng, n):
    """Random values plus the edges of every conversion: the clamps, the unorm/snorm
    rounding steps, half-precision ties, subnormals, overflow and infinities."""
    v = [rng.normal(0.0, 2.0, n), rng.uniform(-1.5, 1.5, n), 10.0 ** rng.uniform(-9, 6, n) * rng.choice([-1, 1], n)]
    steps = np.arange(-130, 260) / 255.0
    ties = (np.arange(2048, 4096, dtype=np.float64) + 0.5) * 2.0 ** -11  # exact half-way between halves
    sub = np.array([2.0 ** -25, 2.0 ** -24, 1.5 * 2.0 ** -24, 2.0 ** -14, 65504.0, 65520.0, 65519.0, 1e9,
                    np.inf, -np.inf, 0.0, -0.0])
    flat = np.concatenate(v + [steps, -steps, ties, -ties, sub]).astype(np.float32)
    k = -(-len(flat) // 4) * 4
    return np.resize(flat, k).reshape(-1, 4)


@pytest.mark.skipif(not refharness.available(), reason="reference library not built (needs the reference tree)")
@pytest.mark.parametrize("fmt", [rb.FLOAT32, rb.FLOAT16, rb.UNORM8, rb.SNORM8, rb.INT32])
def test_restatement_pinned_to_reference_render_buffer(fmt):
    """oracle/render_buffer.py against the reference's own HdRestirRenderBuffer
    (hydra/hd_restir_render_buffer.cpp, compiled in place against the HdFormat and
    GfHalf stand-ins): CopyFromFrameBuffer from 1-, 3- and 4-component float
    buffers into 1..4-component render buffers, then Resolve, bit for bit. NaN and
    int32 out of range (undefined in the reference's casts) stay out."""
    rng = np.random.default_rng(fmt)
    vals = _edge_values(rng, 4000)
    if fmt == rb.INT32:
        vals = np.clip(np.nan_to_num(vals, posinf=2e9, neginf=-2e9), -2e9, 2e9).astype(np.float32)
    checked = 0
    for src in (1, 3, 4):
        v = np.ascontiguousarray(vals[:, :src])
        for comps in (1, 2, 3, 4):
            same_stride = src * 4 == comps * rb._COMPONENT_BYTES[fmt]
            if src > 1 and not same_stride:
                # the conversion path reads the frame buffer with As<const float>(), whose
                # precondition (a 4-byte stride) stops the reference program here
                continue
            want = refharness.resolve(v, _TYPES[fmt], comps)
            got = rb.copy_from_frame_buffer(v, fmt, comps)
            assert got.dtype == want.dtype, (src, comps)
            assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), (src, comps)
            checked += 1
    assert checked >= 4


def test_known_answers():
    v = np.array([[0.5, 1.2, -0.1, 2.0], [0.999, -1.5, 0.0039, 1.0]], np.float32)
    assert rb.write_output(v, rb.UNORM8, 4).tolist() == [[127, 255, 0, 255], [254, 0, 0, 255]]
    assert rb.write_output(v, rb.SNORM8, 4).tolist() == [[63, 127, -12, 127], [126, -128, 0, 127]]
    assert rb.write_output(v, rb.INT32, 4).tolist() == [[0, 1, 0, 2], [0, -1, 0, 1]]
    h = rb.write_output(v, rb.FLOAT16, 2)
    assert h.dtype == np.uint16 and h[0, 0] == 0x3800 and h[0, 1] == np.float16(1.2).view(np.uint16)
    # components the source lacks are 0; extra source components are dropped
    assert rb.write_output(v[:, :1], rb.FLOAT32, 3).tolist() == [[0.5, 0.0, 0.0], [0.9990000128746033, 0.0, 0.0]]
    assert rb.write_output(v, rb.UNORM8, 1).shape == (2, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("fmt,comps", [(rb.FLOAT32, 4), (rb.FLOAT16, 4), (rb.UNORM8, 4), (rb.SNORM8, 3),
                                       (rb.INT32, 1), (rb.UNORM8, 1)])
def test_resolve_matches_write_output(fmt, comps):
    import torch
    from hdrestir_b200 import abi, configs
    from hdrestir_b200.context import Context
    sc, cam = configs.small_variant(0, 64, 48)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        ctx.raycast(cam, 0, aovs=("Depth", "Normal"))
        ctx.path_trace(cam, 0, max_depth=3)
        for name, src in (("Color", 4), ("Depth", 1), ("Normal", 3)):
            vals = ctx.download(name).reshape(-1, src).astype(np.float32)
            if name == "Color":
                vals = vals * np.float32(3.0) - np.float32(0.5)  # exercise both clamps
                ctx.upload(name, np.ascontiguousarray(vals))
            want = rb.copy_from_frame_buffer(vals, fmt, comps)
            got = ctx.resolve(name, src, fmt, comps)
            assert got.dtype == want.dtype and np.array_equal(got, want), name
            dev = torch.empty(want.nbytes, dtype=torch.uint8, device="cuda:0")
            ctx.resolve(name, src, fmt, comps, device_ptr=dev.data_ptr())
            ctx.synchronize()
            assert np.array_equal(dev.cpu().numpy().view(want.dtype).reshape(want.shape), want), name
        for bad in ("GBuffer", "__ris_reservoir", "NoSuchBuffer"):  # not float frame buffers
            with pytest.raises(abi.HdrError):
                ctx.resolve(bad, 4, fmt, comps)
