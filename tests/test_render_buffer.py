"""Render-buffer conversion (HdRestirRenderBuffer::_WriteOutput,
hydra/hd_restir_render_buffer.cpp:46-73): known answers of the CPU restatement,
and hdr_resolve on the GPU against it, bit for bit, to host and device memory."""
import numpy as np
import pytest

from oracle import render_buffer as rb


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
            want = rb.write_output(vals, fmt, comps)
            got = ctx.resolve(name, src, fmt, comps)
            assert got.dtype == want.dtype and np.array_equal(got, want), name
            dev = torch.empty(want.nbytes, dtype=torch.uint8, device="cuda:0")
            ctx.resolve(name, src, fmt, comps, device_ptr=dev.data_ptr())
            ctx.synchronize()
            assert np.array_equal(dev.cpu().numpy().view(want.dtype).reshape(want.shape), want), name
        for bad in ("GBuffer", "__ris_reservoir", "NoSuchBuffer"):  # not float frame buffers
            with pytest.raises(abi.HdrError):
                ctx.resolve(bad, 4, fmt, comps)
