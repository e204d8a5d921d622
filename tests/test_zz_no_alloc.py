"""hdr_accumulate_noalloc (static device scratch, no allocation) against
hdr_accumulate on the same inputs, through the C ABI. Kept in a file that
sorts last so it also runs after every other GPU test in one session."""
import ctypes as C

import numpy as np
import pytest

from hdrestir_b200 import abi, configs

pytestmark = pytest.mark.gpu

MAX_PIXELS = 1 << 21


def _frames(n_px, rng):
    """Two RGBA frames with fireflies (a few pixels far above their neighbours)."""
    out = []
    for _ in range(2):
        c = rng.random((n_px, 4), dtype=np.float32) * np.float32(0.8)
        spikes = rng.choice(n_px, size=max(1, n_px // 50), replace=False)
        c[spikes, :3] *= np.float32(200.0)
        out.append(c)
    return out


@pytest.mark.parametrize("mode", ["parity", "shader"])
def test_noalloc_matches_hdr_accumulate(mode):
    import torch

    from hdrestir_b200.context import Context

    sc, cam = configs.small_variant(0, 64, 48)
    w, h = cam.width, cam.height
    frames = _frames(w * h, np.random.default_rng(0xACC))
    m = {"parity": abi.ACCUM_PARITY, "shader": abi.ACCUM_SHADER}[mode]

    ctx = Context(device=0)
    try:
        ctx.upload_scene(sc)
        ctx.raycast(cam, 0)
        ctx.path_trace(cam, 0, max_depth=1)  # sizes "Color" for this frame
        want = []
        for f, c in enumerate(frames):
            ctx.upload("Color", c)
            ctx.accumulate(f, firefly=True, mode=mode)
            want.append((ctx.download("Color").copy(), ctx.download("__accum_color").copy()))
    finally:
        ctx.close()

    L = abi.lib()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    accum = torch.zeros((w * h, 4), dtype=torch.float32, device=dev)
    for f, c in enumerate(frames):
        color = torch.from_numpy(c).to(dev)
        torch.cuda.synchronize(dev)
        st = L.hdr_accumulate_noalloc(C.c_void_p(color.data_ptr()), C.c_void_p(accum.data_ptr()), w, h, f, 1, m,
                                      C.c_void_p(stream.cuda_stream))
        abi.check(st)
        torch.cuda.synchronize(dev)
        got_color, got_accum = color.cpu().numpy(), accum.cpu().numpy()
        want_color, want_accum = want[f]
        assert np.array_equal(got_color.view(np.uint32), want_color.view(np.uint32)), f"frame {f}: Color differs"
        assert np.array_equal(got_accum.view(np.uint32), want_accum.view(np.uint32)), f"frame {f}: accum differs"


def test_noalloc_rejects_oversize_and_bad_args():
    import torch

    L = abi.lib()
    dev = torch.device("cuda", 0)
    buf = torch.zeros((16, 4), dtype=torch.float32, device=dev)
    p = C.c_void_p(buf.data_ptr())
    # rejected on the host, before any launch: the firefly scratch holds 2^21 pixels
    st = L.hdr_accumulate_noalloc(p, p, 2048, 1025, 0, 1, abi.ACCUM_PARITY, None)
    assert st == abi.HDR_EINVAL
    assert b"exceeds the no-alloc firefly scratch" in L.hdr_last_error()
    assert L.hdr_accumulate_noalloc(None, p, 4, 4, 0, 1, abi.ACCUM_PARITY, None) == abi.HDR_EINVAL
    assert L.hdr_accumulate_noalloc(p, p, 0, 4, 0, 1, abi.ACCUM_PARITY, None) == abi.HDR_EINVAL
    assert L.hdr_accumulate_noalloc(p, p, 4, 4, -1, 1, abi.ACCUM_PARITY, None) == abi.HDR_EINVAL
    assert 2048 * 1025 > MAX_PIXELS
