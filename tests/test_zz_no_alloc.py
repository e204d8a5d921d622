"""hdr_accumulate_noalloc (static device scratch, no allocation) against
hdr_accumulate and the accumulation restatements on the same inputs, through
the C ABI. Some hosts cannot allocate device memory while they accumulate (a
renderer running inside its own memory pool, or one that must not pay the
device-wide synchronisation of cudaMalloc/cudaFree between frames); this entry
point serves them from a fixed static array. Kept in a file that sorts last so
it also runs after every other GPU test in one session."""
import ctypes as C

import numpy as np
import pytest

from hdrestir_b200 import abi, configs
from oracle.oracle import accumulate_frame
from tests.accum_frames import crafted_frames, same_or_both_nan

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


def _noalloc(color, accum, w, h, frame, firefly, mode):
    import torch
    stream = torch.cuda.current_stream(color.device)
    return abi.lib().hdr_accumulate_noalloc(C.c_void_p(color.data_ptr()), C.c_void_p(accum.data_ptr()), w, h,
                                            frame, int(firefly), mode, C.c_void_p(stream.cuda_stream))


def _mode(name):
    return {"parity": abi.ACCUM_PARITY, "shader": abi.ACCUM_SHADER}[name]


@pytest.mark.parametrize("mode", ["parity", "shader"])
@pytest.mark.parametrize("crafted", [False, True])
def test_noalloc_matches_hdr_accumulate(mode, crafted):
    """Two calls in a row equal hdr_accumulate's two frames bit for bit (NaNs by
    position); the crafted frames (chained clamps through infinite luminance,
    negative and NaN luminance) also take parity mode's in-place fallback."""
    import torch

    from hdrestir_b200.context import Context

    sc, cam = configs.small_variant(0, 64, 48)
    w, h = cam.width, cam.height
    frames = crafted_frames(w, h, 2, seed=0xACC) if crafted else _frames(w * h, np.random.default_rng(0xACC))

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

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    accum = torch.zeros((w * h, 4), dtype=torch.float32, device=dev)
    acc_o = np.zeros((w * h, 4), np.float32)
    for f, c in enumerate(frames):
        color = torch.from_numpy(c).to(dev)
        torch.cuda.synchronize(dev)
        abi.check(_noalloc(color, accum, w, h, f, True, _mode(mode)))
        torch.cuda.synchronize(dev)
        got_color, got_accum = color.cpu().numpy(), accum.cpu().numpy()
        want_color, want_accum = want[f]
        assert same_or_both_nan(got_color, want_color), f"frame {f}: Color differs"
        assert same_or_both_nan(got_accum, want_accum), f"frame {f}: accum differs"
        ref = c.copy()
        accumulate_frame(ref, acc_o, w, h, f, firefly=True, mode=mode)
        assert same_or_both_nan(got_color, ref), f"frame {f}: Color differs from the restatement"


def test_noalloc_at_the_limit_and_without_the_clamp():
    """A frame of exactly 2^21 pixels with the clamp (the limit), and a larger
    one without it (the scratch is not used, so any size is accepted), each over
    two calls; free device memory does not change across the calls."""
    import torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    one = torch.zeros((1, 4), dtype=torch.float32, device=dev)
    abi.check(_noalloc(one, one.clone(), 1, 1, 0, True, abi.ACCUM_PARITY))  # loads the module, resolves the scratch
    cases = [(2048, 1024, True, "parity"), (2048, 1024, True, "shader"), (2048, 1025, False, "parity")]
    bufs = []
    for w, h, firefly, mode in cases:
        frames = crafted_frames(w, h, 2, seed=w + h + firefly, chains=True)
        bufs.append(([torch.from_numpy(f).to(dev) for f in frames],
                     torch.zeros((w * h, 4), dtype=torch.float32, device=dev), frames))
    torch.cuda.synchronize(dev)
    free_before, _ = torch.cuda.mem_get_info(dev)
    for (w, h, firefly, mode), (colors, accum, _) in zip(cases, bufs):
        for f, color in enumerate(colors):
            abi.check(_noalloc(color, accum, w, h, f, firefly, _mode(mode)))
    torch.cuda.synchronize(dev)
    free_after, _ = torch.cuda.mem_get_info(dev)
    assert free_after == free_before, "the entry point allocated device memory"
    for (w, h, firefly, mode), (colors, accum, frames) in zip(cases, bufs):
        acc = np.zeros((w * h, 4), np.float32)
        for f, (color, fr) in enumerate(zip(colors, frames)):
            want = fr.copy()
            accumulate_frame(want, acc, w, h, f, firefly=firefly, mode=mode)
            assert same_or_both_nan(color.cpu().numpy(), want), f"{w}x{h} {mode} frame {f}"
        assert same_or_both_nan(accum.cpu().numpy(), acc)


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
    assert L.hdr_accumulate_noalloc(p, p, 4, 4, 0, 1, 7, None) == abi.HDR_EINVAL
    assert 2048 * 1025 > MAX_PIXELS
