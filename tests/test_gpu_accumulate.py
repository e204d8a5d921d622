"""hdr_accumulate against the accumulation restatements on crafted frames
(through the C ABI), bit for bit except NaN payloads.

Parity mode must equal the reference's in-place row-major clamp
(passes/accumulation_pass.cpp:22-60; the oracle's orc_accumulate, pinned to the
reference in tests/test_accumulate_oracle.py) including the frames where that
order and the shader's differ, which only the device's in-place fallback gets
right. Shader mode must equal accumulation.slang:55-97 (orc_accumulate_shader).
The frames hold chained clamps through infinite luminance, negative and NaN
luminance, fireflies on borders and corners, 1-pixel-wide and 1x1 frames.
"""
import numpy as np
import pytest

from hdrestir_b200 import configs
from oracle.oracle import accumulate_frame
from tests.accum_frames import SIZES, crafted_frames, same_or_both_nan

pytestmark = pytest.mark.gpu


def _sized_ctx(ctx, scene, w, h):
    """Makes "Color" exist at w x h on ctx (the accumulation reads the frame size
    the last raycast set)."""
    cam = configs.config_camera(0, w, h)
    ctx.raycast(cam, 0)
    ctx.path_trace(cam, 0, max_depth=1)
    ctx.clear_persistent()


@pytest.fixture(scope="module")
def scene0():
    sc, _ = configs.small_variant(0, 8, 8)
    return sc


@pytest.mark.parametrize("mode", ["parity", "shader"])
@pytest.mark.parametrize("size", SIZES + [(1920, 1080)])
def test_accumulate_matches_restatement(gpu_ctx, scene0, mode, size):
    w, h = size
    gpu_ctx.upload_scene(scene0)
    _sized_ctx(gpu_ctx, scene0, w, h)
    frames = crafted_frames(w, h, 3, seed=w * 7 + h)
    acc = np.zeros((w * h, 4), np.float32)
    for f, fr in enumerate(frames):
        gpu_ctx.upload("Color", fr)
        gpu_ctx.accumulate(f, firefly=True, mode=mode)
        got = gpu_ctx.download("Color").copy()
        got_acc = gpu_ctx.download("__accum_color").copy()
        want = fr.copy()
        accumulate_frame(want, acc, w, h, f, firefly=True, mode=mode)
        assert same_or_both_nan(got, want), f"{mode} {w}x{h} frame {f}: Color differs"
        assert same_or_both_nan(got_acc, acc), f"{mode} {w}x{h} frame {f}: __accum_color differs"


def test_parity_fallback_reached_and_firefly_off(gpu_ctx, scene0):
    """On a chained frame the two modes differ on the GPU as they do on the CPU
    (so parity mode really took the in-place fallback), and with the clamp off
    both modes are the plain running mean."""
    w, h = 64, 48
    gpu_ctx.upload_scene(scene0)
    fr = crafted_frames(w, h, 1, seed=3)[0]
    out = {}
    for mode in ("parity", "shader"):
        _sized_ctx(gpu_ctx, scene0, w, h)
        gpu_ctx.upload("Color", fr)
        gpu_ctx.accumulate(0, firefly=True, mode=mode)
        out[mode] = gpu_ctx.download("Color").copy()
    assert not same_or_both_nan(out["parity"], out["shader"])
    for mode in ("parity", "shader"):
        _sized_ctx(gpu_ctx, scene0, w, h)
        gpu_ctx.upload("Color", fr)
        gpu_ctx.accumulate(0, firefly=False, mode=mode)
        assert same_or_both_nan(gpu_ctx.download("Color"), fr)
