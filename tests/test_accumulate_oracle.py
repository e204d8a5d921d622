"""The accumulation pass's CPU restatements, pinned.

* oracle parity mode (``orc_accumulate``) against the reference's own
  AccumulationPass (passes/accumulation_pass.cpp:22-139) compiled in place,
  bit for bit, on crafted frames: chained clamps through infinite luminance,
  negative and NaN luminance, fireflies on borders and corners, 1-pixel-wide
  frames;
* oracle shader mode (``orc_accumulate_shader``) against an independent numpy
  restatement of accumulation.slang:55-97 (every pixel clamped against the
  unclamped input), since the shader itself needs a graphics API.
"""
import numpy as np
import pytest

from oracle import refharness
from oracle.oracle import accumulate_frame
from tests.accum_frames import SIZES, crafted_frames, same_or_both_nan


def _lum(c):
    return np.float32(0.2126) * c[..., 0] + np.float32(0.7152) * c[..., 1] + np.float32(0.0722) * c[..., 2]


def numpy_shader(color, accum, width, height, frame, firefly=True):
    """accumulation.slang cs_main for every pixel, in float32 numpy."""
    img = color.reshape(height, width, 4)
    out = img.copy()
    if firefly:
        lum = _lum(img)
        with np.errstate(invalid="ignore"):
            mx = np.zeros((height, width), np.float32)
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    if dx == 0 and dy == 0:
                        continue
                    ys = np.clip(np.arange(height) + dy, 0, height - 1)
                    xs = np.clip(np.arange(width) + dx, 0, width - 1)
                    nb = lum[ys][:, xs]
                    mx = np.where(mx < nb, nb, mx)  # max(a, b) = a < b ? b : a
            thr = mx * np.float32(4.0) + np.float32(0.5)
            clamp = (lum > thr) & (lum > np.float32(0.0))
            scale = np.where(clamp, thr / np.where(clamp, lum, np.float32(1.0)), np.float32(1.0)).astype(np.float32)
            out[..., :3] = np.where(clamp[..., None], img[..., :3] * scale[..., None], img[..., :3])
    inv = np.float32(1.0) / np.float32(frame + 1)
    acc = accum.reshape(height, width, 4) + out
    accum[:] = acc.reshape(-1, 4)
    color[:] = (acc * inv).reshape(-1, 4)


@pytest.mark.parametrize("size", SIZES)
def test_shader_restatement_pinned_to_numpy(size):
    w, h = size
    frames = crafted_frames(w, h, 3, seed=w * 131 + h)
    acc_c = np.zeros((w * h, 4), np.float32)
    acc_n = np.zeros((w * h, 4), np.float32)
    for f, fr in enumerate(frames):
        a, b = fr.copy(), fr.copy()
        accumulate_frame(a, acc_c, w, h, f, firefly=True, mode="shader")
        with np.errstate(invalid="ignore"):
            numpy_shader(b, acc_n, w, h, f)
        assert same_or_both_nan(a, b), f"frame {f}"
        assert same_or_both_nan(acc_c, acc_n), f"frame {f}"


@pytest.mark.skipif(not refharness.available(), reason="reference library not built (needs the reference tree)")
@pytest.mark.parametrize("size", SIZES + [(128, 96)])
@pytest.mark.parametrize("firefly", [True, False])
def test_parity_restatement_pinned_to_reference(size, firefly):
    w, h = size
    frames = crafted_frames(w, h, 3, seed=w * 7 + h)
    acc_o = np.zeros((w * h, 4), np.float32)
    acc_r = np.zeros((w * h, 4), np.float32)
    for f, fr in enumerate(frames):
        a, b = fr.copy(), fr.copy()
        accumulate_frame(a, acc_o, w, h, f, firefly=firefly, mode="parity")
        refharness.accumulate(b, acc_r, w, h, f, firefly=firefly)
        # same host arithmetic (x86, no contraction), so NaN payloads agree too
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"frame {f}"
        assert np.array_equal(acc_o.view(np.uint32), acc_r.view(np.uint32)), f"frame {f}"


def test_chained_frames_separate_the_two_orders():
    """The crafted chains make the in-place order and the shader differ, so the
    GPU tests that use them exercise the device's in-place fallback."""
    w, h = 64, 48
    fr = crafted_frames(w, h, 1, seed=3)[0]
    a, b = fr.copy(), fr.copy()
    accumulate_frame(a, np.zeros_like(a), w, h, 0, mode="parity")
    accumulate_frame(b, np.zeros_like(b), w, h, 0, mode="shader")
    assert not same_or_both_nan(a, b)
    plain = crafted_frames(w, h, 1, seed=3, chains=False)[0]
    plain[~np.isfinite(plain)] = 0.0
    a, b = plain.copy(), plain.copy()
    accumulate_frame(a, np.zeros_like(a), w, h, 0, mode="parity")
    accumulate_frame(b, np.zeros_like(b), w, h, 0, mode="shader")
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), "finite frames: both orders agree"
