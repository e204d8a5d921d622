"""Post passes: UpscalePass (passes/upscale_pass.cpp) and the Denoiser without OIDN
(passes/denoiser.cpp). The CPU restatement is pinned to the reference's own passes
compiled in place; the device kernels (hdr_upscale, hdr_denoise) must equal it bit
for bit."""
import numpy as np
import pytest

from oracle import post, refharness

needs_ref = pytest.mark.skipif(not refharness.available(), reason="reference build not present")
COMPS = {"Color": 4, "Albedo": 3, "Depth": 1}


def _image(n, comps, seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-0.5, 8.0, (n, comps)).astype(np.float32)
    a[rng.random(n) < 0.01] *= np.float32(1000.0)  # a few fireflies
    return a


@needs_ref
@pytest.mark.parametrize("name", list(COMPS))
@pytest.mark.parametrize("level,w,h", [(1, 64, 48), (2, 97, 61), (3, 33, 130), (4, 200, 7)])
def test_upscale_restatement_matches_reference(name, level, w, h):
    sw, sh = post.rendered_size(w, level), post.rendered_size(h, level)
    src = _image(sw * sh, COMPS[name], level)
    want = refharness.upscale(name, src, w, h, level)
    got = post.upscale_nearest(src, sw, sh, w, h)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@needs_ref
@pytest.mark.parametrize("w,h", [(64, 48), (1, 1), (3, 17), (130, 2)])
def test_chroma_blur_restatement_matches_reference(w, h):
    img = _image(w * h, 4, w * 1000 + h)
    want = refharness.denoise(img, w, h)
    got = post.chroma_blur(img, w, h)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.array_equal(refharness.denoise(img, w, h, chromaticity_blur=False).view(np.uint32), img.view(np.uint32))


@pytest.mark.gpu
def test_device_post_passes_match_restatement():
    from hdrestir_b200 import abi
    from hdrestir_b200.context import Context
    with Context(device=0) as ctx:
        for name, level, w, h in (("Color", 1, 1920, 1080), ("Albedo", 2, 97, 61), ("Depth", 3, 33, 130)):
            sw, sh = post.rendered_size(w, level), post.rendered_size(h, level)
            src = _image(sw * sh, COMPS[name], level)
            ctx.upload(name, np.ascontiguousarray(src))  # creates the buffer at the rendered size
            ctx.upscale(name, COMPS[name], sw, sh, w, h)
            got = ctx.download(name).reshape(-1, COMPS[name])
            assert np.array_equal(got.view(np.uint32), post.upscale_nearest(src, sw, sh, w, h).view(np.uint32))
        for w, h in ((1920, 1080), (3, 17), (1, 1)):
            img = _image(w * h, 4, w + h)
            ctx.upload("Color", np.ascontiguousarray(img))
            ctx.denoise("Color", w, h)
            got = ctx.download("Color").reshape(-1, 4)
            assert np.array_equal(got.view(np.uint32), post.chroma_blur(img, w, h).view(np.uint32)), (w, h)
        with pytest.raises(abi.HdrError):
            ctx.denoise("Color", 2, 2)  # the buffer is not 2 x 2 RGBA
        with pytest.raises(abi.HdrError):
            ctx.upscale("Color", 4, 5, 5, 10, 10)

