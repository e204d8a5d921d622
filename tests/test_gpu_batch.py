"""Batched RIS frames (several images, one shared scene, one trace launch) give
each image exactly what rendering it alone gives; scene sharing keeps the
scene alive for every context that holds it."""
import numpy as np
import pytest

from hdrestir_b200 import abi, configs
from hdrestir_b200.context import Context, ris_path_trace_batch

pytestmark = pytest.mark.gpu

RIS = dict(candidate_count=32, use_reservoir=True, max_depth=1)
SIZES = ((96, 64), (64, 64), (128, 72))


def _scene():
    sc, _ = configs.small_variant(2, 64, 64, grid=96, n_spheres=60, n_lights=300)
    cams = [configs.orbit_camera(0.7 * k, w, h) for k, (w, h) in enumerate(SIZES)]
    return sc, cams


def _alone(sc, cams, frames, ris):
    out = []
    for cam in cams:
        with Context(device=0) as ctx:
            ctx.upload_scene(sc)
            for f in range(frames):
                ctx.raycast(cam, f)
                ctx.ris_path_trace(cam, f, **ris)
                ctx.accumulate(f)
            res = ctx.download("__ris_reservoir").copy() if ris.get("use_reservoir") else None
            out.append((ctx.download("Color").copy(), res))
    return out


def _batched(sc, cams, frames, ris):
    ctxs = [Context(device=0) for _ in cams]
    try:
        ctxs[0].upload_scene(sc)
        for c in ctxs[1:]:
            c.share_scene(ctxs[0])
        for f in range(frames):
            for c, cam in zip(ctxs, cams):
                c.raycast(cam, f)
            ris_path_trace_batch(ctxs, cams, [f] * len(cams), **ris)
            for c in ctxs:
                c.accumulate(f)
        return [(c.download("Color").copy(), c.download("__ris_reservoir").copy() if ris.get("use_reservoir")
                 else None) for c in ctxs]
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("ris", [RIS, dict(candidate_count=16, use_reservoir=False, max_depth=1),
                                 dict(candidate_count=8, use_reservoir=True, max_depth=2)])
def test_batch_equals_images_rendered_alone(ris):
    sc, cams = _scene()
    want = _alone(sc, cams, 2, ris)
    got = _batched(sc, cams, 2, ris)
    for (wc, wr), (gc, gr) in zip(want, got):
        assert np.array_equal(gc.view(np.uint32), wc.view(np.uint32))
        if wr is not None:
            assert np.array_equal(gr.view(np.uint32), wr.view(np.uint32))


def test_shared_scene_outlives_its_uploader():
    sc, cams = _scene()
    want = _alone(sc, cams[:1], 1, RIS)[0][0]
    src, dst = Context(device=0), Context(device=0)
    src.upload_scene(sc)
    dst.share_scene(src)
    src.close()  # dst still holds the scene memory
    dst.raycast(cams[0], 0)
    dst.ris_path_trace(cams[0], 0, **RIS)
    dst.accumulate(0)
    got = dst.download("Color")
    dst.close()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_batch_rejects_a_context_twice():
    sc, cams = _scene()
    with Context(device=0) as c:
        c.upload_scene(sc)
        with pytest.raises(abi.HdrError) as e:
            ris_path_trace_batch([c, c], cams[:2], [0, 0], **RIS)
        assert e.value.status == abi.HDR_EINVAL
