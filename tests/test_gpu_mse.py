"""Equal MSE: after N accumulated frames, the GPU image and the reference's own
CPU image (compiled in place) are equally far from a high-spp image of the same
estimator, for the ReSTIR and the PathTracer pipelines, and the batched form
gives the plain form's MSE."""
import numpy as np
import pytest

from hdrestir_b200 import configs
from hdrestir_b200.context import Context, ris_path_trace_batch
from oracle import refharness

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refharness.available(), reason="reference build not present")]

N_FRAMES = 12
HIGH_SPP = 384


def _gpu_frames(scene, cam, frames, pipeline, kw, start=0):
    with Context(device=0) as ctx:
        ctx.upload_scene(scene)
        for f in range(start, start + frames):
            ctx.raycast(cam, f)
            if pipeline == "ris":
                ctx.ris_path_trace(cam, f, **kw)
            else:
                ctx.path_trace(cam, f, **kw)
            ctx.accumulate(f - start)
        return ctx.download("Color")[:, :3].astype(np.float64)


def _mse(img, ref):
    peak = max(float(ref.max()), 1e-12)  # normalised by the reference's peak
    return float(np.mean(((img - ref) / peak) ** 2))


@pytest.mark.parametrize("pipeline,kw", [
    ("ris", dict(candidate_count=16, use_reservoir=True, max_depth=1)),
    ("pt", dict(max_depth=3)),
])
def test_gpu_and_reference_reach_equal_mse(pipeline, kw):
    scene, cam = configs.small_variant(2, 48, 32, grid=64, n_spheres=40, n_lights=200)
    # high-spp image: frames N.. of an independent run (other RNG streams than the N-frame images)
    high = _gpu_frames(scene, cam, HIGH_SPP, pipeline, kw, start=10_000)
    gpu = _gpu_frames(scene, cam, N_FRAMES, pipeline, kw)
    ref = refharness.Reference(scene)
    for f in range(N_FRAMES):
        _, col, _ = ref.render(cam, f, ris=(pipeline == "ris"), accumulate=True, firefly=True,
                               outputs=("color",), **kw)
    ref.close()
    cpu = col[:, :3].astype(np.float64)
    m_gpu, m_cpu = _mse(gpu, high), _mse(cpu, high)
    print(f"{pipeline}: MSE gpu {m_gpu:.6e} cpu {m_cpu:.6e}")
    assert m_gpu > 0.0
    assert abs(m_gpu - m_cpu) <= 1e-3 * m_cpu


def test_batched_form_has_the_plain_mse():
    scene, _ = configs.small_variant(2, 48, 32, grid=64, n_spheres=40, n_lights=200)
    cams = [configs.orbit_camera(0.5 * k, 48, 32) for k in range(3)]
    ris = dict(candidate_count=16, use_reservoir=True, max_depth=1)
    plain = [_gpu_frames(scene, c, N_FRAMES, "ris", ris) for c in cams]
    ctxs = [Context(device=0) for _ in cams]
    try:
        ctxs[0].upload_scene(scene)
        for c in ctxs[1:]:
            c.share_scene(ctxs[0])
        for f in range(N_FRAMES):
            for c, cam in zip(ctxs, cams):
                c.raycast(cam, f)
            ris_path_trace_batch(ctxs, cams, [f] * 3, **ris)
            for c in ctxs:
                c.accumulate(f)
        batched = [c.download("Color")[:, :3].astype(np.float64) for c in ctxs]
    finally:
        for c in ctxs:
            c.close()
    for p, b in zip(plain, batched):
        assert np.array_equal(p, b)  # identical images, hence identical MSE against any reference
