"""Drop-in check: the reference's own RenderPipeline driving the GPU passes of
hdrestir_b200/integration/gpu_passes.h renders what the same pipeline renders
with the reference's CPU passes; with the scene hand-off of
hdrestir_b200/integration/scene_handoff.h the device scene is built only from
the reference's Scene inputs (AddMesh / SetMaterialParams /
SetLightFactoryInput), and the frames carry that reference Scene."""
import numpy as np
import pytest

from hdrestir_b200 import configs
from oracle import refharness

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (refharness.available() and refharness.gpu_pipeline_available()),
                                 reason="reference build with the GPU passes not present")]


@pytest.mark.parametrize("cfg,kw", [
    (2, dict(ris=True, candidate_count=32, use_reservoir=True, max_depth=1)),
    (1, dict(ris=True, candidate_count=16, use_reservoir=False, skip_visibility=True, max_depth=1)),
    (0, dict(ris=False, max_depth=4)),
])
def test_reference_pipeline_with_gpu_passes(cfg, kw):
    extra = {1: dict(n_lights=128), 2: dict(grid=96, n_spheres=60, n_lights=300)}.get(cfg, {})
    sc, cam = configs.small_variant(cfg, 48, 32, **extra)
    frames = 3
    gpu = refharness.gpu_pipeline_render(sc, cam, frames, **kw)
    ref = refharness.Reference(sc)
    for f in range(frames):
        _, cpu, _ = ref.render(cam, f, accumulate=True, firefly=True, **kw)
    a, b = gpu[:, :3].astype(np.float64), cpu[:, :3].astype(np.float64)
    bad = (np.abs(a - b) > 1e-6 + 1e-4 * np.maximum(np.abs(a), np.abs(b))).any(1).mean()
    print(f"cfg{cfg}: GPU-pass pipeline vs CPU pipeline, outlier fraction {bad:.4f}")
    assert bad <= 0.01


def test_reference_pipeline_with_gpu_upscale():
    """A pipeline rendering at resolution level 1 ends with GpuUpscalePass (UpscalePass on the
    device); its window-size "Color" is the CPU pipeline's image upscaled by the reference's own
    UpscalePass."""
    sc, cam = configs.small_variant(2, 48, 32, grid=96, n_spheres=60, n_lights=300)
    kw = dict(ris=True, candidate_count=32, use_reservoir=True, max_depth=1)
    frames, level = 2, 1
    gpu = refharness.gpu_pipeline_render(sc, cam, frames, resolution_level=level, **kw)
    ref = refharness.Reference(sc)
    for f in range(frames):
        _, cpu, _ = ref.render(cam, f, accumulate=True, firefly=True, resolution_level=level, **kw)
    want = refharness.upscale("Color", cpu, cam.width, cam.height, level)
    a, b = gpu[:, :3].astype(np.float64), want[:, :3].astype(np.float64)
    bad = (np.abs(a - b) > 1e-6 + 1e-4 * np.maximum(np.abs(a), np.abs(b))).any(1).mean()
    print(f"upscaled GPU-pass pipeline vs CPU pipeline + UpscalePass: outlier fraction {bad:.4f}")
    assert gpu.shape == (48 * 32, 4) and bad <= 0.01


@pytest.mark.parametrize("cfg,kw", [
    (2, dict(ris=True, candidate_count=32, use_reservoir=True, max_depth=1)),
    (0, dict(ris=False, max_depth=4)),
])
def test_scene_from_reference_scene_inputs(cfg, kw):
    """The device scene built from the reference Scene's inputs renders the image of the
    scene description they came from, bit for bit, and the CPU pipeline's within tolerance."""
    extra = {2: dict(grid=96, n_spheres=60, n_lights=300)}.get(cfg, {})
    sc, cam = configs.small_variant(cfg, 48, 32, **extra)
    frames = 2
    via_scene = refharness.gpu_pipeline_render(sc, cam, frames, via_scene=True, **kw)
    direct = refharness.gpu_pipeline_render(sc, cam, frames, **kw)
    assert np.array_equal(via_scene.view(np.uint32), direct.view(np.uint32))
    ref = refharness.Reference(sc)
    for f in range(frames):
        _, cpu, _ = ref.render(cam, f, accumulate=True, firefly=True, **kw)
    a, b = via_scene[:, :3].astype(np.float64), cpu[:, :3].astype(np.float64)
    bad = (np.abs(a - b) > 1e-6 + 1e-4 * np.maximum(np.abs(a), np.abs(b))).any(1).mean()
    assert bad <= 0.01
