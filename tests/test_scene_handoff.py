"""The scene hand-off (hdrestir_b200/integration/scene_handoff.h) on the host:
fed only the reference Scene's inputs (AddMesh / SetMaterialParams /
SetLightFactoryInput, scene/scene.cpp:50-92) that the prims of a scene
description make, it builds that description again: per instance the same mesh
arrays, transform, material and light link (Scene::BuildRenderState's instance
order, scene.cpp:174-238); materials and lights field for field, in SdfPath
order; textures through the loader."""
import pytest

from hdrestir_b200 import configs
from oracle import refharness

pytestmark = pytest.mark.skipif(not refharness.gpu_pipeline_available(),
                                reason="reference build with the GPU passes not present")


@pytest.mark.parametrize("make", [
    lambda: configs.small_variant(0, 32, 32)[0],
    lambda: configs.small_variant(1, 32, 32, n_lights=64)[0],
    lambda: configs.small_variant(2, 32, 32, grid=48, n_spheres=30, n_lights=100)[0],
    lambda: configs.textured_variant(32, 32)[0],
    lambda: configs.mixed_lights(32, 32)[0],
])
def test_handoff_rebuilds_the_description(make):
    assert refharness.handoff_compare(make()) == 0
