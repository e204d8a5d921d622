"""Live pin of the C oracle against the reference's own sources compiled in
place (oracle/_ref). Skipped where that library has not been built (it needs
the reference tree)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from hdrestir_b200 import configs
from oracle import oracle as orc
from oracle import refharness

pytestmark = pytest.mark.skipif(not refharness.available(), reason="oracle/_ref not built (needs the reference tree)")
REF_DIR = Path(refharness.__file__).resolve().parent / "_ref"


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


@pytest.mark.parametrize("name", ["test_reservoir", "test_rng", "test_camera"])
def test_reference_unit_tests_pass_on_the_shim(name):
    """The reference's own unit tests, built against the same shim the oracle build uses."""
    exe = REF_DIR / name
    if not exe.exists():
        pytest.skip(f"{name} not built")
    assert subprocess.run([str(exe)], timeout=120).returncode == 0


def test_rng_matches_reference_for_pixel_seeds():
    seeds = (np.arange(4096, dtype=np.uint64) ^ np.uint64((7 * 12345) & 0xFFFFFFFF)).astype(np.uint32)
    assert np.array_equal(bits(orc.rng_floats(seeds, 160)), bits(refharness.rng_floats(seeds, 160)))


@pytest.mark.parametrize("cfg,kw", [
    (0, dict(ris=False, max_depth=6)),
    (1, dict(ris=True, candidate_count=8, use_reservoir=True, skip_visibility=True, max_depth=1)),
    (2, dict(ris=True, candidate_count=4, use_reservoir=True, skip_visibility=False, max_depth=2)),
    (2, dict(ris=False, max_depth=3)),
])
def test_oracle_equals_reference(cfg, kw):
    extra = {1: dict(n_lights=64), 2: dict(grid=64, n_spheres=40, n_lights=100)}.get(cfg, {})
    sc, cam = configs.small_variant(cfg, 40, 30, **extra)
    ref = refharness.Reference(sc)
    o = orc.Oracle(sc, threads=4)
    for f in range(2):
        g, c, r = ref.render(cam, f, accumulate=True, firefly=True, **kw)
        assert np.array_equal(o.raycast(cam, f)["prim_id"], g["prim_id"])
        o.integrate(cam, f, **kw)
        o.accumulate(cam, f, firefly=True)
        assert np.array_equal(bits(o.color), bits(c))
        assert np.array_equal(o.res["m"], r["m"])


@pytest.mark.parametrize("hour", [6.5, 9.0, 12.0, 15.5, 17.9, 18.2, 2.0])
def test_physical_sky_equals_reference(hour):
    """PhysicalSky::Sample along 4000 directions and the sun of SampleDirect
    (direction, colour, or none after sunset), bit for bit."""
    sc, _ = configs.sky_variant(2, 16, 16, hour=hour, grid=32, n_spheres=4, n_lights=8)
    d = np.random.default_rng(int(hour * 10)).normal(size=(4000, 3)).astype(np.float32)
    a, sun_a = orc.Oracle(sc).sky(d)
    b, sun_b = refharness.Reference(sc).sky(d)
    assert np.array_equal(bits(a), bits(b))
    assert (sun_a is None) == (sun_b is None) == (hour in (18.2, 2.0))
    if sun_a is not None:
        assert np.array_equal(bits(sun_a), bits(sun_b))
        assert float(np.abs(a).max()) > 0.0


@pytest.mark.parametrize("hour", [15.5, 6.5])
@pytest.mark.parametrize("cfg,kw", [
    (2, dict(ris=True, candidate_count=8, use_reservoir=True, skip_visibility=False, max_depth=1)),
    (2, dict(ris=True, candidate_count=6, use_reservoir=True, skip_visibility=True, max_depth=1)),
    (1, dict(ris=True, candidate_count=9, use_reservoir=False, skip_visibility=False, max_depth=1)),
    (2, dict(ris=True, candidate_count=4, use_reservoir=True, skip_visibility=False, max_depth=2)),
    (2, dict(ris=False, max_depth=3)),
])
def test_oracle_equals_reference_under_the_physical_sky(hour, cfg, kw):
    """The environment outside the light sampler: RIS splits its candidates over
    three techniques (sampler NEE, sky NEE = the sun, BSDF), the path tracer adds a
    sun sample per vertex, misses see the sky. Colour bit for bit, reservoir M and
    winner light (the sun is light index len(lights)) over three frames of history."""
    extra = {1: dict(n_lights=64), 2: dict(grid=48, n_spheres=30, n_lights=60)}[cfg]
    sc, cam = configs.sky_variant(cfg, 40, 30, hour=hour, **extra)
    ref = refharness.Reference(sc)
    o = orc.Oracle(sc, threads=4)
    suns = 0
    for f in range(3):
        g, c, r = ref.render(cam, f, accumulate=True, firefly=True, **kw)
        assert np.array_equal(o.raycast(cam, f)["prim_id"], g["prim_id"])
        o.integrate(cam, f, **kw)
        o.accumulate(cam, f, firefly=True)
        assert np.array_equal(bits(o.color), bits(c))
        if kw.get("ris") and kw.get("use_reservoir"):
            assert np.array_equal(o.res["m"], r["m"])
            has = r["has_sample"] == 1
            assert np.array_equal(o.res["has_sample"], r["has_sample"])
            assert np.array_equal(o.res["light"][has], r["light"][has])
            suns += int((r["light"][has] == len(sc.lights)).sum())
    assert (g["hit"] == 0).any()  # the camera sees the sky
    if kw.get("ris") and kw.get("use_reservoir"):
        assert suns > 0  # the sun wins some reservoirs


def test_trace_rays_match_reference():
    sc, cam = configs.small_variant(2, 16, 16, grid=64, n_spheres=40, n_lights=50)
    rng = np.random.default_rng(3)
    o = rng.uniform(-15, 15, (2000, 3)) + np.array([0, 4.0, 0])
    d = rng.normal(size=(2000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    a = orc.Oracle(sc).trace_rays(rays)
    b = refharness.Reference(sc).trace_rays(rays)
    assert np.array_equal(a["prim_id"], b["prim_id"])
    hit = b["hit"] == 1
    assert hit.sum() > 100
    for field in ("position", "depth", "normal", "smooth_normal", "albedo"):
        assert np.array_equal(bits(a[field][hit]), bits(b[field][hit])), field


def test_reference_harness_survives_frame_size_changes():
    """A new frame size clears the persistent buffers before the passes index
    them (the reference renderer does the same), so the CPU baseline can sample
    several resolution levels with one scene."""
    sc, cam = configs.small_variant(2, 64, 48, grid=48, n_spheres=20, n_lights=100)
    ref = refharness.Reference(sc)
    for level in (2, 1, 0, 1):
        _, c, _ = ref.render(cam, 0, ris=True, candidate_count=8, use_reservoir=True, max_depth=1,
                             resolution_level=level, outputs=("color",))
        assert np.isfinite(c).all()
    ref.close()


@pytest.mark.parametrize("kw", [dict(ris=True, candidate_count=8, use_reservoir=True, max_depth=1),
                                dict(ris=False, max_depth=4)])
def test_oracle_equals_reference_with_dome(kw):
    """Config-3 family: rect lights plus a lat-long dome (DomeLight::Prepare CDF,
    Sample, EvalPdf, background)."""
    sc, cam, _ = configs.config3(40, 30, n_small=0, grid=48, n_spheres=20, n_lights=60, dome_size=(64, 32))
    ref = refharness.Reference(sc)
    o = orc.Oracle(sc, threads=4)
    for f in range(2):
        g, c, r = ref.render(cam, f, accumulate=True, firefly=True, **kw)
        o.raycast(cam, f)
        o.integrate(cam, f, **kw)
        o.accumulate(cam, f, firefly=True)
        assert np.array_equal(bits(o.color), bits(c))
        assert np.array_equal(o.res["m"], r["m"])


@pytest.mark.parametrize("kw", [dict(ris=True, candidate_count=8, use_reservoir=True, max_depth=1),
                                dict(ris=True, candidate_count=8, use_reservoir=False, skip_visibility=True,
                                     max_depth=1),
                                dict(ris=False, max_depth=4)])
def test_oracle_equals_reference_with_point_and_distant_lights(kw):
    """Rect, point (cone-shaped, soft and hard edges) and distant lights (PointLight,
    DistantLight: SampleLight, EvalPdf, delta handling in NEE and MIS)."""
    sc, cam = configs.mixed_lights(40, 30)
    ref = refharness.Reference(sc)
    o = orc.Oracle(sc, threads=4)
    for f in range(2):
        g, c, r = ref.render(cam, f, accumulate=True, firefly=True, **kw)
        o.raycast(cam, f)
        o.integrate(cam, f, **kw)
        o.accumulate(cam, f, firefly=True)
        assert np.array_equal(bits(o.color), bits(c))
        assert np.array_equal(o.res["m"], r["m"])
        assert float(c[:, :3].mean()) > 0.0


CAMERA_PARAMS = [
    dict(enable_dof=1, focal_length=50.0, f_stop=1.4, focus_distance=9.0, bokeh_blades=0),
    dict(enable_dof=1, focal_length=35.0, f_stop=2.0, focus_distance=7.5, bokeh_blades=6),
    dict(lens_distortion=-0.15),
    dict(enable_exposure=1, f_stop=4.0, iso=400.0, shutter_speed=0.01),
]


@pytest.mark.parametrize("params", CAMERA_PARAMS)
def test_oracle_equals_reference_with_camera_params(params):
    """GenerateCameraRay with thin-lens depth of field (disc and polygonal bokeh), lens
    distortion, and the exposure multiplier (scene/camera_ray.cpp, camera_params.h)."""
    from hdrestir_b200.scene import make_camera
    sc, _ = configs.small_variant(1, 40, 30, n_lights=64)
    cam = make_camera((0.0, 6.0, 9.0), (0.0, 0.0, 0.0), 40, 30, fov=55.0, params=params)
    kw = dict(ris=True, candidate_count=8, use_reservoir=True, max_depth=1)
    ref = refharness.Reference(sc)
    o = orc.Oracle(sc, threads=4)
    for f in range(2):
        g, c, r = ref.render(cam, f, accumulate=True, firefly=True, **kw)
        assert np.array_equal(o.raycast(cam, f)["prim_id"], g["prim_id"])
        o.integrate(cam, f, **kw)
        o.accumulate(cam, f, firefly=True)
        assert np.array_equal(bits(o.color), bits(c))


@pytest.mark.parametrize("kw", [dict(ris=True, candidate_count=8, use_reservoir=True, max_depth=3),
                                dict(ris=False, max_depth=6)])
def test_oracle_equals_reference_translucent(kw):
    """Partial opacity (stochastic skip of a hit), Beer absorption and thin-walled transmission
    (PathIntegrator::Li opacity loop, BeerAbsorption, PreviewSurface refraction)."""
    sc, cam = configs.translucent_variant(40, 30)
    ref = refharness.Reference(sc)
    o = orc.Oracle(sc, threads=4)
    for f in range(2):
        g, c, r = ref.render(cam, f, accumulate=True, firefly=True, **kw)
        assert np.array_equal(o.raycast(cam, f)["prim_id"], g["prim_id"])
        o.integrate(cam, f, **kw)
        o.accumulate(cam, f, firefly=True)
        assert np.array_equal(bits(o.color), bits(c))
        assert np.array_equal(o.res["m"], r["m"])


@pytest.mark.parametrize("kw", [dict(ris=True, candidate_count=8, use_reservoir=True, max_depth=1),
                                dict(ris=False, max_depth=4)])
def test_oracle_equals_reference_textured(kw):
    """PreviewSurface textures: diffuse, metallic, roughness and normal maps, sampled by the
    reference's own BoundTextureSampler from texels its ImageTextureSamplerFactory loads
    (preview_surface.cpp:68-95, image_texture_sampler.h:41-68)."""
    import dataclasses

    from hdrestir_b200.scene import TEXTURE_FIELDS

    sc, cam = configs.textured_variant(40, 30)
    ref = refharness.Reference(sc)
    o = orc.Oracle(sc, threads=4)
    for f in range(2):
        g, c, r = ref.render(cam, f, accumulate=True, firefly=True, **kw)
        assert np.array_equal(o.raycast(cam, f)["prim_id"], g["prim_id"])
        o.integrate(cam, f, **kw)
        o.accumulate(cam, f, firefly=True)
        assert np.array_equal(bits(o.color), bits(c))
        assert np.array_equal(o.res["m"], r["m"])
    # the textures take effect on both sides
    plain = dataclasses.replace(sc, materials=[dataclasses.replace(m, **{k: None for k in TEXTURE_FIELDS})
                                               for m in sc.materials])
    _, c_plain, _ = refharness.Reference(plain).render(cam, 1, accumulate=True, firefly=True, **kw)
    assert np.abs(c_plain[..., :3] - c[..., :3]).mean() > 1e-3 * np.abs(c[..., :3]).mean()
