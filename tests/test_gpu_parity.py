"""Parity of the CUDA passes (through the C ABI) with the CPU oracle.

Integer / index / hit results must be bit-identical (closest-hit instance and
triangle, hit distance bits, RNG streams, reservoir candidate counts M).
Radiance goes through expf/powf/sinf/cosf, which CUDA and glibc round
differently by a few ulp, so colours are compared with a relative tolerance
on the pixels, plus a bound on the fraction of pixels allowed to differ more
(a ulp-level direction change can move a secondary ray across an edge).
"""
import numpy as np
import pytest

from hdrestir_b200 import abi, configs
from oracle.oracle import Oracle, rng_floats
from tests.parity_checks import check_nee, check_reservoirs

pytestmark = pytest.mark.gpu

SMALL = {
    0: dict(width=64, height=48),
    1: dict(width=64, height=48, n_lights=128),
    2: dict(width=64, height=48, grid=96, n_spheres=60, n_lights=300),
}
RTOL = 1e-4          # per-pixel relative tolerance on RGB (north-star: 1e-4 relative)
ATOL = 1e-6
MAX_OUTLIERS = 0.01  # fraction of pixels allowed outside the tolerance


def _scene(cfg):
    kw = dict(SMALL[cfg])
    return configs.small_variant(cfg, **kw)


def _color_outliers(a, b):
    a = a[:, :3].astype(np.float64)
    b = b[:, :3].astype(np.float64)
    bad = np.abs(a - b) > (ATOL + RTOL * np.maximum(np.abs(a), np.abs(b)))
    return bad.any(1).mean()


def test_rng_streams_bit_exact(gpu_ctx):
    seeds = np.array([0, 1, 7, 1234 ^ 56, 0xFFFFFFFF, 0xC0FFEE00] + list(range(100, 160)), np.uint32)
    dev = gpu_ctx.rng_floats(seeds, 700)  # crosses the 156 / 311 / 312 cursor boundaries
    ref = rng_floats(seeds, 700)
    assert np.array_equal(dev.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_raycast_gbuffer_bit_exact(gpu_ctx, cfg):
    sc, cam = _scene(cfg)
    gpu_ctx.upload_scene(sc)
    gpu_ctx.raycast(cam, 0, aovs=("Depth", "Albedo", "Normal"))
    g = gpu_ctx.download("GBuffer")
    o = Oracle(sc).raycast(cam, 0)
    assert g["hit"].sum() > 0
    assert np.array_equal(g["prim_id"], o["prim_id"])
    assert np.array_equal(g["tri_id"], o["tri_id"])
    for f in ("position", "depth", "normal", "smooth_normal", "albedo", "uv", "dpdu", "dpdv"):
        hit = o["hit"] == 1
        assert np.array_equal(g[f][hit].view(np.uint32), o[f][hit].view(np.uint32)), f
    depth = gpu_ctx.download("Depth")
    assert np.array_equal(depth[o["hit"] == 0], np.ones((o["hit"] == 0).sum(), np.float32))


@pytest.mark.parametrize("cfg", [1, 2])
def test_trace_rays_closest_and_any_hit(gpu_ctx, cfg):
    sc, cam = _scene(cfg)
    gpu_ctx.upload_scene(sc)
    rng = np.random.default_rng(5)
    n = 4096
    o = rng.uniform(-6, 6, (n, 3)) + np.array([0, 3.0, 0])
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    orc = Oracle(sc)
    a = gpu_ctx.trace_rays(rays)
    b = orc.trace_rays(rays)
    assert np.array_equal(a["prim_id"], b["prim_id"]) and np.array_equal(a["tri_id"], b["tri_id"])
    assert np.array_equal(a["depth"].view(np.uint32), b["depth"].view(np.uint32))
    tmax = rng.uniform(0.0, 10.0, n).astype(np.float32)
    a = gpu_ctx.trace_rays(rays, tmax, any_hit=True)
    b = orc.trace_rays(rays, tmax, any_hit=True)
    assert np.array_equal(a["hit"], b["hit"])


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_traversal_forms_identical(cfg):
    """The binary walk and its 4-wide collapse give the same closest hits
    (instance, triangle, t, u, v bits) and the same shadow answers."""
    from hdrestir_b200.context import Context
    sc, cam = _scene(cfg)
    rng = np.random.default_rng(11 + cfg)
    n = 1 << 15
    o = rng.uniform(-8, 8, (n, 3)) + np.array([0, 2.0, 0])
    d = rng.uniform(-1.5, 1.5, (n, 3)) - o  # mostly towards the middle of the scene
    d[: n // 8, 1] = 0.0  # rays parallel to the ground plane and to slab faces
    d[n // 8: n // 4, 0] = 0.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    tmax = rng.uniform(0.0, 12.0, n).astype(np.float32)
    out = []
    for kw in ({}, dict(wide_bvh=True)):
        with Context(device=0, **kw) as ctx:
            ctx.upload_scene(sc)
            out.append((ctx.trace_rays(rays), ctx.trace_rays(rays, tmax, any_hit=True)))
    (ba, bh) = out[0]
    for wa, wh in out[1:]:
        assert np.array_equal(wa.view(np.uint8), ba.view(np.uint8))
        assert np.array_equal(wh["hit"], bh["hit"])
    assert ba["hit"].sum() > n // 50
    assert 0 < bh["hit"].sum() < n


def test_path_trace_matches_oracle(gpu_ctx):
    sc, cam = _scene(0)
    gpu_ctx.upload_scene(sc)
    orc = Oracle(sc)
    gpu_ctx.clear_persistent()
    for frame in range(2):
        gpu_ctx.raycast(cam, frame)
        gpu_ctx.path_trace(cam, frame, max_depth=4)
        gpu = gpu_ctx.download("Color")
        orc.raycast(cam, frame)
        ref, _ = orc.integrate(cam, frame, ris=False, max_depth=4)
        frac = _color_outliers(gpu, ref)
        print(f"PT frame {frame}: outlier fraction {frac:.4f}")
        assert frac <= MAX_OUTLIERS
        gpu_ctx.accumulate(frame, firefly=True)
        orc.accumulate(cam, frame, firefly=True)


MODES = {"wavefront": {}, "one_kernel": dict(one_kernel=True), "all_rays": dict(trace_all_rays=True)}


@pytest.mark.parametrize("mode", list(MODES))
def test_ris_plain_matches_oracle(gpu_ctx, mode):
    sc, cam = _scene(1)
    gpu_ctx.upload_scene(sc)
    orc = Oracle(sc)
    gpu_ctx.raycast(cam, 0)
    gpu_ctx.ris_path_trace(cam, 0, candidate_count=16, use_reservoir=False, skip_visibility=True, max_depth=1,
                           **MODES[mode])
    gpu = gpu_ctx.download("Color")
    orc.raycast(cam, 0)
    ref, _ = orc.integrate(cam, 0, ris=True, candidate_count=16, use_reservoir=False, skip_visibility=True,
                           max_depth=1)
    frac = _color_outliers(gpu, ref)
    print(f"RIS: outlier fraction {frac:.4f}, mean {gpu[:, :3].mean():.5f} vs {ref[:, :3].mean():.5f}")
    assert frac <= MAX_OUTLIERS


@pytest.mark.parametrize("mode", list(MODES))
def test_restir_temporal_matches_oracle(mode):
    """Reservoir M bit-exact, winner (light index) and WSum / W per the parity
    contract, NEE light-selection indices bit-exact (recorded by the wavefront
    forms), colour within the tolerance."""
    from hdrestir_b200.context import Context
    sc, cam = _scene(2)
    orc = Oracle(sc)
    idx = np.arange(cam.width * cam.height)
    with Context(device=0, record_lights=True) as ctx:
        ctx.upload_scene(sc)
        ctx.clear_persistent()
        for frame in range(3):
            ctx.raycast(cam, frame)
            ctx.ris_path_trace(cam, frame, candidate_count=32, use_reservoir=True, max_depth=1, **MODES[mode])
            gpu = ctx.download("Color")
            res = ctx.download("__ris_reservoir")
            o = orc.raycast(cam, frame)
            ref, tr = orc.integrate(cam, frame, ris=True, candidate_count=32, use_reservoir=True, max_depth=1,
                                    trace=True)
            check_reservoirs(res, orc.res, idx, f"ReSTIR {mode} frame {frame}")
            if mode != "one_kernel":
                lights = ctx.download("__ris_nee_lights").view(np.int32)
                check_nee(lights, tr, o["hit"] == 1, 16, f"ReSTIR {mode} frame {frame}")
            frac = _color_outliers(gpu, ref)
            print(f"ReSTIR frame {frame}: outlier fraction {frac:.4f}")
            assert frac <= MAX_OUTLIERS


def test_restir_multibounce_one_kernel_matches_oracle(gpu_ctx):
    """maxDepth 2 runs in the one-thread-per-pixel form (the bounce loop casts its own rays)."""
    sc, cam = _scene(2)
    gpu_ctx.upload_scene(sc)
    gpu_ctx.clear_persistent()
    orc = Oracle(sc)
    for frame in range(2):
        gpu_ctx.raycast(cam, frame)
        gpu_ctx.ris_path_trace(cam, frame, candidate_count=8, use_reservoir=True, max_depth=2)
        gpu = gpu_ctx.download("Color")
        orc.raycast(cam, frame)
        ref, _ = orc.integrate(cam, frame, ris=True, candidate_count=8, use_reservoir=True, max_depth=2)
        frac = _color_outliers(gpu, ref)
        print(f"ReSTIR depth 2 frame {frame}: outlier fraction {frac:.4f}")
        assert frac <= MAX_OUTLIERS


def test_wavefront_modes_identical(gpu_ctx):
    """Skipping rays whose result cannot matter and the one-kernel form give bit-identical images."""
    sc, cam = _scene(2)
    gpu_ctx.upload_scene(sc)
    outs = []
    for mode in MODES.values():
        gpu_ctx.clear_persistent()
        frames = []
        for frame in range(2):
            gpu_ctx.raycast(cam, frame)
            gpu_ctx.ris_path_trace(cam, frame, candidate_count=32, use_reservoir=True, max_depth=1, **mode)
            frames.append(gpu_ctx.download("Color").copy())
        outs.append(np.stack(frames))
    for o in outs[1:]:
        assert np.array_equal(o.view(np.uint32), outs[0].view(np.uint32))


def test_trace_kernel_forms_give_identical_images():
    """ReSTIR frames of the config-2 scene family are bit-identical whichever
    walk (binary or 4-wide) and lane schedule (refill or one ray per lane) the
    wavefront trace kernels use."""
    from hdrestir_b200.context import Context
    sc, cam = configs.small_variant(2, 160, 96, grid=128, n_spheres=200, n_lights=2000)
    outs = []
    for kw in ({}, dict(split_stack=True), dict(unphased=True), dict(lane_per_ray=True), dict(wide_bvh=True),
               dict(wide_bvh=True, unphased=True), dict(wide_bvh=True, lane_per_ray=True), dict(tuning=(3, 2)),
               dict(wide_bvh=True, tuning=(8, 6)), dict(tuning=(16, 16, 1)),
               dict(tuning=(16, 16, 2)), dict(tuning=(16, 16, 3))):
        tuning = kw.pop("tuning", None)
        with Context(device=0, **kw) as ctx:
            ctx.upload_scene(sc)
            if tuning:
                ctx.set_trace_tuning(*tuning)
            frames = []
            for frame in range(2):
                ctx.raycast(cam, frame)
                ctx.ris_path_trace(cam, frame, candidate_count=32, use_reservoir=True, max_depth=1)
                ctx.accumulate(frame, firefly=True)
                frames.append(ctx.download("Color").copy())
            outs.append(np.stack(frames))
    for o in outs[1:]:
        assert np.array_equal(o.view(np.uint32), outs[0].view(np.uint32))


def test_autotune_trace_keeps_results():
    """The trace-schedule autotuner picks a schedule from its grid, and frames
    rendered with it are those rendered before tuning."""
    from hdrestir_b200.context import Context
    sc, cam = configs.small_variant(2, 96, 64, grid=96, n_spheres=60, n_lights=300)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        with pytest.raises(abi.HdrError):
            ctx.autotune_trace()  # no wavefront frame yet
        ris = dict(candidate_count=32, use_reservoir=False, max_depth=1)
        ctx.raycast(cam, 0)
        ctx.ris_path_trace(cam, 0, **ris)
        before = ctx.download("Color").copy()
        best = ctx.autotune_trace()
        assert best["node_quorum"] in (8, 12, 16, 20, 24, 28) and best["blocks_per_sm"] in (4, 6, 8, 16)
        assert best["trace_ms"] > 0.0 and ctx.trace_tuning()["node_quorum"] == best["node_quorum"]
        ctx.ris_path_trace(cam, 0, **ris)
        assert np.array_equal(ctx.download("Color").view(np.uint32), before.view(np.uint32))


@pytest.mark.parametrize("kw", [dict(), dict(skip_visibility=True), dict(trace_all_rays=True),
                                dict(spatial_neighbors=4, spatial_radius=6.0, m_cap=20)])
def test_autotune_frame_renders_the_frame(kw):
    """A tuning frame (every trace schedule and resampling launch shape run on the
    same queues and reservoir copies) leaves exactly the buffers of the plain
    frame, reservoirs with history included, and the frames after it too."""
    from hdrestir_b200.context import Context
    sc, cam = configs.small_variant(2, 96, 64, grid=96, n_spheres=60, n_lights=300)
    ris = dict(candidate_count=32, use_reservoir=True, max_depth=1, **kw)
    out = []
    for tune in (False, True):
        with Context(device=0) as ctx:
            ctx.upload_scene(sc)
            snaps = []
            for f in range(3):
                ctx.raycast(cam, f)
                if tune and f == 1:
                    best = ctx.autotune_frame(cam, f, **ris)
                    assert best["shade_shape"] in range(4) and best["shade_ms"] > 0.0 and best["trace_ms"] > 0.0
                    assert ctx.trace_tuning()["shade_shape"] == best["shade_shape"]
                else:
                    ctx.ris_path_trace(cam, f, **ris)
                ctx.accumulate(f)
                snaps.append([ctx.download(n).copy() for n in ("Color", "__ris_reservoir", "__accum_color")])
            out.append(snaps)
    for f, (plain, tuned) in enumerate(zip(*out)):
        for a, b in zip(plain, tuned):
            assert np.array_equal(np.ascontiguousarray(a).view(np.uint32),
                                  np.ascontiguousarray(b).view(np.uint32)), f"frame {f}"


def test_autotune_frame_rejects_the_one_kernel_form():
    from hdrestir_b200.context import Context
    sc, cam = configs.small_variant(2, 32, 32, grid=64, n_spheres=10, n_lights=50)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        ctx.raycast(cam, 0)
        with pytest.raises(abi.HdrError) as e:
            ctx.autotune_frame(cam, 0, candidate_count=8, use_reservoir=True, max_depth=2)
        assert e.value.status == abi.HDR_EINVAL


def _dome_scene(w=64, h=48):
    sc, cam, cams = configs.config3(w, h, n_small=3, small=32, grid=96, n_spheres=60, n_lights=300,
                                    dome_size=(128, 64))
    return sc, cam, cams


@pytest.mark.parametrize("ris", [True, False])
def test_dome_lit_scene_matches_oracle(ris):
    """Config-3 family (terrain, spheres, rect lights and a lat-long dome): ReSTIR
    (BSDF candidates traced, the environment is a light) and PathTracer."""
    from hdrestir_b200.context import Context
    sc, cam, _ = _dome_scene()
    orc = Oracle(sc)
    kw = dict(candidate_count=16, use_reservoir=True, max_depth=1) if ris else dict(max_depth=6)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        for frame in range(2):
            ctx.raycast(cam, frame)
            if ris:
                ctx.ris_path_trace(cam, frame, **kw)
            else:
                ctx.path_trace(cam, frame, **kw)
            gpu = ctx.download("Color")
            orc.raycast(cam, frame)
            ref, _ = orc.integrate(cam, frame, ris=ris, **kw)
            if ris:
                m_gpu = ctx.download("__ris_reservoir")[4, :, 2].view(np.int32)
                assert np.array_equal(m_gpu, orc.res["m"])
            frac = _color_outliers(gpu, ref)
            print(f"dome {'ReSTIR' if ris else 'PT'} frame {frame}: outlier fraction {frac:.4f}")
            assert frac <= MAX_OUTLIERS


def test_path_trace_batch_equals_images_alone():
    """One PathTracePass launch over several images gives each image its own result."""
    from hdrestir_b200.context import Context, path_trace_batch
    sc, cam, cams = _dome_scene()
    cams = [cam] + cams
    want = []
    for c in cams:
        with Context(device=0) as ctx:
            ctx.upload_scene(sc)
            for f in range(2):
                ctx.raycast(c, f)
                ctx.path_trace(c, f, max_depth=8)
                ctx.accumulate(f)
            want.append(ctx.download("Color").copy())
    ctxs = [Context(device=0) for _ in cams]
    try:
        ctxs[0].upload_scene(sc)
        for x in ctxs[1:]:
            x.share_scene(ctxs[0])
        for f in range(2):
            for x, c in zip(ctxs, cams):
                x.raycast(c, f)
            path_trace_batch(ctxs, cams, [f] * len(cams), max_depth=8)
            for x in ctxs:
                x.accumulate(f)
        got = [x.download("Color").copy() for x in ctxs]
    finally:
        for x in ctxs:
            x.close()
    for g, w in zip(got, want):
        assert np.array_equal(g.view(np.uint32), w.view(np.uint32))


@pytest.mark.parametrize("case", ["cfg0", "cfg2", "dome"])
def test_wavefront_path_trace_equals_one_thread_form(case):
    """PathTracePass in wavefront form (per-vertex kernels, compacted live paths)
    gives the one-thread-per-pixel form's image bit for bit, roulette included."""
    from hdrestir_b200.context import Context
    if case == "dome":
        sc, cam, _ = _dome_scene()
        depth = 16
    else:
        sc, cam = _scene(0 if case == "cfg0" else 2)
        depth = 6 if case == "cfg0" else 8
    outs = []
    for one in (False, True):
        with Context(device=0, pt_one_kernel=one) as ctx:
            ctx.upload_scene(sc)
            frames = []
            for f in range(3):
                ctx.raycast(cam, f)
                ctx.path_trace(cam, f, max_depth=depth)
                ctx.accumulate(f)
                frames.append(ctx.download("Color").copy())
            outs.append(np.stack(frames))
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


def _lobe_scene(emissive=False):
    """The config-2 family with spheres of every PreviewSurface lobe: coat and sheen (rough
    and mirror), transmission (refraction and total internal reflection), mirror specular,
    metal, and DefaultMaterial instances; `emissive` adds glowing spheres (emissive
    materials that are no light's geometry)."""
    import dataclasses
    from hdrestir_b200.scene import Material
    sc, cam = configs.small_variant(2, 96, 64, grid=64, n_spheres=80, n_lights=200)
    kinds = [
        dict(coat=0.8, coat_roughness=0.2), dict(coat=1.0, coat_roughness=0.0, coat_ior=1.8),
        dict(sheen=0.9, sheen_roughness=0.4), dict(sheen=1.0, sheen_roughness=0.0),
        dict(transmission=0.7, ior=1.3, roughness=0.3), dict(transmission=0.9, ior=2.4, roughness=0.0),
        dict(roughness=0.0, specular=0.8), dict(metallic=1.0, roughness=0.15),
        dict(subsurface=0.5, subsurface_color=(0.9, 0.3, 0.2)),
    ] + ([dict(emission=4.0, emission_color=(1.0, 0.6, 0.2))] if emissive else [])
    for k, inst in enumerate(sc.instances[1:]):
        if k % (len(kinds) + 1) == len(kinds):
            inst.material = -1
        else:
            sc.materials[inst.material] = dataclasses.replace(sc.materials[inst.material], **kinds[k % (len(kinds) + 1)])
    return sc, cam


@pytest.mark.parametrize("use_reservoir,emissive", [(True, False), (False, False), (True, True)])
def test_wavefront_modes_identical_on_every_lobe(gpu_ctx, use_reservoir, emissive):
    """Where BSDF-candidate rays are not cast, the resampling pass only advances the stream past
    those candidates (or jumps to the saved end of generation), and where nothing emits the
    path's bounce ray is not cast either; images stay bit-identical to casting every ray and
    to the one-kernel form on materials that take every sampling branch."""
    sc, cam = _lobe_scene(emissive)
    gpu_ctx.upload_scene(sc)
    outs = []
    for mode in MODES.values():
        gpu_ctx.clear_persistent()
        frames = []
        for frame in range(2):
            gpu_ctx.raycast(cam, frame)
            gpu_ctx.ris_path_trace(cam, frame, candidate_count=32, use_reservoir=use_reservoir, max_depth=1, **mode)
            frames.append(gpu_ctx.download("Color").copy())
        outs.append(np.stack(frames))
    for o in outs[1:]:
        assert np.array_equal(o.view(np.uint32), outs[0].view(np.uint32))


def test_every_lobe_matches_oracle(gpu_ctx):
    """ReSTIR frame of the every-lobe scene against the oracle (reservoir M exactly, colour
    within the tolerance)."""
    sc, cam = _lobe_scene()
    gpu_ctx.upload_scene(sc)
    orc = Oracle(sc)
    gpu_ctx.clear_persistent()
    for frame in range(2):
        gpu_ctx.raycast(cam, frame)
        gpu_ctx.ris_path_trace(cam, frame, candidate_count=32, use_reservoir=True, max_depth=1)
        got = gpu_ctx.download("Color")
        res = gpu_ctx.download("__ris_reservoir")
        orc.raycast(cam, frame)
        want, _ = orc.integrate(cam, frame, ris=True, candidate_count=32, use_reservoir=True, max_depth=1)
        assert np.array_equal(res[4, :, 2].view(np.int32), orc.res["m"])
        check_reservoirs(res, orc.res, np.arange(len(orc.res)), f"every lobe frame {frame}")
        frac = _color_outliers(got, want)
        print(f"every lobe, frame {frame}: outlier fraction {frac:.4f}")
        assert frac <= MAX_OUTLIERS


def _mse_vs(img, ref):
    peak = max(float(ref[:, :3].max()), 1e-12)
    return float(np.mean(((img[:, :3].astype(np.float64) - ref[:, :3]) / peak) ** 2))


def test_spatial_reuse_off_is_identical_and_on_lowers_error():
    """Spatial reuse (extension): spatial_neighbors = 0 gives the reference's images bit for bit;
    with 5 neighbours the frames after warm-up are closer to a high-sample image than temporal
    reuse alone, and the pass rejects the one-kernel form."""
    from hdrestir_b200.context import Context
    sc, cam = configs.small_variant(2, 128, 96, grid=96, n_spheres=120, n_lights=1500)
    ris = dict(candidate_count=32, use_reservoir=True, max_depth=1)

    def run(frames, start=0, accumulate=False, **kw):
        with Context(device=0) as ctx:
            ctx.upload_scene(sc)
            out = []
            for f in range(start, start + frames):
                ctx.raycast(cam, f)
                ctx.ris_path_trace(cam, f, **ris, **kw)
                if accumulate:
                    ctx.accumulate(f - start)
                out.append(ctx.download("Color").astype(np.float64))
            return out

    plain = run(4)
    off = run(4, spatial_neighbors=0, spatial_radius=12.0)
    assert all(np.array_equal(a, b) for a, b in zip(plain, off))
    high = run(256, start=50_000, accumulate=True)[-1]  # converged image of the same estimator
    on = run(4, spatial_neighbors=5, spatial_radius=20.0)
    e_plain = np.mean([_mse_vs(x, high) for x in plain[1:]])
    e_on = np.mean([_mse_vs(x, high) for x in on[1:]])
    print(f"per-frame MSE vs converged: temporal only {e_plain:.4e}, + spatial {e_on:.4e}")
    assert np.isfinite(e_on) and e_on < e_plain
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        ctx.raycast(cam, 0)
        with pytest.raises(abi.HdrError):
            ctx.ris_path_trace(cam, 0, **ris, spatial_neighbors=4, one_kernel=True)


def test_reprojected_history_lowers_error_on_an_orbit():
    """Temporal reuse across camera motion (extension): on a slow orbit, history reprojected
    from the previous frame brings each frame closer to that pose's converged image than
    starting without history (what the reference's renderer does on a camera change); a
    static camera with the flag off keeps the reference's images."""
    from hdrestir_b200.context import Context
    sc, _ = configs.small_variant(2, 128, 96, grid=96, n_spheres=120, n_lights=1500)
    cams = [configs.orbit_camera(0.004 * k, 128, 96) for k in range(6)]
    ris = dict(candidate_count=32, use_reservoir=True, max_depth=1)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        conv = []
        for k, cam in enumerate(cams):
            ctx.clear_persistent()
            for f in range(160):
                ctx.raycast(cam, 70_000 + 1000 * k + f)
                ctx.ris_path_trace(cam, 70_000 + 1000 * k + f, **ris)
                ctx.accumulate(f)
            conv.append(ctx.download("Color").astype(np.float64))
        errs = {}
        for name, kw in (("reset", {}), ("reproject", dict(reproject=True))):
            ctx.clear_persistent()
            e = []
            for k, cam in enumerate(cams):
                if name == "reset":
                    ctx.clear_persistent()
                ctx.raycast(cam, k)
                ctx.ris_path_trace(cam, k, **ris, **kw)
                e.append(_mse_vs(ctx.download("Color"), conv[k]))
            errs[name] = float(np.mean(e[2:]))
    print(f"per-frame MSE on the orbit: no history {errs['reset']:.4e}, reprojected {errs['reproject']:.4e}")
    assert np.isfinite(errs["reproject"]) and errs["reproject"] < errs["reset"]


def test_download_async_equals_download():
    """The overlapped read-back returns each frame's image as hdr_download does, with later
    passes running while it copies."""
    from hdrestir_b200.context import Context
    sc, cam = _scene(2)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        n = cam.width * cam.height
        outs, want = [np.empty((n, 4), np.float32) for _ in range(3)], []
        for f in range(3):
            ctx.raycast(cam, f)
            ctx.ris_path_trace(cam, f, candidate_count=32, use_reservoir=True, max_depth=1)
            ctx.accumulate(f)
            ctx.download_async("Color", outs[f])
            ctx.synchronize()
            want.append(ctx.download("Color").copy())
        ctx.download_wait()
        for o, w in zip(outs, want):
            assert np.array_equal(o.view(np.uint32), w.view(np.uint32))


@pytest.mark.parametrize("kw", [dict(ris=True, candidate_count=16, use_reservoir=True, max_depth=1),
                                dict(ris=True, candidate_count=16, use_reservoir=False, skip_visibility=True,
                                     max_depth=1),
                                dict(ris=False, max_depth=4)])
def test_point_and_distant_lights_match_oracle(gpu_ctx, kw):
    """Rect, point (cone-shaped) and distant lights: the GPU passes against the oracle (pinned
    to the reference on the same scene), reservoir M exactly, colour within the tolerance."""
    sc, cam = configs.mixed_lights(96, 64)
    gpu_ctx.upload_scene(sc)
    gpu_ctx.clear_persistent()
    orc = Oracle(sc)
    kw = dict(kw)
    ris = kw.pop("ris")
    for frame in range(2):
        gpu_ctx.raycast(cam, frame)
        if ris:
            gpu_ctx.ris_path_trace(cam, frame, **kw)
        else:
            gpu_ctx.path_trace(cam, frame, **kw)
        gpu = gpu_ctx.download("Color")
        orc.raycast(cam, frame)
        ref, _ = orc.integrate(cam, frame, ris=ris, **kw)
        if ris and kw.get("use_reservoir"):
            assert np.array_equal(gpu_ctx.download("__ris_reservoir")[4, :, 2].view(np.int32), orc.res["m"])
        frac = _color_outliers(gpu, ref)
        print(f"mixed lights {kw}, frame {frame}: outlier fraction {frac:.4f}")
        assert frac <= MAX_OUTLIERS and float(ref[:, :3].mean()) > 0.0



@pytest.mark.parametrize("params", [
    dict(enable_dof=1, focal_length=50.0, f_stop=1.4, focus_distance=9.0, bokeh_blades=0),
    dict(enable_dof=1, focal_length=35.0, f_stop=2.0, focus_distance=7.5, bokeh_blades=6),
    dict(lens_distortion=-0.15),
    dict(enable_exposure=1, f_stop=4.0, iso=400.0, shutter_speed=0.01),
])
def test_camera_params_match_oracle(gpu_ctx, params):
    """Thin-lens depth of field (disc and polygonal bokeh), lens distortion and exposure: GBuffer
    hits and colour against the oracle. The lens samples go through sinf/cosf, which CUDA and
    glibc round differently by an ulp, so a ray on a triangle edge may pick the neighbour: hits
    must agree on 99.9 % of pixels, colour within the usual tolerance."""
    from hdrestir_b200.scene import make_camera
    sc, _ = configs.small_variant(1, 96, 64, n_lights=64)
    cam = make_camera((0.0, 6.0, 9.0), (0.0, 0.0, 0.0), 96, 64, fov=55.0, params=params)
    gpu_ctx.upload_scene(sc)
    gpu_ctx.clear_persistent()
    orc = Oracle(sc)
    for frame in range(2):
        gpu_ctx.raycast(cam, frame)
        g = gpu_ctx.download("GBuffer")
        o = orc.raycast(cam, frame)
        dof = params.get("enable_dof", 0)
        same = np.mean(g["prim_id"] == o["prim_id"])
        assert same >= (0.999 if dof else 1.0), same
        gpu_ctx.ris_path_trace(cam, frame, candidate_count=16, use_reservoir=True, max_depth=1)
        ref, _ = orc.integrate(cam, frame, ris=True, candidate_count=16, use_reservoir=True, max_depth=1)
        assert _color_outliers(gpu_ctx.download("Color"), ref) <= MAX_OUTLIERS



@pytest.mark.parametrize("kw", [dict(ris=True, candidate_count=16, use_reservoir=True, max_depth=1),
                                dict(ris=True, candidate_count=16, use_reservoir=True, max_depth=3),
                                dict(ris=False, max_depth=6)])
def test_translucent_scene_matches_oracle(gpu_ctx, kw):
    """Partial opacity, Beer absorption and thin-walled transmission: a scene that is not opaque
    runs the one-thread forms (rays cast on the spot); against the oracle."""
    sc, cam = configs.translucent_variant(96, 64)
    gpu_ctx.upload_scene(sc)
    gpu_ctx.clear_persistent()
    orc = Oracle(sc)
    kw = dict(kw)
    ris = kw.pop("ris")
    for frame in range(2):
        gpu_ctx.raycast(cam, frame)
        if ris:
            gpu_ctx.ris_path_trace(cam, frame, **kw)
        else:
            gpu_ctx.path_trace(cam, frame, **kw)
        gpu = gpu_ctx.download("Color")
        orc.raycast(cam, frame)
        ref, _ = orc.integrate(cam, frame, ris=ris, **kw)
        if ris:
            assert np.array_equal(gpu_ctx.download("__ris_reservoir")[4, :, 2].view(np.int32), orc.res["m"])
        frac = _color_outliers(gpu, ref)
        print(f"translucent {kw}, frame {frame}: outlier fraction {frac:.4f}")
        assert frac <= MAX_OUTLIERS


@pytest.mark.parametrize("kw", [dict(use_reservoir=False, skip_visibility=True),
                                dict(use_reservoir=True, skip_visibility=True),
                                dict(use_reservoir=True, skip_visibility=False, reproject=True)])
def test_queued_winner_visibility_equals_on_the_spot(kw):
    """Winners whose visibility is still untested (skipVisibility, or taken from reprojected
    history) have their shadow rays traced by the shadow kernel in the wavefront form and cast on
    the spot in the one-kernel form; the frames of an orbit are bit-identical."""
    from hdrestir_b200.context import Context
    sc, _ = configs.small_variant(1, 96, 64, n_lights=256)
    outs = []
    for mode in ({}, dict(one_kernel=True)):
        with Context(device=0) as ctx:
            ctx.upload_scene(sc)
            frames = []
            for f in range(3):
                cam = configs.config_camera(1, 96, 64) if not kw.get("reproject") else \
                    configs.make_camera((0.3 * f, 6.0, 9.0), (0.0, 0.0, 0.0), 96, 64, fov=55.0)
                ctx.raycast(cam, f)
                ctx.ris_path_trace(cam, f, candidate_count=16, max_depth=1, **kw, **mode)
                frames.append(ctx.download("Color").copy())
            outs.append(np.stack(frames))
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


def test_spatial_reuse_queued_visibility_is_deterministic():
    """Spatial reuse with its moved samples' shadow rays queued for the shadow kernel: two runs of
    the same frames give the same images (the queue order may differ; the answers may not)."""
    from hdrestir_b200.context import Context
    sc, cam = configs.small_variant(2, 96, 64, grid=64, n_spheres=60, n_lights=400)
    outs = []
    for _ in range(2):
        with Context(device=0) as ctx:
            ctx.upload_scene(sc)
            frames = []
            for f in range(3):
                ctx.raycast(cam, f)
                ctx.ris_path_trace(cam, f, candidate_count=32, use_reservoir=True, max_depth=1,
                                   spatial_neighbors=5, spatial_radius=16.0)
                frames.append(ctx.download("Color").copy())
            outs.append(np.stack(frames))
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


@pytest.mark.parametrize("kw", [dict(ris=True, candidate_count=16, use_reservoir=True, max_depth=1),
                                dict(ris=True, candidate_count=8, use_reservoir=True, max_depth=3),
                                dict(ris=False, max_depth=4)])
def test_textured_scene_matches_oracle(gpu_ctx, kw):
    """PreviewSurface textures (diffuse, metallic, roughness, normal maps) through the wavefront
    RIS pass, the one-thread RIS form and path tracing; against the oracle, which is pinned to
    the reference's own texture sampler."""
    sc, cam = configs.textured_variant(96, 64)
    gpu_ctx.upload_scene(sc)
    gpu_ctx.clear_persistent()
    orc = Oracle(sc)
    kw = dict(kw)
    ris = kw.pop("ris")
    for frame in range(2):
        gpu_ctx.raycast(cam, frame)
        if ris:
            gpu_ctx.ris_path_trace(cam, frame, **kw)
        else:
            gpu_ctx.path_trace(cam, frame, **kw)
        gpu = gpu_ctx.download("Color")
        orc.raycast(cam, frame)
        ref, _ = orc.integrate(cam, frame, ris=ris, **kw)
        if ris:
            assert np.array_equal(gpu_ctx.download("__ris_reservoir")[4, :, 2].view(np.int32), orc.res["m"])
        frac = _color_outliers(gpu, ref)
        print(f"textured {kw}, frame {frame}: outlier fraction {frac:.4f}")
        assert frac <= MAX_OUTLIERS
