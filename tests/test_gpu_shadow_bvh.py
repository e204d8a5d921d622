"""The shadow BVH (4-wide SAH trees for "hit nearer than the light" queries)
against the reference-order walk of the reference's own trees, through the C ABI.

The answer of a shadow query does not depend on the tree: the same triangle
test (IntersectTriangle, bvh.cpp:8-30) in the same instance space decides it,
and the shadow BVH's box tests are conservative. The reference culls with its
own rounded slab tests, so a ray grazing one of its box faces by an ulp could
still differ; such rays are counted, and must stay below 1e-4 of 10^6 random and
frame rays (none have been seen). Whole frames rendered with either structure
must agree within the radiance tolerance.
"""
import numpy as np
import pytest

from hdrestir_b200 import configs
from oracle.oracle import Oracle
from tests.parity_checks import MAX_OUTLIERS, outliers

pytestmark = pytest.mark.gpu

MAX_MISMATCH = 1e-4


def _frame_shadow_rays(ctx, sc, cam, rng, per_pixel=1, stride=3):
    """Shadow rays as the NEE candidates cast them: from primary hits (offset along
    the shading normal) to uniformly chosen points on uniformly chosen rect lights."""
    ctx.raycast(cam, 0)
    g = ctx.download("GBuffer")[::stride]
    g = g[g["hit"] == 1]
    p = np.repeat(g["position"].astype(np.float64), per_pixel, 0)
    nrm = np.repeat(g["smooth_normal"].astype(np.float64), per_pixel, 0)
    li = rng.integers(0, len(sc.lights), len(p))
    mats = np.stack([sc.lights[k].transform for k in range(len(sc.lights))])
    wh = np.array([[sc.lights[k].width, sc.lights[k].height] for k in range(len(sc.lights))])
    uv = rng.uniform(-0.5, 0.5, (len(p), 2)) * wh[li]
    loc = np.concatenate([uv, np.zeros((len(p), 1)), np.ones((len(p), 1))], 1)
    lp = np.einsum("ni,nij->nj", loc, mats[li])[:, :3]
    o = p + nrm * 1e-4
    d = lp - o
    dist = np.linalg.norm(d, axis=1)
    d /= dist[:, None]
    keep = np.sum(d * nrm, 1) > 0
    rays = np.concatenate([o, d], 1)[keep].astype(np.float32)
    return rays, (dist[keep] - 1e-3).astype(np.float32)


def _random_rays(rng, n, center=(0.0, 2.0, 0.0), extent=20.0):
    o = rng.uniform(-extent, extent, (n, 3)) + np.array(center)
    d = rng.normal(size=(n, 3))
    d[: n // 16, 1] = 0.0  # rays parallel to the ground and to slab faces
    d[n // 16: n // 8, 0] = 0.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], 1).astype(np.float32), rng.uniform(0.0, 2 * extent, n).astype(np.float32)


def test_shadow_bvh_answers_equal_reference_walk_on_config2():
    from hdrestir_b200.context import Context
    sc, cam = configs.config2()
    rng = np.random.default_rng(0x5AD0)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        fr, fl = _frame_shadow_rays(ctx, sc, cam, rng)
        rr, rl = _random_rays(rng, 1_000_000 - len(fr))
        rays = np.concatenate([fr, rr])
        lim = np.concatenate([fl, rl])
        assert len(rays) == 1_000_000
        ref = ctx.trace_stats(rays, 2, lim)   # the reference trees' shadow walk
        new = ctx.trace_stats(rays, 4, lim)   # the shadow BVH
        mism = int((ref[:, 3] != new[:, 3]).sum())
        n_f = len(fr)
        print(f"config 2: {len(rays)} rays ({n_f} frame rays), occluded {ref[:, 3].mean():.4f}; mismatches {mism}; "
              f"frame rays: pops {ref[:n_f, 0].mean():.1f} -> {new[:n_f, 0].mean():.1f}, "
              f"triangles {ref[:n_f, 2].mean():.1f} -> {new[:n_f, 2].mean():.1f}")
        assert mism <= MAX_MISMATCH * len(rays)
        assert 0.1 < ref[:n_f, 3].mean() < 0.9
        assert new[:n_f, 0].mean() < 0.5 * ref[:n_f, 0].mean()
        # the same through hdr_trace_rays' any-hit query, which the shadow BVH answers
        hit = ctx.trace_rays(rays[:200_000], lim[:200_000], any_hit=True)["hit"]
        assert int((hit != new[:200_000, 3]).sum()) == 0


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_shadow_bvh_answers_equal_oracle(cfg):
    """Against the oracle's recursive walk of the reference's trees (small scenes)."""
    from hdrestir_b200.context import Context
    sc, cam = configs.small_variant(cfg, 64, 48, **({} if cfg == 0 else dict(n_lights=200)))
    rng = np.random.default_rng(cfg)
    extent = 1.0 if cfg == 0 else 8.0
    rays, lim = _random_rays(rng, 50_000, center=(0.0, 0.0 if cfg == 0 else 2.0, 0.0), extent=extent)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        got = ctx.trace_rays(rays, lim, any_hit=True)["hit"]
        fr, fl = _frame_shadow_rays(ctx, sc, cam, rng, per_pixel=4, stride=1) if cfg else (rays[:0], lim[:0])
        got_f = ctx.trace_rays(fr, fl, any_hit=True)["hit"] if len(fr) else got[:0]
    orc = Oracle(sc)
    want = orc.trace_rays(rays, lim, any_hit=True)["hit"]
    want_f = orc.trace_rays(fr, fl, any_hit=True)["hit"] if len(fr) else want[:0]
    assert 0 < want.sum() < len(want)
    assert int((got != want).sum()) + int((got_f != want_f).sum()) == 0


def test_frames_with_shadow_bvh_match_reference_shadows():
    """ReSTIR frames of the config-2 family: the shadow BVH and the reference trees
    give the same images (every pixel within the tolerance; in practice equal)."""
    from hdrestir_b200.context import Context
    sc, cam = configs.small_variant(2, 160, 96, grid=128, n_spheres=200, n_lights=2000)
    out = []
    for ref_shadows in (False, True):
        with Context(device=0, reference_shadows=ref_shadows) as ctx:
            ctx.upload_scene(sc)
            frames = []
            for f in range(3):
                ctx.raycast(cam, f)
                ctx.ris_path_trace(cam, f, candidate_count=32, use_reservoir=True, max_depth=1)
                ctx.accumulate(f)
                frames.append(ctx.download("Color").copy())
            out.append(np.stack(frames))
    differ = int((out[0].view(np.uint32) != out[1].view(np.uint32)).any(-1).sum())
    print(f"pixels that differ between the two shadow structures: {differ}")
    for f in range(3):
        assert outliers(out[0][f][:, :3], out[1][f][:, :3]) <= MAX_OUTLIERS


def test_shadow_bvh_follows_moved_instances():
    """After hdr_scene_set_instance_transforms the shadow BVH's TLAS is rebuilt: shadow
    answers equal those of a fresh upload of the moved scene and of the reference walk."""
    import copy

    from hdrestir_b200.context import Context
    sc, cam = configs.small_variant(2, 64, 48, grid=64, n_spheres=80, n_lights=200)
    rng = np.random.default_rng(7)
    moved = copy.deepcopy(sc)
    for inst in moved.instances[1:]:
        t = np.array(inst.transform, np.float64)
        t[3, :3] += rng.uniform(-3, 3, 3) * np.array([1.0, 0.2, 1.0])
        inst.transform = t
    xf = np.stack([np.asarray(i.transform, np.float32) for i in moved.instances])
    rays, lim = _random_rays(rng, 100_000, extent=10.0)
    with Context(device=0) as a, Context(device=0) as b:
        a.upload_scene(sc)
        a.set_instance_transforms(xf)
        b.upload_scene(moved)
        got = a.trace_stats(rays, 4, lim)
        fresh = b.trace_stats(rays, 4, lim)
        ref = a.trace_stats(rays, 2, lim)
    assert np.array_equal(got, fresh)
    assert int((got[:, 3] != ref[:, 3]).sum()) == 0


@pytest.mark.parametrize("cfg", [1, 2])
def test_checked_sah_closest_hits_equal_reference_walk(cfg):
    """The default closest hits: the 4-wide SAH walk, each hit checked against the
    reference walk's box tests on the way down to it, the reference walk for the
    rays the check rejects. Every answer (instance, triangle, t, u, v through the
    GBuffer attributes) equals the reference walk's, on 500,000 random rays and on
    whole 1080p GBuffers, including config 1's coplanar boxes where the unchecked
    SAH walk differs."""
    from hdrestir_b200.context import Context
    sc, _ = (configs.config1() if cfg == 1 else configs.config2())
    rng = np.random.default_rng(50 + cfg)
    rays, _ = _random_rays(rng, 500_000, extent=15.0)
    with Context(device=0, reference_closest=True) as ref, Context(device=0) as chk, \
            Context(device=0, sah_closest=True) as sah:
        for c in (ref, chk, sah):
            c.upload_scene(sc)
        want, got, loose = ref.trace_rays(rays), chk.trace_rays(rays), sah.trace_rays(rays)
        assert np.array_equal(want.view(np.uint8), got.view(np.uint8))
        differ = int((want.view(np.uint8).reshape(len(want), -1) != loose.view(np.uint8).reshape(len(loose), -1))
                     .any(1).sum())
        cam2 = configs.config_camera(cfg, 1920, 1080)
        for c in (ref, chk):
            c.raycast(cam2, 3)
        assert np.array_equal(ref.download("GBuffer").view(np.uint8), chk.download("GBuffer").view(np.uint8))
        print(f"config {cfg}: checked SAH closest hits equal the reference on all rays; the unchecked walk "
              f"differs on {differ} of {len(rays)}")


@pytest.mark.parametrize("cfg,max_frac", [(1, 2e-3), (2, 1e-4)])
def test_sah_closest_hits_against_reference_walk(cfg, max_frac):
    """Opt-in HDR_CTX_SAH_CLOSEST: closest hits on the 4-wide SAH trees, ties broken
    in the reference's walk order. They equal the reference walk except where the
    reference's own rounded box tests cull the nearest hit (coplanar surfaces, such
    as config 1's boxes on its ground plane): counted here on random rays and on
    whole 1080p GBuffers."""
    from hdrestir_b200.context import Context
    sc, cam = (configs.config1() if cfg == 1 else configs.config2())
    rng = np.random.default_rng(40 + cfg)
    rays, _ = _random_rays(rng, 500_000, extent=15.0)
    with Context(device=0, reference_closest=True) as ref, Context(device=0, sah_closest=True) as sah:
        ref.upload_scene(sc)
        sah.upload_scene(sc)
        a = ref.trace_stats(rays, 0)  # the reference's trees, reference order
        b = sah.trace_stats(rays, 5)  # the 4-wide SAH trees
        want = ref.trace_rays(rays)
        got = sah.trace_rays(rays)
        same = ((want["prim_id"] == got["prim_id"]) & (want["tri_id"] == got["tri_id"])
                & (want["depth"].view(np.uint32) == got["depth"].view(np.uint32)))
        frac = 1.0 - same.mean()
        cam2 = configs.config_camera(cfg, 1920, 1080)
        ref.raycast(cam2, 0)
        sah.raycast(cam2, 0)
        ga, gb = ref.download("GBuffer"), sah.download("GBuffer")
        px = 1.0 - (ga.view(np.uint8).reshape(len(ga), -1) == gb.view(np.uint8).reshape(len(gb), -1)).all(1).mean()
        print(f"config {cfg}: closest-hit mismatches {frac:.2e} of random rays, {px:.2e} of 1080p GBuffer "
              f"pixels; pops {a[:, 0].mean():.1f} -> {b[:, 0].mean():.1f}")
        assert frac <= max_frac and px <= max_frac
        assert b[:, 0].mean() < a[:, 0].mean()
