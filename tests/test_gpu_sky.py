"""The physical sky (PhysicalSky, scene/physical_sky.cpp) on the device against
the oracle, which is pinned to the reference's own sky and integrators in
tests/test_reference_pin.py: sky radiance on misses, the RIS pass's sky
technique (the sun as a delta light outside the light sampler, light index
len(lights) in the reservoir) with temporal reuse, and the path tracer's
separate sun sample. GBuffer and M bit-exact; reservoir winners, WSum, W and
radiance within the parity tolerances (parity_checks)."""
import numpy as np
import pytest

from hdrestir_b200 import configs
from oracle.oracle import Oracle
from tests.parity_checks import MAX_OUTLIERS, check_gbuffer, check_reservoirs, outliers

pytestmark = pytest.mark.gpu


def _scene(cfg, hour, w=80, h=48):
    extra = {1: dict(n_lights=64), 2: dict(grid=64, n_spheres=60, n_lights=200)}[cfg]
    return configs.sky_variant(cfg, w, h, hour=hour, **extra)


@pytest.mark.parametrize("hour", [15.5, 6.5])
@pytest.mark.parametrize("cfg,kw", [
    (2, dict(candidate_count=32, use_reservoir=True, skip_visibility=False, max_depth=1)),
    (2, dict(candidate_count=12, use_reservoir=True, skip_visibility=True, max_depth=1)),
    (1, dict(candidate_count=16, use_reservoir=False, skip_visibility=False, max_depth=1)),
])
def test_ris_under_the_physical_sky_matches_oracle(hour, cfg, kw):
    from hdrestir_b200.context import Context
    sc, cam = _scene(cfg, hour)
    orc = Oracle(sc, threads=8)
    suns = 0
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        for frame in range(3):
            ctx.raycast(cam, frame)
            ctx.ris_path_trace(cam, frame, **kw)
            gpu = ctx.download("Color")[:, :3]
            orc.raycast(cam, frame)
            ref, _ = orc.integrate(cam, frame, ris=True, **kw)
            check_gbuffer(ctx.download("GBuffer"), orc.gbuf)
            frac = outliers(gpu, ref[:, :3])
            print(f"sky {hour} cfg {cfg} frame {frame}: colour outliers {frac:.4f}")
            assert frac <= MAX_OUTLIERS
            if kw["use_reservoir"]:
                res = ctx.download("__ris_reservoir")
                hit = orc.gbuf["hit"] == 1
                check_reservoirs(res, orc.res, np.nonzero(hit)[0], f"sky {hour} frame {frame}")
                suns += int((orc.res["light"][hit & (orc.res["has_sample"] == 1)] == len(sc.lights)).sum())
    assert (orc.gbuf["hit"] == 0).any()  # the sky is in view
    if kw["use_reservoir"]:
        assert suns > 0


@pytest.mark.parametrize("hour", [15.5, 6.5, 2.0])
def test_path_tracer_under_the_physical_sky_matches_oracle(hour):
    from hdrestir_b200.context import Context
    sc, cam = _scene(2, hour)
    orc = Oracle(sc, threads=8)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        for frame in range(2):
            ctx.raycast(cam, frame)
            ctx.path_trace(cam, frame, max_depth=4)
            gpu = ctx.download("Color")[:, :3]
            orc.raycast(cam, frame)
            ref, _ = orc.integrate(cam, frame, ris=False, max_depth=4)
            frac = outliers(gpu, ref[:, :3])
            print(f"sky {hour} PT frame {frame}: colour outliers {frac:.4f}")
            assert frac <= MAX_OUTLIERS
    bg = orc.gbuf["hit"] == 0
    assert bg.any()
    if hour != 2.0:
        assert float(ref[bg, :3].max()) > 0.0  # daylight sky on the misses
