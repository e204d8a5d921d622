"""Parity at the benchmarked sizes: configs 0, 1 and 2 at full resolution on
their full scenes, against the CPU oracle, through the C ABI.

* config 0: 256x256, PathTracer, maxDepth 4, four frames with accumulation;
* config 1: 512x512, 1,024 rect lights, RIS 16 candidates, no reservoir,
  skipVisibility; every pixel;
* config 2: 1920x1080, 1.03 M triangles (depth-38 trees, just under the
  40-entry shared-memory traversal stack), 10,000 rect lights, ReSTIR 32
  candidates with temporal reuse; the GPU renders whole frames, the oracle
  renders row bands spread over the frame (its reservoirs keep their history
  band by band, since reuse is per pixel: ris_direct_light_integrator.cpp:
  121-185), three frames.

Contract (hazards H1-H5 of the parity plan): GBuffer (instance, triangle, t and
every attribute) bit-exact; NEE light-selection indices
(UniformLightSampler::ProposeCandidate, uniform_light_sampler.cpp:22-35)
bit-exact; reservoir CandidateCount (M) bit-exact; reservoir winner (engaged
sample, light index) equal except on at most 1e-4 of the pixels, which a
ulp-level weight difference can flip (reservoir.h:76-125); WSum, W and colour
within 1e-4 relative on all but 1 % of the pixels.
"""
import numpy as np
import pytest

from hdrestir_b200 import configs
from oracle.oracle import TRACE_DTYPE, Oracle
from tests.parity_checks import MAX_OUTLIERS, check_gbuffer, check_nee, check_reservoirs, outliers

pytestmark = pytest.mark.gpu


def test_config0_full_path_trace_matches_oracle():
    from hdrestir_b200.context import Context
    sc, cam = configs.config0()
    assert (cam.width, cam.height) == (256, 256)
    orc = Oracle(sc)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        ctx.clear_persistent()
        for frame in range(4):
            ctx.raycast(cam, frame)
            ctx.path_trace(cam, frame, max_depth=4)
            gpu = ctx.download("Color").copy()
            g = ctx.download("GBuffer")
            o = orc.raycast(cam, frame)
            check_gbuffer(g, o)
            ref, _ = orc.integrate(cam, frame, ris=False, max_depth=4)
            frac = outliers(gpu[:, :3], ref[:, :3])
            print(f"config 0 frame {frame}: colour outliers {frac:.2e}")
            assert frac <= MAX_OUTLIERS
            ctx.accumulate(frame, firefly=True)
            orc.accumulate(cam, frame, firefly=True)
            frac = outliers(ctx.download("Color")[:, :3], orc.color[:, :3])
            print(f"config 0 frame {frame}: accumulated outliers {frac:.2e}")
            assert frac <= MAX_OUTLIERS


def test_config1_full_ris_matches_oracle():
    from hdrestir_b200.context import Context
    sc, cam = configs.config1()
    assert (cam.width, cam.height) == (512, 512) and len(sc.lights) == 1024
    orc = Oracle(sc)
    ris = dict(candidate_count=16, use_reservoir=False, skip_visibility=True, max_depth=1)
    with Context(device=0, record_lights=True) as ctx:
        ctx.upload_scene(sc)
        for frame in range(2):
            ctx.raycast(cam, frame)
            ctx.ris_path_trace(cam, frame, **ris)
            gpu = ctx.download("Color").copy()
            g = ctx.download("GBuffer")
            lights = ctx.download("__ris_nee_lights").view(np.int32)
            o = orc.raycast(cam, frame)
            check_gbuffer(g, o)
            ref, tr = orc.integrate(cam, frame, ris=True, trace=True, **ris)
            check_nee(lights, tr, o["hit"] == 1, 8, f"config 1 frame {frame}")
            frac = outliers(gpu[:, :3], ref[:, :3])
            print(f"config 1 frame {frame}: colour outliers {frac:.2e}")
            assert frac <= MAX_OUTLIERS


def _bands(height, n_bands=8, rows=4):
    step = height // n_bands
    return [(k * step + step // 3, k * step + step // 3 + rows) for k in range(n_bands)]


@pytest.mark.parametrize("skip_visibility", [False])
def test_config2_full_scene_restir_bands_match_oracle(skip_visibility):
    from hdrestir_b200.context import Context
    sc, cam = configs.config2()
    assert (cam.width, cam.height) == (1920, 1080) and len(sc.lights) == 10000
    w, h = cam.width, cam.height
    bands = _bands(h)
    idx = np.concatenate([np.arange(y0 * w, y1 * w) for y0, y1 in bands])
    orc = Oracle(sc)
    ris = dict(candidate_count=32, use_reservoir=True, skip_visibility=skip_visibility, max_depth=1)
    trace = np.zeros(w * h, TRACE_DTYPE)
    with Context(device=0, record_lights=True) as ctx:
        ctx.upload_scene(sc)
        ctx.clear_persistent()
        for frame in range(3):
            ctx.raycast(cam, frame)
            ctx.ris_path_trace(cam, frame, **ris)
            gpu = ctx.download("Color").copy()
            g = ctx.download("GBuffer")
            res = ctx.download("__ris_reservoir")
            lights = ctx.download("__ris_nee_lights").view(np.int32)
            trace[:] = np.zeros(1, TRACE_DTYPE)
            for y0, y1 in bands:
                orc.frame_band(cam, frame, y0, y1, trace=trace, **ris)
            label = f"config 2 frame {frame}"
            check_gbuffer(g, orc.gbuf, idx)
            hit = np.zeros(w * h, bool)
            hit[idx] = orc.gbuf["hit"][idx] == 1
            assert hit.sum() > 0.5 * len(idx)
            check_nee(lights, trace, hit, 16, label)
            check_reservoirs(res, orc.res, idx, label)
            frac = outliers(gpu[idx, :3], orc.color[idx, :3])
            print(f"{label}: colour outliers {frac:.2e} over {len(idx)} pixels")
            assert frac <= MAX_OUTLIERS
