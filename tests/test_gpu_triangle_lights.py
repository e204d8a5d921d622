"""Emissive-triangle lights (extension, HDR_LIGHT_TRIANGLE; the reference has no
emissive-geometry light, so the oracle's restatement of the same sampling is the check):
a scene whose lights alternate rect and triangle, rendered by the GPU passes and by the
oracle. Reservoir M bit-exact, winner light index and WSum / W through the usual checks,
colour within the radiance tolerance; the triangle lights must receive winners. The same
for spectral blackbody emission (extension, hdr_light_desc.temperature)."""
import numpy as np
import pytest

from hdrestir_b200 import abi, configs
from oracle.oracle import Oracle
from tests.parity_checks import MAX_OUTLIERS, check_reservoirs, outliers, reservoir_fields

pytestmark = pytest.mark.gpu


def _scene():
    sc, cam = configs.small_variant(2, 96, 64, grid=64, n_spheres=40, n_lights=200)
    for k, light in enumerate(sc.lights):
        if k % 2 == 0 and light.type == abi.LIGHT_RECT:
            light.type = abi.LIGHT_TRIANGLE
    return sc, cam


@pytest.mark.parametrize("kw", [dict(ris=True, candidate_count=32, use_reservoir=True, max_depth=1),
                                dict(ris=True, candidate_count=16, use_reservoir=False, max_depth=1),
                                dict(ris=False, max_depth=3)])
def test_triangle_lights_match_oracle(kw):
    from hdrestir_b200.context import Context
    sc, cam = _scene()
    kw = dict(kw)
    ris = kw.pop("ris")
    tri = np.array([light.type == abi.LIGHT_TRIANGLE for light in sc.lights])
    assert 0 < tri.sum() < len(tri)
    orc = Oracle(sc)
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
            if ris and kw.get("use_reservoir"):
                res = ctx.download("__ris_reservoir")
                idx = np.arange(res.shape[1])
                check_reservoirs(res, orc.res, idx, f"triangle lights, frame {frame}")
                has, light, _, _, _ = reservoir_fields(res)
                won = light[has == 1]
                assert tri[won].mean() > 0.1  # triangle lights win reservoirs
            frac = outliers(gpu[:, :3], ref[:, :3])
            print(f"triangle lights {kw}, frame {frame}: outlier fraction {frac:.4f}")
            assert frac <= MAX_OUTLIERS and float(ref[:, :3].mean()) > 0.0


@pytest.mark.parametrize("kw", [dict(ris=True, candidate_count=32, use_reservoir=True, max_depth=1),
                                dict(ris=False, max_depth=3)])
def test_blackbody_lights_match_oracle(kw):
    """Spectral blackbody emission (extension, hdr_light_desc.temperature): every third light,
    rect or triangle, emits Planck's spectrum at 2000-9000 K. GPU against the oracle as above;
    the image must differ from the one the lights' colours give."""
    from hdrestir_b200.context import Context
    sc, cam = _scene()
    temps = np.linspace(2000.0, 9000.0, len(sc.lights))
    for k, light in enumerate(sc.lights):
        if k % 3 == 0:
            light.temperature = float(temps[k])
    kw = dict(kw)
    ris = kw.pop("ris")
    orc = Oracle(sc)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        ctx.raycast(cam, 0)
        (ctx.ris_path_trace if ris else ctx.path_trace)(cam, 0, **kw)
        gpu = ctx.download("Color")
        if ris:
            res = ctx.download("__ris_reservoir")
    orc.raycast(cam, 0)
    ref, _ = orc.integrate(cam, 0, ris=ris, **kw)
    if ris:
        check_reservoirs(res, orc.res, np.arange(res.shape[1]), "blackbody lights")
    frac = outliers(gpu[:, :3], ref[:, :3])
    print(f"blackbody lights {kw}: outlier fraction {frac:.4f}")
    assert frac <= MAX_OUTLIERS and float(ref[:, :3].mean()) > 0.0
    plain, _ = _scene()
    orc_plain = Oracle(plain)
    orc_plain.raycast(cam, 0)
    ref_plain, _ = orc_plain.integrate(cam, 0, ris=ris, **kw)
    assert outliers(ref[:, :3], ref_plain[:, :3]) > 0.05
