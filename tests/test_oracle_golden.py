"""The C oracle against the golden vectors produced by the reference's own
sources (tests/golden/make_golden.py). Everything here is bit-exact: the
oracle and the reference are both float-in-source-order C/C++ built with
-ffp-contract=off on the same libm."""
from pathlib import Path

import numpy as np
import pytest

from hdrestir_b200 import configs
from oracle import oracle as orc

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = {
    0: (dict(width=32, height=24), dict(ris=False, max_depth=4)),
    1: (dict(width=32, height=24, n_lights=128),
        dict(ris=True, candidate_count=16, use_reservoir=False, skip_visibility=True, max_depth=1)),
    2: (dict(width=32, height=24, grid=96, n_spheres=60, n_lights=300),
        dict(ris=True, candidate_count=32, use_reservoir=True, max_depth=1)),
}
RES_FIELDS_ALWAYS = ("m", "wsum", "w")
RES_FIELDS_SAMPLE = ("has_lc", "origin", "vis_tested", "target", "tp")
RES_FIELDS_LIGHT = ("light", "dir", "color", "normal", "dist", "pdf", "pdf_solid")


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def test_rng_streams_match_reference():
    g = np.load(GOLDEN / "rng.npz")
    got = orc.rng_floats(g["seeds"], g["floats"].shape[1])
    assert np.array_equal(bits(got), bits(g["floats"]))


def test_reservoir_known_answers():
    """tests/test_reservoir.cpp:67-76 (weight 6, p-hat 3 -> W = 2) and the zero cases."""
    g = np.load(GOLDEN / "reservoir_kat.npz")["w"]
    lib = orc.lib()
    got = np.array([lib.orc_reservoir_known_answer(6.0, 3.0, 1), lib.orc_reservoir_known_answer(0.0, 1.0, 1),
                    lib.orc_reservoir_known_answer(2.0, 0.0, 1)], np.float32)
    assert got[0] == 2.0 and got[1] == 0.0 and got[2] == 0.0
    assert np.array_equal(bits(got), bits(g))


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_frames_match_reference(cfg):
    scene_kw, kw = CASES[cfg]
    g = np.load(GOLDEN / f"frames_cfg{cfg}.npz")
    sc, cam = configs.small_variant(cfg, **scene_kw)
    o = orc.Oracle(sc, threads=2)
    for f in range(3):
        gb = o.raycast(cam, f)
        ref = g[f"gbuf{f}"]
        assert np.array_equal(gb["prim_id"], ref["prim_id"])
        hit = ref["hit"] == 1
        for field in ("position", "depth", "normal", "smooth_normal", "albedo", "uv", "dpdu", "dpdv"):
            assert np.array_equal(bits(gb[field][hit]), bits(ref[field][hit])), field
        o.integrate(cam, f, **kw)
        o.accumulate(cam, f, firefly=True)
        assert np.array_equal(bits(o.color), bits(g[f"color{f}"])), f"colour frame {f}"
        if kw.get("use_reservoir") and kw.get("ris"):
            r = g[f"res{f}"]
            for field in RES_FIELDS_ALWAYS:
                assert np.array_equal(bits(o.res[field]), bits(r[field])), field
            assert np.array_equal(o.res["has_sample"], r["has_sample"])
            s = r["has_sample"] == 1
            for field in RES_FIELDS_SAMPLE:
                assert np.array_equal(bits(o.res[field][s]), bits(r[field][s])), field
            lc = s & (r["has_lc"] == 1)
            for field in RES_FIELDS_LIGHT:
                assert np.array_equal(bits(o.res[field][lc]), bits(r[field][lc])), field


def test_textured_frames_match_reference():
    """The oracle's texture sampling against the reference's own loader and sampler
    (fixture from tests/golden/make_golden.py textured)."""
    scene_kw, kw = dict(width=32, height=24), dict(ris=True, candidate_count=16, use_reservoir=True, max_depth=1)
    g = np.load(GOLDEN / "frames_textured.npz")
    sc, cam = configs.textured_variant(**scene_kw)
    o = orc.Oracle(sc, threads=2)
    for f in range(2):
        gb = o.raycast(cam, f)
        assert np.array_equal(gb["prim_id"], g[f"gbuf{f}"]["prim_id"])
        o.integrate(cam, f, **kw)
        o.accumulate(cam, f, firefly=True)
        assert np.array_equal(bits(o.color), bits(g[f"color{f}"])), f"colour frame {f}"
        r = g[f"res{f}"]
        for field in RES_FIELDS_ALWAYS:
            assert np.array_equal(bits(o.res[field]), bits(r[field])), field
