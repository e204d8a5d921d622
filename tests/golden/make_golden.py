"""Generates the golden fixtures from the reference's own sources compiled in
place (oracle/_ref, ``make -C oracle ref``). Run where the reference tree is
present:

    python tests/golden/make_golden.py

Outputs (small, committed):
  rng.npz            Restir::Rng NextFloat streams for a set of seeds
  frames_cfg{0,1,2}.npz
                     GBuffer / Color (after AccumulationPass) / "__ris_reservoir"
                     of the reference passes on test-sized variants of the
                     benchmark scenes, frames 0-2
  reservoir_kat.npz  WeightedReservoir known answers (tests/test_reservoir.cpp)
  frames_textured.npz
                     the same for the textured config-2 variant (PreviewSurface
                     diffuse / metallic / roughness / normal textures), frames 0-1
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from hdrestir_b200 import configs  # noqa: E402
from oracle import refharness  # noqa: E402

# test-sized variants of the three benchmark scenes and their pipelines
CASES = {
    0: (dict(width=32, height=24), dict(ris=False, max_depth=4)),
    1: (dict(width=32, height=24, n_lights=128),
        dict(ris=True, candidate_count=16, use_reservoir=False, skip_visibility=True, max_depth=1)),
    2: (dict(width=32, height=24, grid=96, n_spheres=60, n_lights=300),
        dict(ris=True, candidate_count=32, use_reservoir=True, max_depth=1)),
}
FRAMES = 3
TEXTURED = (dict(width=32, height=24), dict(ris=True, candidate_count=16, use_reservoir=True, max_depth=1))
RNG_SEEDS = np.array([0, 1, 7, 1234 ^ 56, 0xFFFFFFFF, 0xC0FFEE00, 12345 * 3 ^ 77] + list(range(1000, 1025)), np.uint32)
RNG_COUNT = 700


def textured():
    scene_kw, kw = TEXTURED
    sc, cam = configs.textured_variant(**scene_kw)
    ref = refharness.Reference(sc)
    out = {}
    for f in range(2):
        g, c, r = ref.render(cam, f, accumulate=True, firefly=True, **kw)
        out[f"gbuf{f}"], out[f"color{f}"], out[f"res{f}"] = g, c, r
    np.savez_compressed(HERE / "frames_textured.npz", **out)
    ref.close()


def main():
    if not refharness.build():
        raise SystemExit("the reference tree is needed to build oracle/_ref")
    np.savez_compressed(HERE / "rng.npz", seeds=RNG_SEEDS, floats=refharness.rng_floats(RNG_SEEDS, RNG_COUNT))
    L = refharness.lib()
    kat = np.array([L.ref_reservoir_known_answer(6.0, 3.0, 1), L.ref_reservoir_known_answer(0.0, 1.0, 1),
                    L.ref_reservoir_known_answer(2.0, 0.0, 1)], np.float32)
    np.savez_compressed(HERE / "reservoir_kat.npz", w=kat)
    for cfg, (scene_kw, kw) in CASES.items():
        sc, cam = configs.small_variant(cfg, **scene_kw)
        ref = refharness.Reference(sc)
        out = {}
        for f in range(FRAMES):
            g, c, r = ref.render(cam, f, accumulate=True, firefly=True, **kw)
            out[f"gbuf{f}"], out[f"color{f}"], out[f"res{f}"] = g, c, r
        np.savez_compressed(HERE / f"frames_cfg{cfg}.npz", **out)
        ref.close()
    textured()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    if sys.argv[1:] == ["textured"]:  # only the textured fixture
        refharness.build()
        textured()
    else:
        main()
