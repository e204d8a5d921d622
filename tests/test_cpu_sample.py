"""The CPU baseline's frame sample: the reference's own passes run on chosen
16x16 tile rows of the real frame (the work-loop selection of the oracle shim)
compute exactly those rows of a full frame, reservoir history included, so the
timed sample is a part of the real frame's work and nothing else."""
import numpy as np
import pytest

from hdrestir_b200 import configs
from oracle import refharness

pytestmark = pytest.mark.skipif(not refharness.available(), reason="reference library not built")


def test_sampled_tile_rows_equal_full_frame_rows():
    sc, cam = configs.small_variant(2, 96, 80, grid=64, n_spheres=40, n_lights=200)
    stride, offset = 3, 1
    full = refharness.Reference(sc)
    part = refharness.Reference(sc)
    out = np.zeros((cam.width * cam.height, 4), np.float32)
    rows = [y for ty in range(offset, (cam.height + 15) // 16, stride)
            for y in range(ty * 16, min(cam.height, ty * 16 + 16))]
    for f in range(3):
        _, c_full, _ = full.render(cam, f, ris=True, candidate_count=32, use_reservoir=True, max_depth=1,
                                   accumulate=False)
        got = refharness.cpu_sample(sc, cam, 4, frames=(f,), stride=stride, offset=offset, ref=part,
                                    accumulate=False, color_out=out)
        assert got[0][2] == len(rows)
        img_full = c_full.reshape(cam.height, cam.width, 4)
        img_part = out.reshape(cam.height, cam.width, 4)
        assert np.array_equal(img_part[rows].view(np.uint32), img_full[rows].view(np.uint32)), f"frame {f}"
        others = np.setdiff1d(np.arange(cam.height), rows)
        assert not img_part[others].any(), "rows outside the sample must not be rendered"
