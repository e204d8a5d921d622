"""Moved instances (hdr_scene_set_instance_transforms): the instance records and
the TLAS rebuilt on the device give the images of a fresh upload of the scene
with the new transforms, bit for bit, for the GBuffer, a RIS frame and a
path-traced frame, through several moves, with the transforms in host or
device memory."""
import copy

import numpy as np
import pytest

from hdrestir_b200 import abi, configs
from hdrestir_b200.context import Context
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

RIS = dict(candidate_count=16, use_reservoir=True, max_depth=1)
PT = dict(max_depth=3)


def _scene():
    return configs.small_variant(2, 64, 48, grid=64, n_spheres=60, n_lights=200)


def _moved(sc, seed, mode="random"):
    """The scene's spheres (instances 1..) under new transforms; the ground keeps its own."""
    rng = np.random.default_rng(seed)
    xf = np.stack([np.asarray(i.transform, np.float32).reshape(4, 4) for i in sc.instances])
    for k in range(1, len(xf)):
        if mode == "stacked":  # every sphere at one point: the partition falls back to halves
            t = np.eye(4, dtype=np.float32)
            t[:3, :3] *= 0.3
            t[3, :3] = (0.0, 0.3, 0.0)
        elif mode == "flat" and k % 7 == 0:  # singular: the inverse takes GfMatrix4d's FLT_MAX scale
            t = xf[k].copy()
            t[:, 1] = 0.0
            t[3, 3] = 1.0
        else:
            t = xf[k].copy()
            s = float(rng.uniform(0.6, 1.6))
            t[:3, :3] *= s
            t[3, :3] += rng.uniform(-1.5, 1.5, 3).astype(np.float32) * np.float32([1, 0, 1])
        xf[k] = t
    out = copy.deepcopy(sc)
    for inst, t in zip(out.instances, xf):
        inst.transform = t.copy()
    return out, xf


def _render(ctx, cam, frames=(0,)):
    imgs = []
    for f in frames:
        ctx.raycast(cam, f)
        g = ctx.download("GBuffer").copy()
        ctx.ris_path_trace(cam, f, **RIS)
        ris = ctx.download("Color").copy()
        ctx.path_trace(cam, f, **PT)
        pt = ctx.download("Color").copy()
        imgs.append((g, ris, pt))
    return imgs


def _same(a, b):
    for (ga, ra, pa), (gb, rb, pb) in zip(a, b):
        assert np.array_equal(ga.view(np.uint8), gb.view(np.uint8))
        assert np.array_equal(ra.view(np.uint32), rb.view(np.uint32))
        assert np.array_equal(pa.view(np.uint32), pb.view(np.uint32))


@pytest.mark.parametrize("mode", ["random", "stacked", "flat"])
def test_moved_instances_equal_a_fresh_upload(mode):
    sc, cam = _scene()
    moved, xf = _moved(sc, 11, mode)
    with Context(device=0) as a, Context(device=0) as b:
        a.upload_scene(sc)
        a.set_instance_transforms(xf)
        b.upload_scene(moved)
        _same(_render(a, cam, (0, 1)), _render(b, cam, (0, 1)))


def test_a_sequence_of_moves_keeps_the_reservoir_history():
    """Frames rendered between moves carry their reservoirs on; each frame equals a
    context that re-uploads the moved scene (an upload keeps the reservoir buffers too)."""
    sc, cam = _scene()
    steps = [_moved(sc, 100 + k) for k in range(3)]
    with Context(device=0) as a, Context(device=0) as b:
        a.upload_scene(sc)
        b.upload_scene(sc)
        for f, (moved, xf) in enumerate(steps):
            a.set_instance_transforms(xf)
            b.upload_scene(moved)
            _same(_render(a, cam, (f,)), _render(b, cam, (f,)))


def test_transforms_from_device_memory():
    torch = pytest.importorskip("torch")
    sc, cam = _scene()
    moved, xf = _moved(sc, 5)
    with Context(device=0) as a, Context(device=0) as b:
        a.upload_scene(sc)
        a.set_instance_transforms(torch.from_numpy(xf.reshape(-1, 16)).cuda())
        b.upload_scene(moved)
        _same(_render(a, cam), _render(b, cam))


def test_moved_gbuffer_matches_the_oracle():
    sc, cam = _scene()
    moved, xf = _moved(sc, 23)
    with Context(device=0) as a:
        a.upload_scene(sc)
        a.set_instance_transforms(xf)
        a.raycast(cam, 0)
        g = a.download("GBuffer")
    o = Oracle(moved).raycast(cam, 0)
    hit = o["hit"] == 1
    assert hit.sum() > 0 and np.array_equal(g["hit"], o["hit"])
    for f in ("prim_id", "tri_id"):
        assert np.array_equal(g[f], o[f])
    for f in ("position", "depth", "normal"):
        assert np.array_equal(g[f][hit].view(np.uint32), o[f][hit].view(np.uint32)), f


def test_rejected_moves():
    sc, cam = _scene()
    _, xf = _moved(sc, 1)
    with Context(device=0) as a, Context(device=0) as b, Context(device=0, wide_bvh=True) as w:
        with pytest.raises(abi.HdrError) as e:
            a.set_instance_transforms(xf)
        assert e.value.status == abi.HDR_ENOSCENE
        a.upload_scene(sc)
        with pytest.raises(abi.HdrError):  # one transform short
            a.set_instance_transforms(xf[:-1])
        w.upload_scene(sc)
        with pytest.raises(abi.HdrError):  # the wide walk keeps its host-built TLAS
            w.set_instance_transforms(xf)
        b.share_scene(a)
        with pytest.raises(abi.HdrError):  # a shared scene is not moved under the other context
            a.set_instance_transforms(xf)
        b.upload_scene(sc)  # b lets go of a's scene
        a.set_instance_transforms(xf)
        with pytest.raises(abi.HdrError):  # the moved scene's wide TLAS was not rebuilt
            w.share_scene(a)
