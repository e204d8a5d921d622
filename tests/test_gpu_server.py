"""Render-job server: every job's image equals the image of the same job
rendered alone with the per-frame passes, in the batched and the serial mode,
and admission by HBM budget queues what does not fit."""
import numpy as np
import pytest

from hdrestir_b200 import abi, configs
from hdrestir_b200.context import Context
from hdrestir_b200.server import Server

pytestmark = pytest.mark.gpu

RIS = dict(candidate_count=16, use_reservoir=True, max_depth=1)
PT = dict(max_depth=3)


def _scenes():
    s2, _ = configs.small_variant(2, 64, 64, grid=64, n_spheres=40, n_lights=200)
    s0, c0 = configs.small_variant(0, 48, 48)
    return s2, s0, c0


def _jobs(c0):
    # (scene index, camera, frames, pipeline, settings)
    return [
        (0, configs.orbit_camera(0.0, 64, 48), 3, "ris", RIS),
        (0, configs.orbit_camera(1.1, 80, 64), 2, "ris", RIS),
        (1, c0, 2, "pt", PT),
        (0, configs.orbit_camera(2.3, 48, 48), 4, "ris", dict(candidate_count=8, use_reservoir=False, max_depth=1)),
        (0, configs.orbit_camera(0.4, 64, 64), 2, "pt", PT),
    ]


def _alone(scene, cam, frames, pipeline, settings):
    with Context(device=0) as ctx:
        ctx.upload_scene(scene)
        for f in range(frames):
            ctx.raycast(cam, f)
            if pipeline == "ris":
                ctx.ris_path_trace(cam, f, **settings)
            else:
                ctx.path_trace(cam, f, **settings)
            ctx.accumulate(f, mode="shader")  # the server accumulates as GpuAccumulationPass
        return ctx.download("Color").copy()


@pytest.mark.parametrize("serial,step_pixels", [(False, 0), (True, 0), (False, 6000)])
def test_server_images_equal_jobs_rendered_alone(serial, step_pixels):
    s2, s0, c0 = _scenes()
    scenes = [s2, s0]
    jobs = _jobs(c0)
    with Server(device=0, serial=serial, step_pixels=step_pixels) as sv:
        ids = [sv.add_scene(s) for s in scenes]
        jid = [sv.submit(ids[si], cam, fr, pipe, **kw) for si, cam, fr, pipe, kw in jobs]
        done, steps, drained = 0, 0, []
        while done < len(jobs):
            n = sv.step()
            done += n
            steps += 1
            fin = sv.finished()
            assert len(fin) == n  # each finished job is reported once, in the step that ends it
            drained += fin
            assert steps < 100
        assert sorted(drained) == sorted(jid) and sv.finished() == []
        assert all(sv.state(j)[0] == abi.JOB_DONE for j in jid)
        got = [sv.take(j) for j in jid]
    if serial:
        assert steps == sum(j[2] for j in jobs)  # one frame of one job per step
    elif step_pixels:
        assert steps > max(j[2] for j in jobs)  # fewer jobs per step
    else:
        assert steps == max(j[2] for j in jobs)  # every admitted job advances each step
    for (si, cam, fr, pipe, kw), g in zip(jobs, got):
        want = _alone(scenes[si], cam, fr, pipe, kw)
        assert np.array_equal(g.view(np.uint32), want.view(np.uint32))


def test_server_admission_by_budget():
    s2, _, _ = _scenes()
    cam = configs.orbit_camera(0.0, 128, 128)
    budget = 24 << 20  # room for one 128x128 RIS job (about 17.7 MB) at a time
    with Server(device=0, hbm_budget=budget) as sv:
        sid = sv.add_scene(s2)
        jid = [sv.submit(sid, cam, 2, "ris", **RIS) for _ in range(3)]
        done = sv.step()
        queued, running, in_use = sv.load()
        assert (queued, running) == (2, 1) and 0 < in_use <= budget
        for _ in range(10):
            done += sv.step()
        assert done == 3 and sv.load()[:2] == (0, 0)
        imgs = [sv.take(j) for j in jid]
    assert all(np.array_equal(imgs[0].view(np.uint32), im.view(np.uint32)) for im in imgs[1:])


def test_server_rejects_bad_jobs():
    s2, _, _ = _scenes()
    cam = configs.orbit_camera(0.0, 32, 32)
    with Server(device=0, hbm_budget=1 << 20) as sv:
        sid = sv.add_scene(s2)
        with pytest.raises(abi.HdrError):
            sv.submit(sid + 5, cam, 1, "ris", **RIS)
        with pytest.raises(abi.HdrError):
            sv.submit(sid, cam, 0, "ris", **RIS)
        with pytest.raises(abi.HdrError) as e:  # above the whole budget
            sv.submit(sid, configs.orbit_camera(0.0, 512, 512), 1, "ris", **RIS)
        assert e.value.status == abi.HDR_ENOMEM


@pytest.mark.parametrize("serial", [False, True])
def test_reused_contexts_give_the_images_of_fresh_ones(serial):
    """Jobs taken one after another hand their contexts (buffers kept, history zeroed) to the
    next jobs of the same size; every image equals the job rendered alone."""
    s2, _, _ = _scenes()
    jobs = [(configs.orbit_camera(0.3 * k, 64, 48), 2 + (k % 2), "ris", RIS) for k in range(4)]
    jobs += [(configs.orbit_camera(0.5 * k, 48, 48), 2, "pt", PT) for k in range(2)]
    with Server(device=0, serial=serial) as sv:
        sid = sv.add_scene(s2)
        for cam, fr, pipe, kw in jobs:
            jid = sv.submit(sid, cam, fr, pipe, **kw)
            for _ in range(20):
                if sv.state(jid)[0] == abi.JOB_DONE:
                    break
                sv.step()
            got = sv.take(jid)
            want = _alone(s2, cam, fr, pipe, kw)
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("age_weight,big_last", [(-1.0, True), (0.0, False)])
def test_age_credit_bounds_the_wait_of_an_early_large_job(age_weight, big_last):
    """One job per step (step_pixels below every job's size), a large job submitted first and a
    small one arriving at every step. Least remaining work alone (age_weight < 0) runs the large
    job only after the small ones stop arriving; with the default credit (half the pixels served
    since it arrived) it finishes while they still arrive."""
    s2, _, _ = _scenes()
    with Server(device=0, step_pixels=256, age_weight=age_weight) as sv:
        sid = sv.add_scene(s2)
        big = sv.submit(sid, configs.orbit_camera(0.0, 32, 32), 4, "ris", **RIS)
        small = configs.orbit_camera(1.0, 16, 16)
        order = []
        for _ in range(60):
            sv.submit(sid, small, 1, "ris", **RIS)
            sv.step()
            order += sv.finished()
        for _ in range(10):
            sv.step()
            order += sv.finished()
        assert len(order) == 61
    assert (order[-1] == big) == big_last
    if not big_last:  # 4096 px of work starts once its credit has passed 3,840 px: after 30 small jobs
        assert order.index(big) < 40
