"""A frame's pass chain recorded as one CUDA graph (hdr_graph_begin / _end /
_launch) gives exactly the buffers of the same calls made one by one: ReSTIR
(wavefront), the one-kernel RIS form, the wavefront PathTracer, and the orbit
extensions (reprojection, spatial reuse). Later frames update the executable
graph in place; calls that cannot be recorded fail and leave the recording
usable; a pass that fails while recording gets the recording discarded."""
import numpy as np
import pytest

from hdrestir_b200 import abi, configs
from hdrestir_b200.context import Context

pytestmark = pytest.mark.gpu

BUFFERS = ("Color", "__accum_color")


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _run(sc, cams, frames, passes, graph, moving=False):
    """Renders `frames` frames (camera cams(f)); frame 0 always eagerly (it sizes
    the buffers), the rest eagerly or as a graph: a static camera's frame 1 is
    recorded and every later frame replays it with its own frame index; a moving
    camera records every frame. Returns the buffers after every frame and the
    graph statistics."""
    out = []
    with Context(device=0, timings=True) as ctx:
        ctx.upload_scene(sc)
        for f in range(frames):
            if graph and (f == 1 or (moving and f > 1)):
                ctx.record_frame(lambda: passes(ctx, cams(f), f))
            elif graph and f > 1:
                ctx.graph_launch(f)
            else:
                passes(ctx, cams(f), f)
            ctx.synchronize()
            snap = {n: ctx.download(n).copy() for n in BUFFERS}
            try:
                snap["__ris_reservoir"] = ctx.download("__ris_reservoir").copy()
            except abi.HdrError:
                pass
            out.append(snap)
        info = ctx.graph_info()
    return out, info


def _restir(ctx, cam, f, **kw):
    ctx.raycast(cam, f)
    ctx.ris_path_trace(cam, f, candidate_count=32, use_reservoir=True, max_depth=1, **kw)
    ctx.accumulate(f, firefly=True, mode="parity")


def _pt(ctx, cam, f):
    ctx.raycast(cam, f)
    ctx.path_trace(cam, f, max_depth=4)
    ctx.accumulate(f, firefly=True, mode="shader")


CASES = {
    "restir_wavefront": (2, lambda c, cam, f: _restir(c, cam, f), False),
    "restir_one_kernel": (2, lambda c, cam, f: _restir(c, cam, f, one_kernel=True), False),
    "path_tracer_wavefront": (0, _pt, False),
    "orbit_reproject_spatial": (2, lambda c, cam, f: _restir(c, cam, f, m_cap=20, spatial_neighbors=5,
                                                              spatial_radius=8.0, reproject=True), True),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_recorded_frames_equal_eager_frames(name):
    cfg, passes, moving = CASES[name]
    sc, cam = configs.small_variant(cfg, 80, 48, **({"grid": 96, "n_spheres": 60, "n_lights": 300}
                                                      if cfg == 2 else {}))
    cams = (lambda f: configs.orbit_camera(0.01 * f, 80, 48)) if moving else (lambda f: cam)
    frames = 5
    want, _ = _run(sc, cams, frames, passes, graph=False)
    got, info = _run(sc, cams, frames, passes, graph=True, moving=moving)
    for f in range(frames):
        for n in want[f]:
            assert np.array_equal(_bits(got[f][n]), _bits(want[f][n])), f"{name}: frame {f} {n} differs"
    assert info["instantiations"] == 1, info
    # a moving camera's frames 2.. are recorded again and update the first graph in place
    assert info["updates"] == (frames - 2 if moving else 0), info
    assert info["kernels"] >= 3, info


def test_recorded_passes_render_one_frame_index():
    sc, cam = configs.small_variant(2, 64, 32, grid=96, n_spheres=40, n_lights=100)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        _restir(ctx, cam, 0)
        ctx.graph_begin()
        ctx.raycast(cam, 1)
        with pytest.raises(abi.HdrError) as e:
            ctx.ris_path_trace(cam, 2, candidate_count=32, use_reservoir=True, max_depth=1)
        assert e.value.status == abi.HDR_EINVAL
        with pytest.raises(abi.HdrError):
            ctx.graph_end()  # discarded: a recorded pass failed


def test_calls_that_cannot_be_recorded_fail_and_the_recording_survives():
    sc, cam = configs.small_variant(2, 64, 32, grid=96, n_spheres=40, n_lights=100)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        _restir(ctx, cam, 0)
        want_launches = ctx.launch_count()
        ctx.graph_begin()
        _restir(ctx, cam, 1)
        for call in (lambda: ctx.download("Color"), ctx.synchronize, lambda: ctx.region_begin(0),
                     lambda: ctx.pass_times(), ctx.clear_persistent, ctx.graph_launch, ctx.graph_begin):
            with pytest.raises(abi.HdrError) as e:
                call()
            assert e.value.status == abi.HDR_EINVAL
        assert ctx.launch_count() == want_launches  # recorded kernels count when the graph runs
        ctx.graph_end()
        ctx.graph_launch()
        ctx.synchronize()
        rec = ctx.graph_info()["kernels"]
        assert ctx.launch_count() == want_launches + 1 + rec  # the frame-slot store, then the graph
        got = ctx.download("Color").copy()
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        _restir(ctx, cam, 0)
        _restir(ctx, cam, 1)
        assert np.array_equal(_bits(ctx.download("Color")), _bits(got))


def test_a_pass_that_fails_while_recording_discards_the_recording():
    sc, cam = configs.small_variant(2, 64, 32, grid=96, n_spheres=40, n_lights=100)
    big = configs.orbit_camera(0.0, 96, 40)
    with Context(device=0) as ctx:
        ctx.upload_scene(sc)
        with pytest.raises(abi.HdrError):
            ctx.graph_launch()  # nothing recorded yet
        _restir(ctx, cam, 0)
        ctx.record_frame(lambda: _restir(ctx, cam, 1))
        ctx.graph_begin()
        with pytest.raises(abi.HdrError) as e:
            ctx.raycast(big, 2)  # another frame size: its GBuffer would be allocated
        assert e.value.status == abi.HDR_EINVAL
        with pytest.raises(abi.HdrError):
            ctx.graph_end()  # discarded: the record lacks the failed pass
        ctx.graph_launch()  # the previous graph (frame 1) is kept and still runs
        ctx.synchronize()
        assert ctx.graph_info()["instantiations"] == 1
