"""ctypes wrapper of the reference's own hot-path sources compiled in place
(oracle/_ref/libhdr_ref.so, built by ``make -C oracle ref`` where the reference
tree is present) — TEST INFRASTRUCTURE.

Used to pin the C oracle (tests/test_oracle_pin.py), to generate the golden
fixtures, and as bench.py's CPU baseline when the library is available.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libhdr_ref.so"
# the reference checkout: HDR_REFERENCE_TREE, else "reference" beside this repository
REFERENCE_TREE = Path(os.environ.get("HDR_REFERENCE_TREE", str(HERE.parent.parent / "reference")))

import sys  # noqa: E402

sys.path.insert(0, str(HERE.parent))
from hdrestir_b200 import abi  # noqa: E402
from oracle.oracle import RESERVOIR_DTYPE  # noqa: E402


class RefParams(C.Structure):
    _fields_ = [("pipeline", C.c_int32), ("candidate_count", C.c_int32), ("use_reservoir", C.c_int32),
                ("skip_visibility", C.c_int32), ("max_depth", C.c_int32), ("enable_subsurface", C.c_int32),
                ("max_refl", C.c_int32), ("max_refr", C.c_int32), ("render_ibl_background", C.c_int32),
                ("roulette", C.c_float), ("firefly", C.c_int32), ("accumulate", C.c_int32),
                ("resolution_level", C.c_int32)]


def available() -> bool:
    return LIB.exists()


def build() -> bool:
    """Builds the in-place reference library when the reference tree is present."""
    if not (REFERENCE_TREE / "source" / "restir").exists():
        return LIB.exists()
    targets = ["ref"]
    if (HERE.parent / "hdrestir_b200" / "libhdrestir_b200.so").exists():
        targets.append("ref-gpu")  # the reference pipeline with the GPU passes dropped in
    subprocess.run(["make", "-s", "-C", str(HERE), f"REF={REFERENCE_TREE}", *targets, f"-j{os.cpu_count() or 4}"],
                   check=True)
    return LIB.exists()


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise RuntimeError(f"{LIB} is not built (needs the reference tree: make -C oracle ref)")
        L = C.CDLL(str(LIB))
        vp = C.c_void_p
        L.ref_create.restype = vp
        L.ref_create.argtypes = [C.POINTER(abi.SceneDesc)]
        L.ref_destroy.argtypes = [vp]
        L.ref_clear_persistent.argtypes = [vp]
        L.ref_render_frame.restype = C.c_int
        L.ref_render_frame.argtypes = [vp, C.POINTER(abi.CameraDesc), C.c_int, C.POINTER(RefParams), vp, vp, vp]
        L.ref_render_frame_sampled.restype = C.c_int
        L.ref_render_frame_sampled.argtypes = [vp, C.POINTER(abi.CameraDesc), C.c_int, C.POINTER(RefParams),
                                               C.c_int, C.c_int, vp, C.POINTER(C.c_double)]
        L.ref_trace_rays.argtypes = [vp, vp, C.c_int, vp]
        L.ref_rng_floats.argtypes = [vp, C.c_int, C.c_int, vp]
        L.ref_reservoir_known_answer.restype = C.c_float
        L.ref_reservoir_known_answer.argtypes = [C.c_float, C.c_float, C.c_int]
        L.ref_upscale.restype = C.c_int
        L.ref_upscale.argtypes = [C.c_char_p, vp, C.c_int, C.c_int, C.c_int, vp]
        L.ref_denoise.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.ref_accumulate.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.ref_resolve.restype = C.c_int
        L.ref_resolve.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp]
        L.ref_sky.restype = C.c_int
        L.ref_sky.argtypes = [vp, vp, C.c_int, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Reference:
    """The reference's Scene + passes for one scene description."""

    def __init__(self, scene):
        self._lib = lib()
        self._desc = scene.c_desc()
        self._s = self._lib.ref_create(C.byref(self._desc))
        if not self._s:
            raise RuntimeError("reference harness rejected the scene")

    def close(self):
        if self._s:
            self._lib.ref_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clear_persistent(self):
        self._lib.ref_clear_persistent(self._s)

    def sky(self, dirs):
        """PhysicalSky::Sample along each direction (n x 3 float32) and SampleDirect's
        sun (direction + colour, or None)."""
        d = np.ascontiguousarray(dirs, np.float32)
        out = np.zeros_like(d)
        sun = np.zeros(6, np.float32)
        got = self._lib.ref_sky(self._s, _p(d), len(d), _p(out), _p(sun))
        if got < 0:
            raise RuntimeError("the scene has no physical sky")
        return out, (sun if got else None)

    def render(self, cam, frame, ris=False, candidate_count=16, use_reservoir=True, skip_visibility=False,
               max_depth=32, firefly=True, accumulate=True, resolution_level=0, enable_subsurface=True,
               max_reflection_bounces=8, max_refraction_bounces=8, render_ibl_background=True,
               roulette_aggressiveness=1.0, outputs=("gbuf", "color", "res")):
        div = 1 << max(0, min(4, resolution_level))
        w, h = max(1, (cam.width + div - 1) // div), max(1, (cam.height + div - 1) // div)
        n = w * h
        g = np.zeros(n, abi.GBUFFER_DTYPE) if "gbuf" in outputs else None
        c = np.zeros((n, 4), np.float32) if "color" in outputs else None
        r = np.zeros(n, RESERVOIR_DTYPE) if "res" in outputs else None
        p = RefParams(1 if ris else 0, candidate_count, int(use_reservoir), int(skip_visibility), max_depth,
                      int(enable_subsurface), max_reflection_bounces, max_refraction_bounces,
                      int(render_ibl_background), roulette_aggressiveness, int(firefly), int(accumulate),
                      resolution_level)
        got = self._lib.ref_render_frame(self._s, C.byref(cam.c_desc()), int(frame), C.byref(p), _p(g), _p(c), _p(r))
        if got != n:
            raise RuntimeError(f"reference render failed ({got})")
        return g, c, r

    def trace_rays(self, rays):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.zeros(len(rays), abi.GBUFFER_DTYPE)
        self._lib.ref_trace_rays(self._s, _p(rays), len(rays), _p(out))
        return out


GPU_LIB = HERE / "_ref" / "libhdr_ref_gpu.so"


class RefGpuParams(C.Structure):
    _fields_ = [("pipeline", C.c_int32), ("candidate_count", C.c_int32), ("use_reservoir", C.c_int32),
                ("skip_visibility", C.c_int32), ("max_depth", C.c_int32), ("firefly", C.c_int32),
                ("resolution_level", C.c_int32)]


def gpu_pipeline_available() -> bool:
    return GPU_LIB.exists()


def gpu_pipeline_render(scene, cam, frames, ris=True, candidate_count=16, use_reservoir=True, skip_visibility=False,
                        max_depth=1, firefly=True, resolution_level=0, via_scene=False) -> np.ndarray:
    """The reference's RenderPipeline with the GPU passes of
    hdrestir_b200/integration/gpu_passes.h; returns "Color" after `frames` frames (window size:
    with resolution_level > 0 the pipeline ends with the GPU upscale pass). via_scene: the
    device scene comes only from the reference's Scene inputs, through the scene hand-off of
    hdrestir_b200/integration/scene_handoff.h, and the frames carry that reference Scene."""
    L = C.CDLL(str(GPU_LIB))
    fn = L.refgpu_render_scene if via_scene else L.refgpu_render
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(abi.SceneDesc), C.POINTER(abi.CameraDesc), C.c_int, C.POINTER(RefGpuParams),
                   C.c_void_p]
    desc = scene.c_desc()
    out = np.zeros((cam.width * cam.height, 4), np.float32)
    p = RefGpuParams(1 if ris else 0, candidate_count, int(use_reservoir), int(skip_visibility), max_depth,
                     int(firefly), int(resolution_level))
    n = fn(C.byref(desc), C.byref(cam.c_desc()), int(frames), C.byref(p), _p(out))
    if n != len(out):
        raise RuntimeError("GPU pipeline render failed")
    return out


def handoff_compare(scene) -> int:
    """The scene hand-off's descriptor, built from the reference Scene inputs the
    prims of `scene` make, against `scene`'s own descriptor (host only); 0 = equal."""
    L = C.CDLL(str(GPU_LIB))
    L.refgpu_handoff_compare.restype = C.c_int
    L.refgpu_handoff_compare.argtypes = [C.POINTER(abi.SceneDesc)]
    desc = scene.c_desc()
    return int(L.refgpu_handoff_compare(C.byref(desc)))


def rng_floats(seeds, count) -> np.ndarray:
    seeds = np.ascontiguousarray(seeds, np.uint32)
    out = np.empty((len(seeds), count), np.float32)
    lib().ref_rng_floats(_p(seeds), len(seeds), int(count), _p(out))
    return out


TILE = 16  # the passes' tile size (integration_pass.cpp:184-190, raycast_pass.cpp:91-97)


def cpu_sample(scene, cam, threads: int, frames=(0,), stride: int = 8, offset: int = 3,
               ref: "Reference | None" = None, candidate_count: int = 32, accumulate: bool = True,
               color_out: np.ndarray | None = None):
    """Times the reference pipeline (RaycastPass -> RISPathTracePass(32 candidates,
    reservoir) -> AccumulationPass) on a bounded sample of the real frame.

    Each frame in `frames` runs the reference's own passes on the full-size frame,
    with their 16x16 tile loops restricted to the tile rows offset, offset+stride,
    ... (the shim's WorkParallelForN selection), and AccumulationPass over the whole
    frame. The persistent store carries those rows' reservoirs from frame to frame,
    so later frames do the temporal merge as the GPU frames do. A frame's time is
    (raycast + integration time) x (image rows / rows run) + accumulation time.
    Returns a list of (frame, seconds per full frame, image rows run); `color_out`
    (width*height x 4 float32), when given, receives the last frame's "Color"."""
    os.environ["HDR_REF_THREADS"] = str(threads)
    own = ref is None
    if own:
        ref = Reference(scene)
    p = RefParams(1, candidate_count, 1, 0, 1, 1, 8, 8, 1, 1.0, 1, int(accumulate), 0)
    tiles_y = (cam.height + TILE - 1) // TILE
    out = []
    times = (C.c_double * 3)()
    for f in frames:
        got = ref._lib.ref_render_frame_sampled(ref._s, C.byref(cam.c_desc()), int(f), C.byref(p), stride, offset,
                                                _p(color_out), times)
        if got != cam.width * cam.height:
            raise RuntimeError(f"reference render failed ({got})")
        rows = sum(min(TILE, cam.height - ty * TILE) for ty in range(offset % stride, tiles_y, stride))
        assert int(times[2]) == len(range(offset % stride, tiles_y, stride))
        out.append((int(f), times[0] * cam.height / rows + times[1], rows))
    if own:
        ref.close()
    return out


def upscale(name: str, src: np.ndarray, window_w: int, window_h: int, level: int) -> np.ndarray:
    """The reference's UpscalePass on one buffer: src at the level's rendered size -> window size."""
    comps = {"Color": 4, "Albedo": 3, "Normal": 3, "Depth": 1}[name]
    src = np.ascontiguousarray(src, np.float32)
    out = np.empty((window_w * window_h, comps), np.float32)
    got = lib().ref_upscale(name.encode(), src.ctypes.data_as(C.c_void_p), window_w, window_h, level,
                            out.ctypes.data_as(C.c_void_p))
    assert got == comps
    return out


def denoise(rgba: np.ndarray, width: int, height: int, chromaticity_blur: bool = True) -> np.ndarray:
    """The reference's Denoiser::Run (no OIDN) on an RGBA float image."""
    img = np.ascontiguousarray(rgba, np.float32).copy()
    lib().ref_denoise(img.ctypes.data_as(C.c_void_p), width, height, int(chromaticity_blur))
    return img


def accumulate(color: np.ndarray, accum: np.ndarray, width: int, height: int, frame: int,
               firefly: bool = True) -> None:
    """The reference's AccumulationPass on a caller frame, in place: color and
    accum are (width*height, 4) float32 arrays ("Color" and "__accum_color")."""
    assert color.dtype == np.float32 and accum.dtype == np.float32
    assert color.flags.c_contiguous and accum.flags.c_contiguous
    lib().ref_accumulate(color.ctypes.data_as(C.c_void_p), accum.ctypes.data_as(C.c_void_p), width, height,
                         int(frame), int(firefly))


# component type order of the HdFormat shim (each followed by its 2/3/4-component variants)
_HD_TYPES = {"unorm8": (0, np.uint8), "snorm8": (1, np.int8), "float16": (2, np.uint16), "float32": (3, np.float32),
             "int32": (4, np.int32)}


def resolve(values: np.ndarray, component_type: str, components: int) -> np.ndarray:
    """The reference's HdRestirRenderBuffer filled from a float frame buffer
    (CopyFromFrameBuffer) and resolved: values (pixels, source components) float32
    -> (pixels, components) in the render buffer's component type (float16 as bits)."""
    values = np.ascontiguousarray(values, np.float32)
    pixels, src = values.shape
    code, dt = _HD_TYPES[component_type]
    fmt = 4 * code + components - 1
    out = np.zeros((pixels, components), dt)
    got = lib().ref_resolve(values.ctypes.data_as(C.c_void_p), pixels, src, fmt, out.ctypes.data_as(C.c_void_p))
    assert got == out.nbytes, got
    return out
