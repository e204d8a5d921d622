"""ctypes wrapper of the C oracle (liboracle.so) — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, as the checker / the timed CPU restatement. It is never on the
product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SOURCES = ["orc_core.c", "orc_shade.c"]

import sys  # noqa: E402

sys.path.insert(0, str(HERE.parent))
from hdrestir_b200 import abi  # noqa: E402  (plain struct layouts of include/hdrestir.h)


def build() -> Path:
    srcs = [HERE / s for s in SOURCES]
    hdrs = list(HERE.glob("*.h")) + [HERE.parent / "include" / "hdrestir.h"]
    if LIB.exists() and all(LIB.stat().st_mtime >= p.stat().st_mtime for p in srcs + hdrs):
        return LIB
    cmd = ["gcc", "-O2", "-std=gnu11", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(LIB),
           *map(str, srcs), "-lm", "-lpthread"]
    subprocess.run(cmd, check=True)
    return LIB


class PathParams(C.Structure):
    _fields_ = [("max_depth", C.c_int), ("enable_subsurface", C.c_int), ("max_refl", C.c_int),
                ("max_refr", C.c_int), ("render_ibl_background", C.c_int), ("roulette", C.c_float)]


class RisParams(C.Structure):
    _fields_ = [("candidate_count", C.c_int), ("use_reservoir", C.c_int), ("skip_visibility", C.c_int),
                ("m_cap", C.c_int)]


class FrameParams(C.Structure):
    _fields_ = [("ris", C.c_int), ("path", PathParams), ("ris_params", RisParams)]


MAX_TRACE = 64
RESERVOIR_DTYPE = np.dtype([("has_sample", "<i4"), ("has_lc", "<i4"), ("light", "<i4"), ("origin", "<i4"),
                            ("vis_tested", "<i4"), ("pdf_solid", "<i4"), ("m", "<i4"), ("dir", "<f4", 3),
                            ("color", "<f4", 3), ("normal", "<f4", 3), ("dist", "<f4"), ("pdf", "<f4"),
                            ("target", "<f4"), ("wsum", "<f4"), ("w", "<f4"), ("tp", "<f4", 4)])
TRACE_DTYPE = np.dtype([("n_candidates", "<i4"), ("n_nee_idx", "<i4"), ("nee_light", "<i4", MAX_TRACE),
                        ("ris_choice", "<i4"), ("draws", "<i4"), ("L", "<f4", 4), ("lambda", "<f4", 4)])

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        vp = C.c_void_p
        L.orc_scene_create.restype = vp
        L.orc_scene_create.argtypes = [C.POINTER(abi.SceneDesc)]
        L.orc_scene_destroy.argtypes = [vp]
        L.orc_raycast.argtypes = [vp, C.POINTER(abi.CameraDesc), C.c_int, vp, C.c_int]
        L.orc_integrate.argtypes = [vp, C.POINTER(abi.CameraDesc), C.c_int, C.POINTER(FrameParams), vp, vp, vp,
                                    vp, C.c_int]
        L.orc_raycast_band.argtypes = [vp, C.POINTER(abi.CameraDesc), C.c_int, vp, C.c_int, C.c_int, C.c_int]
        L.orc_integrate_band.argtypes = [vp, C.POINTER(abi.CameraDesc), C.c_int, C.POINTER(FrameParams), vp, vp,
                                         vp, vp, C.c_int, C.c_int, C.c_int]
        L.orc_accumulate.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_accumulate_shader.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_rng_floats.argtypes = [vp, C.c_int, C.c_int, vp]
        L.orc_reservoir_known_answer.restype = C.c_float
        L.orc_reservoir_known_answer.argtypes = [C.c_float, C.c_float, C.c_int]
        L.orc_trace_rays.argtypes = [vp, vp, vp, C.c_int, C.c_int, vp]
        L.orc_scene_sky.restype = C.c_int
        L.orc_scene_sky.argtypes = [vp, vp, C.c_int, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    """CPU restatement of the pipeline for one scene (RaycastPass ->
    PathTracePass | RISPathTracePass -> AccumulationPass)."""

    def __init__(self, scene, threads: int | None = None):
        self._lib = lib()
        self._desc = scene.c_desc()
        self._s = self._lib.orc_scene_create(C.byref(self._desc))
        self.threads = threads or os.cpu_count() or 1
        self.gbuf = self.color = self.accum = self.res = None

    def close(self):
        if self._s:
            self._lib.orc_scene_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ensure(self, n):
        if self.gbuf is None or len(self.gbuf) != n:
            self.gbuf = np.zeros(n, abi.GBUFFER_DTYPE)
            self.color = np.zeros((n, 4), np.float32)
            self.accum = np.zeros((n, 4), np.float32)
            self.res = np.zeros(n, RESERVOIR_DTYPE)

    def clear_persistent(self):
        if self.accum is not None:
            self.accum[:] = 0
            self.res[:] = np.zeros(1, RESERVOIR_DTYPE)

    def sky(self, dirs):
        """The physical sky along each direction (n x 3 float32) and its sun
        (direction + colour, or None)."""
        d = np.ascontiguousarray(dirs, np.float32)
        out = np.zeros_like(d)
        sun = np.zeros(6, np.float32)
        got = self._lib.orc_scene_sky(self._s, _p(d), len(d), _p(out), _p(sun))
        if got < 0:
            raise RuntimeError("the scene has no physical sky")
        return out, (sun if got else None)

    def raycast(self, cam, frame=0) -> np.ndarray:
        n = cam.width * cam.height
        self._ensure(n)
        self._lib.orc_raycast(self._s, C.byref(cam.c_desc()), int(frame), _p(self.gbuf), self.threads)
        return self.gbuf

    def integrate(self, cam, frame, ris=False, candidate_count=16, use_reservoir=True, skip_visibility=False,
                  m_cap=0, max_depth=32, enable_subsurface=True, max_reflection_bounces=8,
                  max_refraction_bounces=8, render_ibl_background=True, roulette_aggressiveness=1.0,
                  trace=False):
        n = cam.width * cam.height
        self._ensure(n)
        fp = FrameParams(int(ris), PathParams(max_depth, int(enable_subsurface), max_reflection_bounces,
                                              max_refraction_bounces, int(render_ibl_background),
                                              roulette_aggressiveness),
                         RisParams(candidate_count, int(use_reservoir), int(skip_visibility), m_cap))
        tr = np.zeros(n, TRACE_DTYPE) if trace else None
        self._lib.orc_integrate(self._s, C.byref(cam.c_desc()), int(frame), C.byref(fp), _p(self.gbuf),
                                _p(self.color), _p(self.res), _p(tr), self.threads)
        return self.color, tr

    def frame_band(self, cam, frame, y0, y1, ris=True, candidate_count=32, use_reservoir=True,
                   skip_visibility=False, max_depth=1, trace=None):
        """Raycast + integration of image rows [y0, y1) (a bounded CPU sample of one frame).
        The pixels of those rows in gbuf / color / res (full-frame arrays) and, when given,
        in `trace` (a full-frame TRACE_DTYPE array) are written; the others are left alone,
        so the reservoirs of a band keep their history from frame to frame."""
        n = cam.width * cam.height
        self._ensure(n)
        cd = cam.c_desc()
        fp = FrameParams(int(ris), PathParams(max_depth, 1, 8, 8, 1, 1.0),
                         RisParams(candidate_count, int(use_reservoir), int(skip_visibility), 0))
        if trace is not None:
            assert trace.dtype == TRACE_DTYPE and len(trace) == n
        self._lib.orc_raycast_band(self._s, C.byref(cd), int(frame), _p(self.gbuf), int(y0), int(y1), self.threads)
        self._lib.orc_integrate_band(self._s, C.byref(cd), int(frame), C.byref(fp), _p(self.gbuf), _p(self.color),
                                     _p(self.res), _p(trace), int(y0), int(y1), self.threads)

    def accumulate(self, cam, frame, firefly=True):
        self._lib.orc_accumulate(_p(self.color), _p(self.accum), cam.width, cam.height, int(frame), int(firefly))
        return self.color

    def trace_rays(self, rays, tmax=None, any_hit=False):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.zeros(len(rays), abi.GBUFFER_DTYPE)
        tm = None if tmax is None else np.ascontiguousarray(tmax, np.float32)
        self._lib.orc_trace_rays(self._s, _p(rays), _p(tm), len(rays), int(any_hit), _p(out))
        return out


def accumulate_frame(color, accum, width, height, frame, firefly=True, mode="parity"):
    """AccumulationPass (mode "parity": the in-place row-major clamp) or the
    GpuAccumulationPass shader (mode "shader") on caller arrays, in place:
    color and accum are (width*height, 4) float32."""
    fn = lib().orc_accumulate if mode == "parity" else lib().orc_accumulate_shader
    assert color.dtype == np.float32 and accum.dtype == np.float32
    assert color.flags.c_contiguous and accum.flags.c_contiguous
    fn(_p(color), _p(accum), int(width), int(height), int(frame), int(firefly))
    return color


def rng_floats(seeds, count) -> np.ndarray:
    seeds = np.ascontiguousarray(seeds, np.uint32)
    out = np.empty((len(seeds), count), np.float32)
    lib().orc_rng_floats(_p(seeds), len(seeds), int(count), _p(out))
    return out
