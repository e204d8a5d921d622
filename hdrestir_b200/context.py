"""Python handle on one ``hdr_ctx``: resident scene, named device frame
buffers and the pass entry points of include/hdrestir.h."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .scene import Camera, Scene

BUFFER_LAYOUT = {  # name -> (dtype, trailing shape)
    "Color": (np.float32, (4,)),
    "__accum_color": (np.float32, (4,)),
    "Depth": (np.float32, ()),
    "Albedo": (np.float32, (3,)),
    "Normal": (np.float32, (3,)),
}


def ris_params(candidate_count=16, use_reservoir=True, skip_visibility=False, m_cap=0, trace_all_rays=False,
               one_kernel=False, spatial_neighbors=0, spatial_radius=0.0, reproject=False,
               **settings) -> abi.RisParams:
    p = abi.RisParams()
    p.path = path_settings(**settings)
    p.candidate_count, p.use_reservoir, p.skip_visibility = int(candidate_count), int(use_reservoir), int(
        skip_visibility)
    p.m_cap = int(m_cap)
    p.spatial_neighbors, p.spatial_radius = int(spatial_neighbors), float(spatial_radius)
    p.flags = ((abi.RIS_TRACE_ALL_RAYS if trace_all_rays else 0) | (abi.RIS_ONE_KERNEL if one_kernel else 0)
               | (abi.RIS_REPROJECT if reproject else 0))
    return p


def ris_path_trace_batch(contexts, cameras, frame_indices, **ris) -> None:
    """One wavefront RIS frame for several images (one Context each, all sharing
    one scene via Context.share_scene); each image gets what ris_path_trace gives it."""
    n = len(contexts)
    ctxs = (C.c_void_p * n)(*[c._h for c in contexts])
    cams = (abi.CameraDesc * n)(*[cam.c_desc() for cam in cameras])
    frames = (C.c_int32 * n)(*[int(f) for f in frame_indices])
    p = ris_params(**ris)
    params = (abi.RisParams * n)(*([p] * n))
    lib = abi.lib()
    abi.check(lib.hdr_ris_path_trace_batch(ctxs, n, cams, frames, params))


def path_trace_batch(contexts, cameras, frame_indices, **settings) -> None:
    """One PathTracePass launch for several images (Contexts sharing one scene)."""
    n = len(contexts)
    ctxs = (C.c_void_p * n)(*[c._h for c in contexts])
    cams = (abi.CameraDesc * n)(*[cam.c_desc() for cam in cameras])
    frames = (C.c_int32 * n)(*[int(f) for f in frame_indices])
    p = path_settings(**settings)
    params = (abi.PathSettings * n)(*([p] * n))
    abi.check(abi.lib().hdr_path_trace_batch(ctxs, n, cams, frames, params))


def trim_frame_memory(device: int = 0, keep_bytes: int = 0) -> None:
    """Returns the frame-buffer pool's unused memory beyond keep_bytes to the device."""
    abi.check(abi.lib().hdr_trim_frame_memory(int(device), int(keep_bytes)))


def path_settings(max_depth=32, enable_subsurface=True, max_reflection_bounces=8, max_refraction_bounces=8,
                  render_ibl_background=True, roulette_aggressiveness=1.0) -> abi.PathSettings:
    """PathTracePassSettings (integrators/path_integrator.h:12-19) + maxDepth, with the reference defaults."""
    return abi.PathSettings(int(max_depth), int(enable_subsurface), int(max_reflection_bounces),
                            int(max_refraction_bounces), int(render_ibl_background), float(roulette_aggressiveness))


class Context:
    def __init__(self, device: int = 0, timings: bool = True, hbm_budget: int = 0, wide_bvh: bool = False,
                 lane_per_ray: bool = False, unphased: bool = False, pt_one_kernel: bool = False,
                 split_stack: bool = False, device_build: bool = False, record_lights: bool = False,
                 reference_shadows: bool = False, sah_closest: bool = False, reference_closest: bool = False):
        self._lib = abi.lib()
        self.device = int(device)
        self._h = C.c_void_p()
        flags = ((abi.CTX_TIMINGS if timings else 0) | (abi.CTX_WIDE_BVH if wide_bvh else 0)
                 | (abi.CTX_LANE_PER_RAY if lane_per_ray else 0) | (abi.CTX_UNPHASED if unphased else 0)
                 | (abi.CTX_PT_ONE_KERNEL if pt_one_kernel else 0) | (abi.CTX_SPLIT_STACK if split_stack else 0)
                 | (abi.CTX_DEVICE_BUILD if device_build else 0) | (abi.CTX_RECORD_LIGHTS if record_lights else 0)
                 | (abi.CTX_REFERENCE_SHADOWS if reference_shadows else 0)
                 | (abi.CTX_SAH_CLOSEST if sah_closest else 0)
                 | (abi.CTX_REFERENCE_CLOSEST if reference_closest else 0))
        desc = abi.CtxDesc(int(device), flags, int(hbm_budget))
        abi.check(self._lib.hdr_ctx_create(C.byref(self._h), C.byref(desc)))
        self.width = self.height = 0
        self._cancel = None

    # ------------------------------------------------------------ lifetime
    def close(self) -> None:
        if self._h:
            self._lib.hdr_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ scene
    def upload_scene(self, scene: Scene) -> None:
        desc = scene.c_desc()
        abi.check(self._lib.hdr_scene_upload(self._h, C.byref(desc)))

    def share_scene(self, other: "Context") -> None:
        """Render `other`'s resident scene (no second copy in HBM)."""
        abi.check(self._lib.hdr_scene_share(self._h, other._h))

    def scene_array(self, name: str) -> np.ndarray:
        """A copy of one of the resident scene's device arrays (DeviceScene field name), as bytes."""
        size = C.c_size_t(0)
        abi.check(self._lib.hdr_scene_array(self._h, name.encode(), None, 0, C.byref(size)))
        out = np.empty(size.value, np.uint8)
        abi.check(self._lib.hdr_scene_array(self._h, name.encode(), out.ctypes.data_as(C.c_void_p), out.nbytes, None))
        return out

    def set_instance_transforms(self, transforms) -> None:
        """Move the uploaded scene's instances: `transforms` holds one row-major 4x4
        per instance, in instance order, as a host array (n, 4, 4) / (n, 16) or a
        CUDA tensor of float32 (read after torch's current stream is drained). The
        instance records and the TLAS are rebuilt on the device; the images equal a
        fresh upload of the scene with these transforms."""
        if getattr(transforms, "is_cuda", False):
            import torch

            if transforms.dtype != torch.float32 or not transforms.is_contiguous() or transforms.numel() % 16:
                raise ValueError("transforms: a contiguous float32 tensor of n x 16 values")
            torch.cuda.current_stream(transforms.device).synchronize()
            ptr = C.cast(C.c_void_p(transforms.data_ptr()), C.POINTER(C.c_float))
            abi.check(self._lib.hdr_scene_set_instance_transforms(self._h, ptr, transforms.numel() // 16, 1))
            return
        xf = np.ascontiguousarray(np.asarray(transforms, dtype=np.float32).reshape(-1, 16))
        ptr = xf.ctypes.data_as(C.POINTER(C.c_float))
        abi.check(self._lib.hdr_scene_set_instance_transforms(self._h, ptr, xf.shape[0], 0))

    # ------------------------------------------------------------ passes
    def raycast(self, cam: Camera, frame_index: int = 0, aovs=()) -> None:
        mask = 0
        for a in aovs:
            mask |= {"Depth": abi.AOV_DEPTH, "Albedo": abi.AOV_ALBEDO, "Normal": abi.AOV_NORMAL}[a]
        abi.check(self._lib.hdr_raycast(self._h, C.byref(cam.c_desc()), int(frame_index), mask))
        self.width, self.height = cam.width, cam.height

    def ris_path_trace(self, cam: Camera, frame_index: int, **ris) -> None:
        p = ris_params(**ris)
        abi.check(self._lib.hdr_ris_path_trace(self._h, C.byref(cam.c_desc()), int(frame_index), C.byref(p)))

    def path_trace(self, cam: Camera, frame_index: int, **settings) -> None:
        p = path_settings(**settings)
        abi.check(self._lib.hdr_path_trace(self._h, C.byref(cam.c_desc()), int(frame_index), C.byref(p)))

    def accumulate(self, frame_index: int, firefly: bool = True, mode: str = "parity") -> None:
        m = {"parity": abi.ACCUM_PARITY, "shader": abi.ACCUM_SHADER}[mode]
        abi.check(self._lib.hdr_accumulate(self._h, int(frame_index), int(firefly), m))

    def clear_persistent(self) -> None:
        abi.check(self._lib.hdr_clear_persistent(self._h))

    def synchronize(self) -> None:
        abi.check(self._lib.hdr_synchronize(self._h))

    def set_cancel(self, flag: C.c_int32 | None) -> None:
        self._cancel = flag
        abi.check(self._lib.hdr_set_cancel(self._h, C.byref(flag) if flag is not None else None))

    # ------------------------------------------------------------ buffers
    def buffer_size(self, name: str) -> int:
        n = C.c_size_t()
        abi.check(self._lib.hdr_buffer_size(self._h, name.encode(), C.byref(n)))
        return n.value

    def download(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        nbytes = self.buffer_size(name)
        if name == "GBuffer":
            arr = out if out is not None else np.empty(nbytes // 96, abi.GBUFFER_DTYPE)
        elif name == "__ris_reservoir":
            arr = out if out is not None else np.empty((5, nbytes // 80, 4), np.float32)
        elif name in BUFFER_LAYOUT:
            dt, tail = BUFFER_LAYOUT[name]
            per = int(np.prod(tail)) if tail else 1
            arr = out if out is not None else np.empty((nbytes // (4 * per),) + tail, dt)
        else:
            arr = out if out is not None else np.empty(nbytes, np.uint8)
        if arr.nbytes != nbytes or not arr.flags.c_contiguous:
            raise ValueError(f"{name}: need a contiguous array of {nbytes} bytes")
        abi.check(self._lib.hdr_download(self._h, name.encode(), arr.ctypes.data_as(C.c_void_p), nbytes))
        return arr

    def download_async(self, name: str, out: np.ndarray) -> None:
        """Starts copying `name` into `out` (pinned memory overlaps) while later passes run."""
        if not out.flags.c_contiguous or out.nbytes != self.buffer_size(name):
            raise ValueError(f"{name}: need a contiguous array of {self.buffer_size(name)} bytes")
        abi.check(self._lib.hdr_download_async(self._h, name.encode(), out.ctypes.data_as(C.c_void_p), out.nbytes))

    def download_wait(self) -> None:
        """Waits for the last download_async."""
        abi.check(self._lib.hdr_download_wait(self._h))

    def resolve(self, name: str, src_components: int, component_format: int, dst_components: int,
                device_ptr: int | None = None) -> np.ndarray | None:
        """The named float frame buffer in a render buffer's format (hdr_resolve): a host array,
        or written to `device_ptr` (device memory of this ctx's GPU, ordered on the ctx stream)."""
        pixels = self.buffer_size(name) // (4 * src_components)
        dt = abi.FMT_DTYPES[component_format]
        nbytes = pixels * dst_components * np.dtype(dt).itemsize
        if device_ptr is not None:
            abi.check(self._lib.hdr_resolve(self._h, name.encode(), int(src_components), int(component_format),
                                            int(dst_components), C.c_void_p(device_ptr), nbytes, 1))
            return None
        out = np.empty((pixels, dst_components), dt)
        abi.check(self._lib.hdr_resolve(self._h, name.encode(), int(src_components), int(component_format),
                                        int(dst_components), out.ctypes.data_as(C.c_void_p), nbytes, 0))
        return out

    def upscale(self, name: str, components: int, src_w: int, src_h: int, dst_w: int, dst_h: int) -> None:
        """UpscalePass on the device buffer `name` (hdr_upscale)."""
        abi.check(self._lib.hdr_upscale(self._h, name.encode(), int(components), int(src_w), int(src_h), int(dst_w),
                                        int(dst_h)))

    def denoise(self, name: str, width: int, height: int, chromaticity_blur: bool = True) -> None:
        """Denoiser without OIDN (the chromaticity blur) on the RGBA buffer `name` (hdr_denoise)."""
        abi.check(self._lib.hdr_denoise(self._h, name.encode(), int(width), int(height), int(chromaticity_blur)))

    def upload(self, name: str, arr: np.ndarray) -> None:
        arr = np.ascontiguousarray(arr)
        abi.check(self._lib.hdr_upload(self._h, name.encode(), arr.ctypes.data_as(C.c_void_p), arr.nbytes))

    # ------------------------------------------------------------ queries
    def trace_tuning(self) -> dict:
        t = abi.TraceTuning()
        abi.check(self._lib.hdr_get_trace_tuning(self._h, C.byref(t)))
        return {"node_quorum": t.node_quorum, "blocks_per_sm": t.blocks_per_sm, "shade_shape": t.shade_shape,
                "shadow_shape": t.shadow_shape}

    def set_trace_tuning(self, node_quorum: int, blocks_per_sm: int, shade_shape: int = 0,
                         shadow_shape: int | None = None) -> None:
        if shadow_shape is None:
            shadow_shape = self.trace_tuning()["shadow_shape"]
        t = abi.TraceTuning(int(node_quorum), int(blocks_per_sm), 0.0, int(shade_shape), int(shadow_shape), 0.0)
        abi.check(self._lib.hdr_set_trace_tuning(self._h, C.byref(t)))

    def autotune_trace(self) -> dict:
        """Picks the fastest trace schedule on the last wavefront frame's ray queues."""
        t = abi.TraceTuning()
        abi.check(self._lib.hdr_autotune_trace(self._h, C.byref(t)))
        return {"node_quorum": t.node_quorum, "blocks_per_sm": t.blocks_per_sm, "trace_ms": t.trace_ms,
                "shadow_shape": t.shadow_shape}

    def autotune_frame(self, cam: Camera, frame_index: int, **ris) -> dict:
        """One wavefront RIS frame (the buffers of ris_path_trace) that tunes the trace
        schedule and the resampling kernel's launch shape while it renders."""
        t = abi.TraceTuning()
        abi.check(self._lib.hdr_autotune_frame(self._h, C.byref(cam.c_desc()), int(frame_index),
                                               C.byref(ris_params(**ris)), C.byref(t)))
        return {"node_quorum": t.node_quorum, "blocks_per_sm": t.blocks_per_sm, "trace_ms": t.trace_ms,
                "shadow_shape": t.shadow_shape, "shade_shape": t.shade_shape, "shade_ms": t.shade_ms}

    def trace_stats(self, rays: np.ndarray, walk: int, tmax: np.ndarray | None = None) -> np.ndarray:
        """Per-ray (nodes popped, leaves, triangles tested, answer) of one traversal form
        (0 closest binary, 1 closest wide, 2 shadow binary, 3 shadow wide, 4 shadow BVH)."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.empty((len(rays), 4), np.int32)
        tp = None
        if tmax is not None:
            tmax = np.ascontiguousarray(tmax, np.float32)
            tp = tmax.ctypes.data_as(C.c_void_p)
        abi.check(self._lib.hdr_trace_stats(self._h, rays.ctypes.data_as(C.c_void_p), tp, len(rays), int(walk),
                                            out.ctypes.data_as(C.c_void_p)))
        return out

    def trace_rays(self, rays: np.ndarray, tmax: np.ndarray | None = None, any_hit: bool = False) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.empty(len(rays), abi.GBUFFER_DTYPE)
        tp = None
        if tmax is not None:
            tmax = np.ascontiguousarray(tmax, np.float32)
            tp = tmax.ctypes.data_as(C.c_void_p)
        abi.check(self._lib.hdr_trace_rays(self._h, rays.ctypes.data_as(C.c_void_p), tp, len(rays), int(any_hit),
                                           out.ctypes.data_as(C.c_void_p)))
        return out

    def rng_floats(self, seeds, count: int) -> np.ndarray:
        seeds = np.ascontiguousarray(seeds, np.uint32)
        out = np.empty((len(seeds), count), np.float32)
        abi.check(self._lib.hdr_rng_floats(self._h, seeds.ctypes.data_as(C.c_void_p), len(seeds), int(count),
                                           out.ctypes.data_as(C.c_void_p)))
        return out

    def pass_times(self, reset: bool = False, slots: int = 3) -> tuple[tuple[float, ...], tuple[int, ...]]:
        """(average ms, call count) since the last reset of raycast / integrate /
        accumulate, and with slots=7 also of the wavefront kernels generate /
        trace closest / trace shadow / shade."""
        ms = (C.c_float * slots)()
        n = (C.c_int32 * slots)()
        abi.check(self._lib.hdr_pass_times(self._h, ms, n, slots, int(reset)))
        return tuple(ms), tuple(n)

    def region_begin(self, slot: int = 0) -> None:
        abi.check(self._lib.hdr_region_begin(self._h, int(slot)))

    def region_end(self, slot: int = 0) -> None:
        abi.check(self._lib.hdr_region_end(self._h, int(slot)))

    def region_elapsed(self, slot: int = 0) -> float:
        ms = C.c_float()
        abi.check(self._lib.hdr_region_elapsed(self._h, int(slot), C.byref(ms)))
        return float(ms.value)

    def launch_count(self) -> int:
        n = C.c_uint64()
        abi.check(self._lib.hdr_launch_count(self._h, C.byref(n)))
        return int(n.value)

    # ---- a frame's pass chain as one CUDA graph (hdr_graph_*)
    def graph_begin(self) -> None:
        """Pass calls until graph_end are recorded, not run."""
        abi.check(self._lib.hdr_graph_begin(self._h))

    def graph_end(self) -> None:
        """The record becomes the ctx's executable graph (updated in place when
        it has the launches of the previous one)."""
        abi.check(self._lib.hdr_graph_end(self._h))

    def graph_launch(self, frame_index: int = -1) -> None:
        """Runs the recorded graph for `frame_index` (-1: the recorded frame index)."""
        abi.check(self._lib.hdr_graph_launch(self._h, int(frame_index)))

    def graph_info(self) -> dict:
        k, i, u = C.c_int32(), C.c_int32(), C.c_int32()
        abi.check(self._lib.hdr_graph_info(self._h, C.byref(k), C.byref(i), C.byref(u)))
        return {"kernels": k.value, "instantiations": i.value, "updates": u.value}

    def record_frame(self, passes) -> None:
        """Records the pass calls `passes()` makes on this ctx as its graph and
        runs it: the same work as calling them, submitted as one launch."""
        self.graph_begin()
        try:
            passes()
        except BaseException:
            try:
                self.graph_end()
            except abi.HdrError:
                pass
            raise
        self.graph_end()
        self.graph_launch()
