"""ctypes binding of the C ABI declared in ``include/hdrestir.h``.

The library is the in-tree ``libhdrestir_b200.so``; there is no other
implementation to fall back to, so a missing library or a missing GPU fails
loudly here.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libhdrestir_b200.so"

HDR_OK, HDR_EINVAL, HDR_ENOMEM, HDR_ECANCELLED, HDR_ETIMEOUT, HDR_ECUDA, HDR_ENOSCENE, HDR_EDEVICE = range(8)
STATUS_NAMES = {0: "HDR_OK", 1: "HDR_EINVAL", 2: "HDR_ENOMEM", 3: "HDR_ECANCELLED", 4: "HDR_ETIMEOUT",
                5: "HDR_ECUDA", 6: "HDR_ENOSCENE", 7: "HDR_EDEVICE"}
LIGHT_DISTANT, LIGHT_DOME, LIGHT_RECT, LIGHT_POINT = 0, 1, 2, 3
LIGHT_TRIANGLE = 4  # extension: an emissive triangle (half of the rect of the same size)
AOV_DEPTH, AOV_ALBEDO, AOV_NORMAL = 1, 2, 4
ACCUM_PARITY, ACCUM_SHADER = 0, 1
CTX_TIMINGS, CTX_WIDE_BVH, CTX_LANE_PER_RAY, CTX_UNPHASED, CTX_PT_ONE_KERNEL = 1, 2, 8, 16, 32
CTX_SPLIT_STACK = 64
CTX_DEVICE_BUILD = 128
CTX_RECORD_LIGHTS = 256
CTX_REFERENCE_SHADOWS = 512
CTX_SAH_CLOSEST = 1024
CTX_REFERENCE_CLOSEST = 2048
RIS_REPROJECT = 4
FMT_FLOAT32, FMT_FLOAT16, FMT_UNORM8, FMT_SNORM8, FMT_INT32 = 0, 1, 2, 3, 4
FMT_DTYPES = {0: np.float32, 1: np.uint16, 2: np.uint8, 3: np.int8, 4: np.int32}

_f = C.c_float
_i = C.c_int32
_pf = C.POINTER(C.c_float)
_pi = C.POINTER(C.c_int32)


class MeshDesc(C.Structure):
    _fields_ = [("points", _pf), ("num_points", _i), ("indices", _pi), ("num_triangles", _i),
                ("uvs", _pf), ("num_uvs", _i), ("normals", _pf), ("num_normals", _i),
                ("colors", _pf), ("num_colors", _i), ("material_indices", _pi), ("num_material_indices", _i)]


class InstanceDesc(C.Structure):
    _fields_ = [("mesh", _i), ("material", _i), ("light", _i), ("reserved", _i), ("transform", _f * 16)]


class MaterialDesc(C.Structure):
    _fields_ = [("diffuse_color", _f * 3), ("metallic", _f), ("roughness", _f), ("specular_color", _f * 3),
                ("specular", _f), ("opacity", _f), ("ior", _f), ("transmission", _f),
                ("transmission_color", _f * 3), ("transmission_depth", _f), ("transmission_scatter", _f * 3),
                ("emission_color", _f * 3), ("emission", _f), ("coat", _f), ("coat_color", _f * 3),
                ("coat_roughness", _f), ("coat_ior", _f), ("sheen", _f), ("sheen_color", _f * 3),
                ("sheen_roughness", _f), ("subsurface", _f), ("subsurface_color", _f * 3),
                ("subsurface_radius", _f * 3), ("subsurface_scale", _f), ("subsurface_anisotropy", _f),
                ("thin_walled", _i), ("diffuse_roughness", _f), ("textures", _pf * 4), ("tex_width", _i * 4),
                ("tex_height", _i * 4)]


class LightDesc(C.Structure):
    _fields_ = [("type", _i), ("color", _f * 3), ("intensity", _f), ("exposure", _f),
                ("transform", C.c_double * 16), ("width", _f), ("height", _f), ("shaping_cone_angle", _f),
                ("shaping_cone_softness", _f), ("texture", _pf), ("tex_width", _i), ("tex_height", _i),
                ("temperature", _f)]


class SceneDesc(C.Structure):
    _fields_ = [("meshes", C.POINTER(MeshDesc)), ("num_meshes", _i),
                ("instances", C.POINTER(InstanceDesc)), ("num_instances", _i),
                ("materials", C.POINTER(MaterialDesc)), ("num_materials", _i),
                ("lights", C.POINTER(LightDesc)), ("num_lights", _i),
                ("enable_physical_sky", _i), ("physical_sky_time", _f)]


class CameraDesc(C.Structure):
    _fields_ = [("view", C.c_double * 16), ("proj", C.c_double * 16), ("width", _i), ("height", _i),
                ("has_params", _i), ("enable_dof", _i), ("enable_exposure", _i), ("focal_length", _f),
                ("f_stop", _f), ("focus_distance", _f), ("bokeh_blades", _i), ("lens_distortion", _f),
                ("iso", _f), ("shutter_speed", _f)]


class PathSettings(C.Structure):
    _fields_ = [("max_depth", _i), ("enable_subsurface", _i), ("max_reflection_bounces", _i),
                ("max_refraction_bounces", _i), ("render_ibl_background", _i), ("roulette_aggressiveness", _f)]


class RisParams(C.Structure):
    _fields_ = [("path", PathSettings), ("candidate_count", _i), ("use_reservoir", _i), ("skip_visibility", _i),
                ("m_cap", _i), ("spatial_neighbors", _i), ("spatial_radius", _f), ("flags", C.c_uint32),
                ("reserved", _i)]


RIS_TRACE_ALL_RAYS, RIS_ONE_KERNEL = 1, 2


class TraceTuning(C.Structure):
    _fields_ = [("node_quorum", _i), ("blocks_per_sm", _i), ("trace_ms", _f), ("shade_shape", _i),
                ("shadow_shape", _i), ("shade_ms", _f)]


class ServerDesc(C.Structure):
    _fields_ = [("device", _i), ("flags", C.c_uint32), ("hbm_budget_bytes", C.c_size_t), ("max_batch", _i),
                ("step_pixels", C.c_int64), ("age_weight", C.c_float)]


class JobDesc(C.Structure):
    _fields_ = [("scene", _i), ("pipeline", _i), ("frames", _i), ("firefly", _i), ("camera", CameraDesc),
                ("ris", RisParams)]


SERVER_SERIAL = 1
JOB_PATH_TRACER, JOB_RIS = 0, 1
JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3


MTL_FLOAT, MTL_FLOAT3, MTL_BOOL, MTL_ASSET = 0, 1, 2, 3


class MtlParam(C.Structure):
    _fields_ = [("name", C.c_char_p), ("type", _i), ("value", _f * 3), ("asset", C.c_char_p)]


class MtlConnection(C.Structure):
    _fields_ = [("input", C.c_char_p), ("upstream_node", C.c_char_p)]


class MtlNode(C.Structure):
    _fields_ = [("path", C.c_char_p), ("shader_id", C.c_char_p), ("params", C.POINTER(MtlParam)),
                ("num_params", _i), ("inputs", C.POINTER(MtlConnection)), ("num_inputs", _i)]


class MtlTerminal(C.Structure):
    _fields_ = [("name", C.c_char_p), ("upstream_node", C.c_char_p)]


class MtlNetwork(C.Structure):
    _fields_ = [("nodes", C.POINTER(MtlNode)), ("num_nodes", _i), ("terminals", C.POINTER(MtlTerminal)),
                ("num_terminals", _i)]


class MtlTextures(C.Structure):
    _fields_ = [("path", (C.c_char * 1024) * 4)]


class CtxDesc(C.Structure):
    _fields_ = [("device", _i), ("flags", C.c_uint32), ("hbm_budget_bytes", C.c_size_t)]


GBUFFER_DTYPE = np.dtype([("position", "<f4", 3), ("depth", "<f4"), ("normal", "<f4", 3), ("prim_id", "<i4"),
                          ("smooth_normal", "<f4", 3), ("tri_id", "<i4"), ("albedo", "<f4", 3), ("hit", "<i4"),
                          ("uv", "<f4", 2), ("dpdu", "<f4", 3), ("dpdv", "<f4", 3)])
assert GBUFFER_DTYPE.itemsize == 96

# "__ris_reservoir": five float4 planes per pixel
RESERVOIR_PLANES = ("dir_dist", "color_pdf", "normal_phat", "throughput", "wsum_w_m_meta")
RES_HAS_SAMPLE, RES_HAS_CANDIDATE, RES_VIS_TESTED, RES_PDF_SOLID = 1, 2, 4, 8


class HdrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib() -> C.CDLL:
    """Loads the in-tree library (built by hdrestir_b200.build)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m hdrestir_b200.build` (needs nvcc)")
        L = C.CDLL(str(LIB_PATH))
        vp, i32, sz = C.c_void_p, C.c_int32, C.c_size_t
        sig = {
            "hdr_abi_version": (C.c_int, []),
            "hdr_last_error": (C.c_char_p, []),
            "hdr_ctx_create": (C.c_int, [C.POINTER(vp), C.POINTER(CtxDesc)]),
            "hdr_ctx_destroy": (None, [vp]),
            "hdr_scene_upload": (C.c_int, [vp, C.POINTER(SceneDesc)]),
            "hdr_scene_share": (C.c_int, [vp, vp]),
            "hdr_scene_set_instance_transforms": (C.c_int, [vp, C.POINTER(C.c_float), i32, i32]),
            "hdr_scene_array": (C.c_int, [vp, C.c_char_p, vp, C.c_size_t, C.POINTER(C.c_size_t)]),
            "hdr_path_trace_batch": (C.c_int, [C.POINTER(vp), i32, C.POINTER(CameraDesc), C.POINTER(i32),
                                               C.POINTER(PathSettings)]),
            "hdr_ris_path_trace_batch": (C.c_int, [C.POINTER(vp), i32, C.POINTER(CameraDesc), C.POINTER(i32),
                                                   C.POINTER(RisParams)]),
            "hdr_raycast": (C.c_int, [vp, C.POINTER(CameraDesc), i32, C.c_uint32]),
            "hdr_ris_path_trace": (C.c_int, [vp, C.POINTER(CameraDesc), i32, C.POINTER(RisParams)]),
            "hdr_path_trace": (C.c_int, [vp, C.POINTER(CameraDesc), i32, C.POINTER(PathSettings)]),
            "hdr_accumulate": (C.c_int, [vp, i32, i32, i32]),
            "hdr_accumulate_noalloc": (C.c_int, [vp, vp, i32, i32, i32, i32, i32, vp]),
            "hdr_clear_persistent": (C.c_int, [vp]),
            "hdr_zero_persistent": (C.c_int, [vp]),
            "hdr_download": (C.c_int, [vp, C.c_char_p, vp, sz]),
            "hdr_resolve": (C.c_int, [vp, C.c_char_p, i32, i32, i32, vp, sz, i32]),
            "hdr_download_async": (C.c_int, [vp, C.c_char_p, vp, sz]),
            "hdr_download_wait": (C.c_int, [vp]),
            "hdr_upscale": (C.c_int, [vp, C.c_char_p, i32, i32, i32, i32, i32]),
            "hdr_denoise": (C.c_int, [vp, C.c_char_p, i32, i32, i32]),
            "hdr_upload": (C.c_int, [vp, C.c_char_p, vp, sz]),
            "hdr_buffer_size": (C.c_int, [vp, C.c_char_p, C.POINTER(sz)]),
            "hdr_synchronize": (C.c_int, [vp]),
            "hdr_set_cancel": (C.c_int, [vp, C.POINTER(C.c_int32)]),
            "hdr_trace_rays": (C.c_int, [vp, vp, vp, i32, i32, vp]),
            "hdr_trace_stats": (C.c_int, [vp, vp, vp, i32, i32, vp]),
            "hdr_get_trace_tuning": (C.c_int, [vp, C.POINTER(TraceTuning)]),
            "hdr_set_trace_tuning": (C.c_int, [vp, C.POINTER(TraceTuning)]),
            "hdr_autotune_trace": (C.c_int, [vp, C.POINTER(TraceTuning)]),
            "hdr_autotune_frame": (C.c_int, [vp, C.POINTER(CameraDesc), i32, C.POINTER(RisParams),
                                             C.POINTER(TraceTuning)]),
            "hdr_rng_floats": (C.c_int, [vp, vp, i32, i32, vp]),
            "hdr_pass_times": (C.c_int, [vp, C.POINTER(C.c_float), C.POINTER(C.c_int32), i32, i32]),
            "hdr_launch_count": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
            "hdr_region_begin": (C.c_int, [vp, i32]),
            "hdr_region_end": (C.c_int, [vp, i32]),
            "hdr_region_elapsed": (C.c_int, [vp, i32, C.POINTER(C.c_float)]),
            "hdr_trim_frame_memory": (C.c_int, [i32, sz]),
            "hdr_graph_begin": (C.c_int, [vp]),
            "hdr_graph_end": (C.c_int, [vp]),
            "hdr_graph_launch": (C.c_int, [vp, i32]),
            "hdr_graph_info": (C.c_int, [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]),
            "hdr_server_create": (C.c_int, [C.POINTER(vp), C.POINTER(ServerDesc)]),
            "hdr_server_destroy": (None, [vp]),
            "hdr_server_add_scene": (C.c_int, [vp, C.POINTER(SceneDesc), C.POINTER(i32)]),
            "hdr_server_submit": (C.c_int, [vp, C.POINTER(JobDesc), C.POINTER(C.c_int64)]),
            "hdr_server_step": (C.c_int, [vp, C.POINTER(i32)]),
            "hdr_server_job_state": (C.c_int, [vp, C.c_int64, C.POINTER(i32), C.POINTER(i32)]),
            "hdr_server_take_result": (C.c_int, [vp, C.c_int64, vp, sz]),
            "hdr_server_load": (C.c_int, [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(sz)]),
            "hdr_server_drain_finished": (C.c_int, [vp, C.POINTER(C.c_int64), i32, C.POINTER(i32)]),
            "hdr_material_from_network": (C.c_int, [C.POINTER(MtlNetwork), C.POINTER(MaterialDesc),
                                                    C.POINTER(MtlTextures)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != HDR_OK:
        raise HdrError(status, lib().hdr_last_error().decode(errors="replace"))


def exported_symbols() -> list[str]:
    """Names declared in include/hdrestir.h (used by the export test)."""
    import re
    hdr = (Path(__file__).resolve().parent.parent / "include" / "hdrestir.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:hdr_status|void|int|const char \*)\s*\*?\s*(hdr_\w+)\s*\(", hdr, re.M)))
