"""Host-side scene and camera containers and their C-ABI views.

A ``Scene`` holds what the reference's ``Scene::BuildRenderState`` consumes
(scene/scene.cpp:118-271): mesh subsets, instances with GfMatrix4f
transforms, UsdPreviewSurface parameters and lights. ``Scene.c_desc()``
returns an ``hdr_scene_desc`` that points into the numpy arrays (kept alive
by the Scene object).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi


@dataclass
class Mesh:
    points: np.ndarray                    # (P, 3) f32
    indices: np.ndarray                   # (T, 3) i32
    uvs: np.ndarray | None = None         # (P or 3T, 2) f32
    normals: np.ndarray | None = None     # (P or 3T, 3) f32
    colors: np.ndarray | None = None      # (P or 3T, 3) f32

    def __post_init__(self):
        self.points = np.ascontiguousarray(self.points, np.float32).reshape(-1, 3)
        self.indices = np.ascontiguousarray(self.indices, np.int32).reshape(-1, 3)
        for k in ("uvs", "normals", "colors"):
            v = getattr(self, k)
            if v is not None:
                setattr(self, k, np.ascontiguousarray(v, np.float32).reshape(len(v), -1))


@dataclass
class Material:  # PreviewSurfaceParams defaults (materials/preview_surface_params.h:14-47)
    diffuse_color: tuple = (1.0, 1.0, 1.0)
    metallic: float = 0.0
    roughness: float = 0.5
    specular_color: tuple = (1.0, 1.0, 1.0)
    specular: float = 1.0
    opacity: float = 1.0
    ior: float = 1.5
    transmission: float = 0.0
    transmission_color: tuple = (1.0, 1.0, 1.0)
    transmission_depth: float = 0.0
    emission_color: tuple = (1.0, 1.0, 1.0)
    emission: float = 0.0
    coat: float = 0.0
    coat_color: tuple = (1.0, 1.0, 1.0)
    coat_roughness: float = 0.1
    coat_ior: float = 1.5
    sheen: float = 0.0
    sheen_color: tuple = (1.0, 1.0, 1.0)
    sheen_roughness: float = 0.3
    subsurface: float = 0.0
    subsurface_color: tuple = (1.0, 1.0, 1.0)
    thin_walled: bool = False
    # (H, W, 3) f32 texels as ImageTextureSamplerFactory decodes them, or None
    # (DiffuseTexture / MetallicTexture / RoughnessTexture / NormalTexture, preview_surface_params.h:48-51)
    diffuse_texture: np.ndarray | None = None
    metallic_texture: np.ndarray | None = None
    roughness_texture: np.ndarray | None = None
    normal_texture: np.ndarray | None = None


TEXTURE_FIELDS = ("diffuse_texture", "metallic_texture", "roughness_texture", "normal_texture")


@dataclass
class Light:  # LightFactoryInput / LightParams (sceneInterface/light_params.h:13-28)
    type: int = abi.LIGHT_RECT
    color: tuple = (1.0, 1.0, 1.0)
    intensity: float = 1.0
    exposure: float = 0.0
    transform: np.ndarray = field(default_factory=lambda: np.eye(4))  # GfMatrix4d, row-vector convention
    width: float = 1.0
    height: float = 1.0
    shaping_cone_angle: float = 180.0
    shaping_cone_softness: float = 0.0
    temperature: float = 0.0  # extension: blackbody emission in kelvin (0 = the colour)
    texture: np.ndarray | None = None  # dome: (H, W, 3) f32


@dataclass
class Instance:
    mesh: int
    transform: np.ndarray  # 4x4, row-vector convention (GfMatrix4f)
    material: int = -1
    light: int = -1


@dataclass
class Scene:
    meshes: list = field(default_factory=list)
    instances: list = field(default_factory=list)
    materials: list = field(default_factory=list)
    lights: list = field(default_factory=list)
    name: str = "scene"
    # SceneBuildRenderStateConfig: the physical sky as the environment, its sun at this hour
    # (12 = noon); None = off
    physical_sky_time: float | None = None

    @property
    def num_triangles(self) -> int:
        return int(sum(len(self.meshes[i.mesh].indices) for i in self.instances))

    def c_desc(self) -> abi.SceneDesc:
        keep = []

        def ptr(a, t):
            if a is None or len(a) == 0:
                return C.cast(None, C.POINTER(t)), 0
            a = np.ascontiguousarray(a)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(t)), len(a)

        meshes = (abi.MeshDesc * max(1, len(self.meshes)))()
        for k, m in enumerate(self.meshes):
            d = meshes[k]
            d.points, d.num_points = ptr(m.points.reshape(-1), C.c_float)
            d.num_points //= 3
            d.indices, d.num_triangles = ptr(m.indices.reshape(-1), C.c_int32)
            d.num_triangles //= 3
            for name, cols in (("uvs", 2), ("normals", 3), ("colors", 3)):
                arr = getattr(m, name)
                p, n = ptr(None if arr is None else arr.reshape(-1), C.c_float)
                setattr(d, name, p)
                setattr(d, "num_" + name, n // cols)
            d.material_indices = C.cast(None, C.POINTER(C.c_int32))
            d.num_material_indices = 0
        inst = (abi.InstanceDesc * max(1, len(self.instances)))()
        for k, it in enumerate(self.instances):
            inst[k].mesh, inst[k].material, inst[k].light = it.mesh, it.material, it.light
            inst[k].transform[:] = [float(v) for v in np.asarray(it.transform, np.float32).reshape(-1)]
        mats = (abi.MaterialDesc * max(1, len(self.materials)))()
        for k, m in enumerate(self.materials):
            d = mats[k]
            for f in Material.__dataclass_fields__:
                if f in TEXTURE_FIELDS:
                    continue
                v = getattr(m, f)
                if isinstance(v, tuple):
                    getattr(d, f)[:] = [float(x) for x in v]
                else:
                    setattr(d, f, int(v) if f == "thin_walled" else float(v))
            d.transmission_scatter[:] = [0.0, 0.0, 0.0]
            d.subsurface_radius[:] = [1.0, 1.0, 1.0]
            d.subsurface_scale = 1.0
            d.subsurface_anisotropy = 0.0
            d.diffuse_roughness = 0.0
            for slot, f in enumerate(TEXTURE_FIELDS):
                tex = getattr(m, f)
                if tex is None:
                    continue
                tex = np.ascontiguousarray(tex, np.float32)
                if tex.ndim != 3 or tex.shape[2] != 3:
                    raise ValueError(f"{f}: (H, W, 3) texels expected")
                keep.append(tex)
                d.textures[slot] = tex.ctypes.data_as(C.POINTER(C.c_float))
                d.tex_height[slot], d.tex_width[slot] = tex.shape[0], tex.shape[1]
        lights = (abi.LightDesc * max(1, len(self.lights)))()
        for k, L in enumerate(self.lights):
            d = lights[k]
            d.type = L.type
            d.color[:] = [float(x) for x in L.color]
            d.intensity, d.exposure = float(L.intensity), float(L.exposure)
            d.transform[:] = [float(v) for v in np.asarray(L.transform, np.float64).reshape(-1)]
            d.width, d.height = float(L.width), float(L.height)
            d.shaping_cone_angle, d.shaping_cone_softness = float(L.shaping_cone_angle), float(L.shaping_cone_softness)
            d.temperature = float(L.temperature)
            if L.texture is not None:
                tex = np.ascontiguousarray(L.texture, np.float32)
                keep.append(tex)
                d.texture = tex.ctypes.data_as(C.POINTER(C.c_float))
                d.tex_height, d.tex_width = tex.shape[0], tex.shape[1]
            else:
                d.texture = C.cast(None, C.POINTER(C.c_float))
                d.tex_width = d.tex_height = 0
        desc = abi.SceneDesc(meshes, len(self.meshes), inst, len(self.instances), mats, len(self.materials),
                             lights, len(self.lights), int(self.physical_sky_time is not None),
                             float(self.physical_sky_time if self.physical_sky_time is not None else 12.0))
        desc._keep = (keep, meshes, inst, mats, lights)
        return desc


@dataclass
class Camera:
    view: np.ndarray  # GfMatrix4d world->camera, row-vector convention
    proj: np.ndarray  # GfMatrix4d camera->clip
    width: int
    height: int
    params: dict | None = None  # CameraParams (scene/camera_params.h:8-20) or None = pinhole

    def c_desc(self) -> abi.CameraDesc:
        d = abi.CameraDesc()
        d.view[:] = [float(v) for v in np.asarray(self.view, np.float64).reshape(-1)]
        d.proj[:] = [float(v) for v in np.asarray(self.proj, np.float64).reshape(-1)]
        d.width, d.height = int(self.width), int(self.height)
        p = self.params
        d.has_params = 1 if p is not None else 0
        p = p or {}
        d.enable_dof = int(p.get("enable_dof", 0))
        d.enable_exposure = int(p.get("enable_exposure", 0))
        d.focal_length = float(p.get("focal_length", 50.0))
        d.f_stop = float(p.get("f_stop", 5.6))
        d.focus_distance = float(p.get("focus_distance", 10.0))
        d.bokeh_blades = int(p.get("bokeh_blades", 0))
        d.lens_distortion = float(p.get("lens_distortion", 0.0))
        d.iso = float(p.get("iso", 100.0))
        d.shutter_speed = float(p.get("shutter_speed", 0.02))
        return d


def look_at(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """World->camera matrix (row-vector convention, camera looks down -z)."""
    eye, target, up = (np.asarray(v, np.float64) for v in (eye, target, up))
    back = eye - target
    back /= np.linalg.norm(back)
    right = np.cross(up, back)
    right /= np.linalg.norm(right)
    cup = np.cross(back, right)
    cam_to_world = np.eye(4)
    cam_to_world[0, :3], cam_to_world[1, :3], cam_to_world[2, :3], cam_to_world[3, :3] = right, cup, back, eye
    return np.linalg.inv(cam_to_world)


def perspective(fov_y_deg: float, aspect: float, near: float = 0.1, far: float = 1000.0) -> np.ndarray:
    """GL perspective projection, row-vector convention (the transpose of the column form)."""
    f = 1.0 / np.tan(np.radians(fov_y_deg) / 2.0)
    p = np.zeros((4, 4))
    p[0, 0] = f / aspect
    p[1, 1] = f
    p[2, 2] = (far + near) / (near - far)
    p[3, 2] = 2.0 * far * near / (near - far)
    p[2, 3] = -1.0
    return p


def make_camera(eye, target, width, height, fov=50.0, params=None) -> Camera:
    return Camera(look_at(eye, target), perspective(fov, width / height), width, height, params)


def rect_light_transform(center, facing=(0.0, -1.0, 0.0)) -> np.ndarray:
    """Row-vector transform whose local -z axis (the emitting side) points along `facing`."""
    fz = -np.asarray(facing, np.float64)
    fz /= np.linalg.norm(fz)
    helper = np.array([1.0, 0.0, 0.0]) if abs(fz[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    fx = np.cross(helper, fz)
    fx /= np.linalg.norm(fx)
    fy = np.cross(fz, fx)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3], m[3, :3] = fx, fy, fz, center
    return m
