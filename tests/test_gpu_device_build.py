"""Device BLAS build (HDR_CTX_DEVICE_BUILD): the scene arrays equal the host
builder's byte for byte (tree, node order, triangle order and records, and the
instance records and TLAS built from its counts), and so do the images."""
import numpy as np
import pytest

from hdrestir_b200 import abi, configs
from hdrestir_b200.context import Context
from hdrestir_b200.scene import Camera, Instance, Material, Mesh, Scene  # noqa: F401

pytestmark = pytest.mark.gpu

ARRAYS = ("blas_nodes", "tri_geo", "tri_attr", "instances", "tlas_nodes", "tlas_inst")


def _arrays(scene, device_build):
    with Context(device=0, device_build=device_build) as ctx:
        ctx.upload_scene(scene)
        return {k: ctx.scene_array(k) for k in ARRAYS}


def _no_wide_base(inst):
    """Instance records without their wide-BVH node base (float 30 of 32): the device
    build makes no wide trees, and the binary walk does not read it."""
    rec = inst.view(np.int32).reshape(-1, 32).copy()
    rec[:, 30] = 0
    return rec.view(np.uint8).reshape(-1)


def _same_arrays(scene, nan_payloads=False):
    """Byte-equal arrays. With nan_payloads, a NaN in a float slot of the triangle records
    may differ in its bits: x86 keeps an operand's NaN payload, the GPU returns the
    canonical NaN (the material slot, an integer, stays exact)."""
    host, dev = _arrays(scene, False), _arrays(scene, True)
    host["instances"], dev["instances"] = _no_wide_base(host["instances"]), _no_wide_base(dev["instances"])
    for k in ARRAYS:
        assert host[k].nbytes == dev[k].nbytes, k
        if nan_payloads and k in ("tri_geo", "tri_attr"):
            a, b = host[k].view(np.float32).copy(), dev[k].view(np.float32).copy()
            both = np.isnan(a) & np.isnan(b)
            if k == "tri_attr":
                both.reshape(-1, 36)[:, 31] = False
            a[both] = b[both] = 0.0
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), k
            continue
        assert np.array_equal(host[k], dev[k]), k
    return host


def _one_mesh_scene(mesh):
    sc = Scene()
    sc.meshes.append(mesh)
    sc.instances.append(Instance(0, np.eye(4, dtype=np.float32), -1))
    return sc


@pytest.mark.parametrize("cfg", [0, 1, 2])
def test_config_scenes(cfg):
    kw = {0: {}, 1: dict(n_lights=64), 2: dict(grid=128, n_spheres=60, n_lights=64)}[cfg]
    sc, _ = configs.small_variant(cfg, 32, 32, **kw)
    host = _same_arrays(sc)
    assert host["blas_nodes"].nbytes > 0


def test_full_size_terrain():
    """Config 2's 512 x 512 terrain (522,242 triangles, 25 levels) and its 2000 spheres."""
    sc, _ = configs.config2(64, 64)
    _same_arrays(sc)


def _grid(n, rng, z_noise=0.3):
    xs, zs = np.meshgrid(np.linspace(-1, 1, n, dtype=np.float32), np.linspace(-1, 1, n, dtype=np.float32))
    pts = np.stack([xs, rng.random(xs.shape, np.float32) * z_noise, zs], -1).reshape(-1, 3)
    a = np.arange(n * n, dtype=np.int32).reshape(n, n)
    q = np.stack([a[:-1, :-1], a[1:, :-1], a[:-1, 1:], a[:-1, 1:], a[1:, :-1], a[1:, 1:]], -1).reshape(-1, 3)
    return pts, q


def test_attributes_per_corner_and_per_point():
    rng = np.random.default_rng(1)
    pts, tri = _grid(40, rng)
    t = len(tri)
    per_corner = Mesh(pts, tri, uvs=rng.random((3 * t, 2), np.float32), normals=rng.random((3 * t, 3), np.float32),
                      colors=rng.random((3 * t, 3), np.float32))
    # per-point arrays shorter than the points: the corners past the end take the defaults
    short = Mesh(pts, tri, uvs=rng.random((len(pts) // 2, 2), np.float32),
                 normals=rng.random((len(pts) // 3, 3), np.float32), colors=rng.random((10, 3), np.float32))
    for m in (per_corner, short):
        _same_arrays(_one_mesh_scene(m))


def test_skipped_and_degenerate_triangles():
    rng = np.random.default_rng(2)
    pts, tri = _grid(30, rng)
    bad = tri.copy()
    bad[::7, 1] = len(pts) + 5  # out of range: the triangle is skipped
    bad[::11, 2] = -1
    _same_arrays(_one_mesh_scene(Mesh(pts, bad)))
    same = np.zeros((64, 3), np.float32)  # every centroid equal: each split falls back to halves
    _same_arrays(_one_mesh_scene(Mesh(same, rng.integers(0, 64, (300, 3)).astype(np.int32))))
    tiny = Mesh(pts[:5], np.array([[0, 1, 2], [1, 2, 3], [2, 3, 4]], np.int32))  # one leaf
    _same_arrays(_one_mesh_scene(tiny))


def test_signed_zeros_and_ties():
    """Boxes keep the first vertex of an extreme value: -0 and +0 tie, as do repeated values."""
    rng = np.random.default_rng(3)
    pts = rng.integers(-2, 3, (400, 3)).astype(np.float32) * np.float32(0.5)
    pts[rng.random(pts.shape) < 0.3] = 0.0
    neg = rng.random(pts.shape) < 0.5
    pts[neg & (pts == 0)] = -0.0
    tri = rng.integers(0, len(pts), (900, 3)).astype(np.int32)
    _same_arrays(_one_mesh_scene(Mesh(pts, tri)))


def test_nan_and_huge_vertices():
    rng = np.random.default_rng(4)
    pts = rng.normal(size=(300, 3)).astype(np.float32)
    pts[5] = (np.nan, 0.0, 1.0)
    pts[9] = (3.4e38, -3.4e38, np.inf)
    tri = rng.integers(0, len(pts), (500, 3)).astype(np.int32)
    _same_arrays(_one_mesh_scene(Mesh(pts, tri)), nan_payloads=True)


def test_images_equal():
    sc, cam = configs.small_variant(2, 64, 48, grid=96, n_spheres=60, n_lights=200)
    out = []
    for dev in (False, True):
        with Context(device=0, device_build=dev) as ctx:
            ctx.upload_scene(sc)
            ctx.raycast(cam, 0)
            g = ctx.download("GBuffer").copy()
            ctx.ris_path_trace(cam, 0, candidate_count=16, use_reservoir=True, max_depth=1)
            r = ctx.download("Color").copy()
            ctx.path_trace(cam, 0, max_depth=3)
            p = ctx.download("Color").copy()
            out.append((g, r, p))
    (g0, r0, p0), (g1, r1, p1) = out
    assert np.array_equal(g0.view(np.uint8), g1.view(np.uint8))
    assert np.array_equal(r0.view(np.uint32), r1.view(np.uint32))
    assert np.array_equal(p0.view(np.uint32), p1.view(np.uint32))


def test_moved_instances_on_a_device_built_scene():
    sc, cam = configs.small_variant(2, 48, 32, grid=64, n_spheres=30, n_lights=50)
    xf = np.stack([np.asarray(i.transform, np.float32).reshape(4, 4) for i in sc.instances])
    xf[1:, 3, 0] += 0.25
    with Context(device=0, device_build=True) as a, Context(device=0) as b:
        a.upload_scene(sc)
        b.upload_scene(sc)
        a.set_instance_transforms(xf)
        b.set_instance_transforms(xf)
        assert np.array_equal(_no_wide_base(a.scene_array("instances")), _no_wide_base(b.scene_array("instances")))
        for k in ("tlas_nodes", "tlas_inst"):
            assert np.array_equal(a.scene_array(k), b.scene_array(k)), k


def test_rejected():
    with pytest.raises(abi.HdrError):
        Context(device=0, device_build=True, wide_bvh=True)
    sc, _ = configs.small_variant(0, 16, 16)
    with Context(device=0, device_build=True) as a, Context(device=0, wide_bvh=True) as w:
        a.upload_scene(sc)
        with pytest.raises(abi.HdrError):  # no wide trees to share
            w.share_scene(a)
        with pytest.raises(abi.HdrError):
            a.scene_array("no_such_array")
