"""Seeded synthetic scenes standing in for the benchmark configurations.

No scene files are shipped with the benchmark; these generators build scenes
with the stated shapes, sizes and value distributions from fixed seeds:

* ``config0``: closed box of 12 quads (24 triangles) in [-1,1]^3, 2 rect lights
  0.3x0.3 with radiance U[10,20], PreviewSurface diffuse U[0.2,0.8],
  roughness 0.5, metallic 0 (seed 0xC0FFEE00); 256x256 PathTracer, depth 4.
* ``config1``: ground plane + 64 axis-aligned boxes (770 triangles), 1024 rect
  lights of side U[0.02,0.1] in a 10x10x2 slab, blackbody colour T~U[2000,9000]K
  normalised to luminance 1 times intensity log-uniform over [1,100], GGX
  roughness U[0.05,1], metallic Bernoulli(0.3) (seed 0xC0FFEE01); 512x512 RIS,
  16 candidates, no reservoir, skipVisibility, direct light only.
* ``config2``: 512x512-vertex grid displaced by seeded value noise (522,242
  triangles) + 2000 instances of a 256-triangle sphere with radius
  log-uniform [0.05,0.5]; 10,000 rect lights (equal-area stand-ins for the
  emissive triangles, which the reference's light model does not have)
  (seed 0xC0FFEE02); 1920x1080 ReSTIR, 32 candidates, temporal reuse.

Emission is RGB uplifted by the reference's RGBToSpectrum, so blackbody spectra
enter as their CIE-1931 RGB (the reference has no spectral emission).
"""
from __future__ import annotations

import numpy as np

from . import abi
from .scene import Camera, Instance, Light, Material, Mesh, Scene, make_camera, rect_light_transform

SEEDS = {0: 0xC0FFEE00, 1: 0xC0FFEE01, 2: 0xC0FFEE02, 3: 0xC0FFEE03}


# ---------------------------------------------------------------- geometry
def quad(p0, p1, p2, p3) -> tuple[np.ndarray, np.ndarray]:
    pts = np.array([p0, p1, p2, p3], np.float32)
    return pts, np.array([[0, 1, 2], [0, 2, 3]], np.int32)


def box_mesh(lo, hi, inward=False) -> Mesh:
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    faces = [
        [(x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0)],  # -x
        [(x1, y0, z0), (x1, y1, z0), (x1, y1, z1), (x1, y0, z1)],  # +x
        [(x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1)],  # -y
        [(x0, y1, z0), (x0, y1, z1), (x1, y1, z1), (x1, y1, z0)],  # +y
        [(x0, y0, z0), (x0, y1, z0), (x1, y1, z0), (x1, y0, z0)],  # -z
        [(x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)],  # +z
    ]
    pts, idx = [], []
    for f in faces:
        if inward:
            f = f[::-1]
        base = len(pts)
        pts += f
        idx += [[base, base + 1, base + 2], [base, base + 2, base + 3]]
    return Mesh(np.array(pts, np.float32), np.array(idx, np.int32))


def sphere_mesh(n_lon=16, n_lat=9) -> Mesh:
    """Unit UV sphere with 2*n_lon*(n_lat-1) triangles (256 for 16 x 9)."""
    pts = [(0.0, 1.0, 0.0)]
    for i in range(1, n_lat):
        th = np.pi * i / n_lat
        for j in range(n_lon):
            ph = 2 * np.pi * j / n_lon
            pts.append((np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)))
    pts.append((0.0, -1.0, 0.0))
    bottom = len(pts) - 1
    idx = []
    for j in range(n_lon):
        idx.append([0, 1 + (j + 1) % n_lon, 1 + j])
    for i in range(n_lat - 2):
        r0, r1 = 1 + i * n_lon, 1 + (i + 1) * n_lon
        for j in range(n_lon):
            a, b = r0 + j, r0 + (j + 1) % n_lon
            c, d = r1 + j, r1 + (j + 1) % n_lon
            idx += [[a, b, d], [a, d, c]]
    r0 = 1 + (n_lat - 2) * n_lon
    for j in range(n_lon):
        idx.append([bottom, r0 + j, r0 + (j + 1) % n_lon])
    p = np.array(pts, np.float32)
    return Mesh(p, np.array(idx, np.int32), normals=p.copy())


def value_noise(n: int, rng: np.random.Generator, octaves=4, base=8) -> np.ndarray:
    """Seeded value noise on an n x n grid in [0, 1] (smoothstep-interpolated lattices)."""
    out = np.zeros((n, n))
    amp, total = 1.0, 0.0
    u = np.linspace(0.0, 1.0, n)
    for o in range(octaves):
        cells = base * (2 ** o)
        lat = rng.random((cells + 1, cells + 1))
        x = u * cells
        i0 = np.minimum(x.astype(int), cells - 1)
        t = x - i0
        t = t * t * (3 - 2 * t)
        a = lat[np.ix_(i0, i0)]
        b = lat[np.ix_(i0, i0 + 1)]
        c = lat[np.ix_(i0 + 1, i0)]
        d = lat[np.ix_(i0 + 1, i0 + 1)]
        ty, tx = t[:, None], t[None, :]
        out += amp * ((a * (1 - tx) + b * tx) * (1 - ty) + (c * (1 - tx) + d * tx) * ty)
        total += amp
        amp *= 0.5
    return out / total


def grid_mesh(n: int, extent: float, height: np.ndarray) -> Mesh:
    xs = np.linspace(-extent, extent, n, dtype=np.float64)
    X, Z = np.meshgrid(xs, xs)
    pts = np.stack([X, height, Z], -1).reshape(-1, 3).astype(np.float32)
    i = np.arange(n - 1)
    a = (i[:, None] * n + i[None, :]).reshape(-1)
    b, c, d = a + 1, a + n, a + n + 1
    idx = np.concatenate([np.stack([a, c, b], 1), np.stack([b, c, d], 1)]).astype(np.int32)
    return Mesh(pts, idx)


# ---------------------------------------------------------------- colour
def _cie_fit(w):
    """Wyman 2013 multi-lobe fit of the CIE 1931 observer (public formula)."""
    def g(x, mu, s1, s2):
        s = np.where(x < mu, s1, s2)
        return np.exp(-0.5 * ((x - mu) / s) ** 2)
    X = 1.056 * g(w, 599.8, 37.9, 31.0) + 0.362 * g(w, 442.0, 16.0, 26.7) - 0.065 * g(w, 501.1, 20.4, 26.2)
    Y = 0.821 * g(w, 568.8, 46.9, 40.5) + 0.286 * g(w, 530.9, 16.3, 31.1)
    Z = 1.217 * g(w, 437.0, 11.8, 36.0) + 0.681 * g(w, 459.0, 26.0, 13.8)
    return X, Y, Z


def blackbody_rgb(T: np.ndarray) -> np.ndarray:
    """Linear sRGB of a Planckian radiator at T kelvin, normalised to luminance 1."""
    w = np.linspace(360.0, 830.0, 471)
    lam = w * 1e-9
    h, c, k = 6.62607015e-34, 2.99792458e8, 1.380649e-23
    T = np.asarray(T, np.float64)[:, None]
    spd = 1.0 / (lam ** 5 * (np.exp(h * c / (lam * k * T)) - 1.0))
    X, Y, Z = [(spd * f).sum(1) for f in _cie_fit(w)]
    M = np.array([[3.2404542, -1.5371385, -0.4985314], [-0.9692660, 1.8760108, 0.0415560],
                  [0.0556434, -0.2040259, 1.0572252]])
    rgb = np.stack([X, Y, Z], 1) @ M.T
    rgb = np.maximum(rgb, 0.0)
    lum = rgb @ np.array([0.2126, 0.7152, 0.0722])
    return rgb / lum[:, None]


def _scale_translate(s, t) -> np.ndarray:
    m = np.eye(4)
    m[0, 0] = m[1, 1] = m[2, 2] = s
    m[3, :3] = t
    return m


# ---------------------------------------------------------------- configs
def config0(width=256, height=256):
    rng = np.random.default_rng(SEEDS[0])
    sc = Scene(name="config0_box")
    # closed box: 6 walls facing inward
    walls = box_mesh((-1, -1, -1), (1, 1, 1), inward=True)
    # 6 interior quads: a floating 3-sided step and three panels
    quads = [quad((-0.7, -1.0 + 0.4, -0.5), (-0.1, -0.6, -0.5), (-0.1, -0.6, 0.1), (-0.7, -0.6, 0.1)),
             quad((0.2, -1.0, 0.3), (0.8, -1.0, 0.3), (0.8, -0.2, 0.3), (0.2, -0.2, 0.3)),
             quad((0.2, -1.0, -0.3), (0.2, -0.2, -0.3), (0.8, -0.2, -0.3), (0.8, -1.0, -0.3)),
             quad((0.2, -0.2, -0.3), (0.2, -0.2, 0.3), (0.8, -0.2, 0.3), (0.8, -0.2, -0.3)),
             quad((-0.9, -0.3, 0.6), (-0.4, -0.3, 0.6), (-0.4, 0.5, 0.9), (-0.9, 0.5, 0.9)),
             quad((0.3, 0.2, -0.9), (0.9, 0.2, -0.9), (0.9, 0.7, -0.6), (0.3, 0.7, -0.6))]
    for k in range(6):
        m = Mesh(walls.points[4 * k:4 * k + 4], np.array([[0, 1, 2], [0, 2, 3]], np.int32))
        sc.meshes.append(m)
    for pts, idx in quads:
        sc.meshes.append(Mesh(pts, idx))
    for k in range(12):
        col = tuple(float(v) for v in rng.uniform(0.2, 0.8, 3))
        sc.materials.append(Material(diffuse_color=col, roughness=0.5, metallic=0.0))
        sc.instances.append(Instance(mesh=k, transform=np.eye(4), material=k))
    for c in ((-0.4, 0.95, 0.0), (0.45, 0.95, 0.35)):
        radiance = float(rng.uniform(10.0, 20.0))
        sc.lights.append(Light(abi.LIGHT_RECT, color=(radiance,) * 3, intensity=1.0,
                               transform=rect_light_transform(c, (0, -1, 0)), width=0.3, height=0.3))
    cam = make_camera((0.0, 0.0, 0.95), (0.0, -0.2, 0.0), width, height, fov=70.0)
    return sc, cam


def _box_tris(cx, cz, sx, sy, sz):
    return box_mesh((cx - sx, 0.0, cz - sz), (cx + sx, 2 * sy, cz + sz))


def _random_material(rng) -> Material:
    return Material(diffuse_color=tuple(float(v) for v in rng.uniform(0.2, 0.8, 3)),
                    roughness=float(rng.uniform(0.05, 1.0)), metallic=float(rng.random() < 0.3))


def config1(width=512, height=512, n_lights=1024):
    rng = np.random.default_rng(SEEDS[1])
    sc = Scene(name="config1_boxes")
    pts, idx = quad((-5, 0, -5), (-5, 0, 5), (5, 0, 5), (5, 0, -5))
    sc.meshes.append(Mesh(pts, idx))
    sc.materials.append(Material(diffuse_color=(0.5, 0.5, 0.5), roughness=0.7))
    sc.instances.append(Instance(0, np.eye(4), 0))
    for k in range(64):
        cx, cz = rng.uniform(-4.5, 4.5, 2)
        sx, sy, sz = rng.uniform(0.1, 0.45, 3)
        sc.meshes.append(_box_tris(cx, cz, sx, sy, sz))
        sc.materials.append(_random_material(rng))
        sc.instances.append(Instance(k + 1, np.eye(4), k + 1))
    T = rng.uniform(2000.0, 9000.0, n_lights)
    rgb = blackbody_rgb(T)
    inten = 10.0 ** rng.uniform(0.0, 2.0, n_lights)
    side = rng.uniform(0.02, 0.1, n_lights)
    pos = np.stack([rng.uniform(-5, 5, n_lights), rng.uniform(2.0, 4.0, n_lights), rng.uniform(-5, 5, n_lights)], 1)
    for k in range(n_lights):
        sc.lights.append(Light(abi.LIGHT_RECT, color=tuple(float(v) for v in rgb[k]), intensity=float(inten[k]),
                               transform=rect_light_transform(pos[k], (0, -1, 0)), width=float(side[k]),
                               height=float(side[k])))
    cam = make_camera((0.0, 6.0, 9.0), (0.0, 0.0, 0.0), width, height, fov=55.0)
    return sc, cam


def config2(width=1920, height=1080, grid=512, n_spheres=2000, n_lights=10000, orbit_angle=None):
    rng = np.random.default_rng(SEEDS[2])
    sc = Scene(name="config2_terrain")
    extent = 20.0
    h = value_noise(grid, rng) * 3.0
    sc.meshes.append(grid_mesh(grid, extent, h))
    sc.materials.append(Material(diffuse_color=(0.45, 0.42, 0.38), roughness=0.85))
    sc.instances.append(Instance(0, np.eye(4), 0))
    sc.meshes.append(sphere_mesh())
    radius = np.exp(rng.uniform(np.log(0.05), np.log(0.5), n_spheres))
    xz = rng.uniform(-extent * 0.9, extent * 0.9, (n_spheres, 2))
    cell = 2 * extent / (grid - 1)
    gi = np.clip(np.round((xz + extent) / cell).astype(int), 0, grid - 1)
    ground = h[gi[:, 1], gi[:, 0]]
    for k in range(n_spheres):
        sc.materials.append(_random_material(rng))
        t = (float(xz[k, 0]), float(ground[k] + radius[k] * 1.2), float(xz[k, 1]))
        sc.instances.append(Instance(1, _scale_translate(float(radius[k]), t), k + 1))
    T = rng.uniform(2000.0, 9000.0, n_lights)
    rgb = blackbody_rgb(T)
    inten = 10.0 ** rng.uniform(0.0, 2.0, n_lights)
    side = rng.uniform(0.1, 0.3, n_lights)
    pos = np.stack([rng.uniform(-extent, extent, n_lights), rng.uniform(5.0, 7.0, n_lights),
                    rng.uniform(-extent, extent, n_lights)], 1)
    for k in range(n_lights):
        sc.lights.append(Light(abi.LIGHT_RECT, color=tuple(float(v) for v in rgb[k]), intensity=float(inten[k]),
                               transform=rect_light_transform(pos[k], (0, -1, 0)), width=float(side[k]),
                               height=float(side[k])))
    cam = orbit_camera(0.0 if orbit_angle is None else orbit_angle, width, height)
    return sc, cam


def mixed_lights(width=64, height=48, seed=0xC0FFEE05):
    """The config-1 boxes lit by every analytic light type: rect lights, point lights (some
    shaped by a cone with soft edges) and distant lights. Test scene for the light models."""
    sc, cam = config1(width, height, n_lights=12)
    rng = np.random.default_rng(seed)
    for k in range(10):
        pos = (float(rng.uniform(-4, 4)), float(rng.uniform(1.0, 3.5)), float(rng.uniform(-4, 4)))
        cone = 180.0 if k % 2 == 0 else float(rng.uniform(30.0, 80.0))
        sc.lights.append(Light(abi.LIGHT_POINT, color=tuple(float(v) for v in rng.uniform(0.3, 1.0, 3)),
                               intensity=float(rng.uniform(2.0, 20.0)), transform=rect_light_transform(pos, (0, -1, 0)),
                               shaping_cone_angle=cone, shaping_cone_softness=0.0 if k % 4 == 1 else 0.3))
    for k in range(3):
        d = rng.normal(size=3)
        d[1] = -abs(d[1]) - 0.5
        sc.lights.append(Light(abi.LIGHT_DISTANT, color=(1.0, 0.95, 0.9), intensity=float(rng.uniform(0.5, 2.0)),
                               transform=rect_light_transform((0.0, 0.0, 0.0), tuple(d / np.linalg.norm(d)))))
    return sc, cam


def translucent_variant(width=64, height=48):
    """The config-2 family with see-through and absorbing spheres: partial opacity (stochastic
    pass-through), transmission with Beer absorption (transmission depth), thin-walled
    transmission. Test scene for the non-opaque paths."""
    import dataclasses
    sc, cam = config2(width, height, grid=64, n_spheres=80, n_lights=200)
    kinds = [dict(opacity=0.5), dict(opacity=0.2, roughness=0.3),
             dict(transmission=0.9, ior=1.4, transmission_depth=0.5, transmission_color=(0.9, 0.4, 0.2),
                  roughness=0.1),
             dict(transmission=0.8, ior=1.5, thin_walled=True, roughness=0.0)]
    for k, inst in enumerate(sc.instances[1:]):
        sc.materials[inst.material] = dataclasses.replace(sc.materials[inst.material], **kinds[k % len(kinds)])
    return sc, cam


def sky_variant(cfg: int, width: int, height: int, hour: float = 15.5, **kw):
    """A config-1 or config-2 scene under the physical sky (SceneBuildRenderStateConfig::
    EnablePhysicalSky, its sun at `hour`): no configuration of the benchmark uses the sky,
    so this family exercises the environment outside the light sampler (the RIS pass's sky
    technique, the path tracer's separate sun sample, sky radiance on misses)."""
    sc, cam = small_variant(cfg, width, height, **kw)
    sc.physical_sky_time = float(hour)
    if cfg == 2:  # a camera that sees the horizon, so misses show the sky
        cam = make_camera((22.0 * np.sin(0.4), 3.0, 22.0 * np.cos(0.4)), (0.0, 3.0, 0.0), width, height, fov=70.0)
    return sc, cam


def textured_variant(width=64, height=48, seed=7):
    """The config-2 family with UVs and PreviewSurface textures (diffuse, metallic, roughness,
    tangent-space normal map; preview_surface.cpp:68-95): the terrain's UVs wrap several
    times, each sphere material takes one or all four textures. Seeded texels of odd sizes
    stand in for decoded image files."""
    import dataclasses
    rng = np.random.default_rng(seed)
    sc, cam = config2(width, height, grid=64, n_spheres=80, n_lights=200)
    ground, sphere = sc.meshes[0], sc.meshes[1]
    gp = ground.points
    ext = float(np.abs(gp[:, 0]).max())
    g_uv = np.stack([gp[:, 0] / ext * 1.7 + 0.3, gp[:, 2] / ext * 2.3 - 0.1], -1).astype(np.float32)
    sp = sphere.points
    s_uv = np.stack([np.arctan2(sp[:, 2], sp[:, 0]) / (2 * np.pi) + 0.5,
                     np.arccos(np.clip(sp[:, 1], -1, 1)) / np.pi], -1).astype(np.float32)
    sc.meshes[0] = dataclasses.replace(ground, uvs=g_uv)
    sc.meshes[1] = dataclasses.replace(sphere, uvs=s_uv)

    def tex(h, w, lo=0.0, hi=1.0):
        base = rng.uniform(lo, hi, (h, w, 3)).astype(np.float32)
        return (0.5 * base + 0.5 * np.roll(base, 1, axis=1)).astype(np.float32)

    def normal_map(h, w):
        t = rng.normal(0.0, 0.25, (h, w, 2))
        return np.concatenate([0.5 + 0.5 * t, np.ones((h, w, 1))], -1).astype(np.float32)

    kinds = [dict(diffuse_texture=tex(37, 23)),
             dict(metallic_texture=tex(16, 16), roughness_texture=tex(9, 31, 0.05, 1.0)),
             dict(normal_texture=normal_map(24, 24), roughness=0.2),
             dict(diffuse_texture=tex(5, 7), metallic_texture=tex(3, 3), roughness_texture=tex(12, 4, 0.1, 0.9),
                  normal_texture=normal_map(19, 13))]
    g_mat = sc.instances[0].material
    sc.materials[g_mat] = dataclasses.replace(sc.materials[g_mat], diffuse_texture=tex(64, 48),
                                              roughness_texture=tex(33, 17, 0.2, 1.0))
    for k, inst in enumerate(sc.instances[1:]):
        sc.materials[inst.material] = dataclasses.replace(sc.materials[inst.material], **kinds[k % len(kinds)])
    return sc, cam


def orbit_camera(angle: float, width: int, height: int) -> Camera:
    """Config-2 camera on a circle of radius 22 at height 9 around the terrain centre."""
    eye = (22.0 * np.sin(angle), 9.0, 22.0 * np.cos(angle))
    return make_camera(eye, (0.0, 1.0, 0.0), width, height, fov=55.0)


def small_variant(cfg: int, width: int, height: int, **kw):
    """The same scene at a test-sized resolution (and optionally fewer lights / spheres)."""
    return {0: config0, 1: config1, 2: config2}[cfg](width=width, height=height, **kw)


def config_camera(cfg: int, width: int, height: int) -> Camera:
    """The camera of config 0 / 1 / 2 at another resolution."""
    if cfg == 0:
        return make_camera((0.0, 0.0, 0.95), (0.0, -0.2, 0.0), width, height, fov=70.0)
    if cfg == 1:
        return make_camera((0.0, 6.0, 9.0), (0.0, 0.0, 0.0), width, height, fov=55.0)
    return orbit_camera(0.0, width, height)


CONFIG4_RESOLUTIONS = ((256, 256), (512, 512), (1280, 720), (1920, 1080), (2048, 1152))
CONFIG4_SEED = 0xC0FFEE04


def config4_jobs(n_jobs: int, rate: float = 200.0, seed: int = CONFIG4_SEED) -> list[dict]:
    """Serving workload (config 4): Poisson arrivals at `rate` jobs/s; scene uniform
    over configs 0-2; resolution uniform over CONFIG4_RESOLUTIONS; frames (spp)
    uniform over 1..16; pipeline ReSTIR (config-2 settings: 32 candidates, reservoir,
    maxDepth 1) or PathTracer (maxDepth 4) with equal odds."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_jobs))
    jobs = []
    for k in range(n_jobs):
        w, h = CONFIG4_RESOLUTIONS[int(rng.integers(len(CONFIG4_RESOLUTIONS)))]
        jobs.append({"arrival": float(t[k]), "cfg": int(rng.integers(3)), "width": w, "height": h,
                     "frames": int(rng.integers(1, 17)), "pipeline": "ris" if rng.random() < 0.5 else "pt"})
    return jobs


RIS_CONFIG2 = dict(candidate_count=32, use_reservoir=True, max_depth=1)
PT_CONFIG4 = dict(max_depth=4)


def dome_texture(width: int = 2048, height: int = 1024, sun_uv=(0.3, 0.28), sun_radius=0.012,
                 sun_radiance=400.0) -> np.ndarray:
    """Procedural environment map (H, W, 3) f32, rows from the top of the lat-long
    image: a sky gradient (bluish at the top, warm at the horizon row, dim ground
    below it) and a Gaussian sun lobe."""
    v = (np.arange(height, dtype=np.float64) + 0.5) / height
    u = (np.arange(width, dtype=np.float64) + 0.5) / width
    vv, uu = np.meshgrid(v, u, indexing="ij")
    up = np.clip(1.0 - 2.0 * vv, -1.0, 1.0)  # +1 at the top row, -1 at the bottom
    zen = np.array([0.25, 0.45, 0.95])
    hor = np.array([0.95, 0.85, 0.70])
    gnd = np.array([0.12, 0.10, 0.08])
    t = np.clip(up, 0.0, 1.0)[..., None] ** 0.6
    sky = hor * (1.0 - t) + zen * t
    img = np.where((up >= 0.0)[..., None], sky, gnd * (1.0 + up[..., None]))
    du = np.minimum(np.abs(uu - sun_uv[0]), 1.0 - np.abs(uu - sun_uv[0]))
    d2 = (du * 2.0) ** 2 + (vv - sun_uv[1]) ** 2
    img = img + (sun_radiance * np.exp(-d2 / (2.0 * sun_radius ** 2)))[..., None] * np.array([1.0, 0.95, 0.85])
    return np.ascontiguousarray(img, np.float32)


def config3(width=3840, height=2160, n_small=64, small=512, grid=512, n_spheres=2000, n_lights=10000,
            dome_size=(2048, 1024)):
    """Config 3: the config-2 scene lit also by a procedural 2048x1024 dome; one
    width x height camera and n_small orbit cameras of small x small pixels."""
    sc, cam = config2(width, height, grid=grid, n_spheres=n_spheres, n_lights=n_lights)
    sc.lights.append(Light(abi.LIGHT_DOME, color=(1.0, 1.0, 1.0), intensity=1.0,
                           texture=dome_texture(*dome_size)))
    cams = [orbit_camera(2.0 * np.pi * k / max(1, n_small), small, small) for k in range(n_small)]
    return sc, cam, cams


PT_CONFIG3 = dict(max_depth=16)
