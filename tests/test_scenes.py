"""The synthetic benchmark scenes: sizes and determinism."""
import numpy as np

from hdrestir_b200 import configs


def test_config0_sizes():
    sc, cam = configs.config0()
    assert sc.num_triangles == 24 and len(sc.lights) == 2 and (cam.width, cam.height) == (256, 256)
    for L in sc.lights:
        assert L.width == 0.3 and L.height == 0.3 and 10.0 <= L.color[0] <= 20.0


def test_config1_sizes():
    sc, cam = configs.config1()
    assert sc.num_triangles == 2 + 64 * 12 and len(sc.lights) == 1024
    side = np.array([L.width for L in sc.lights])
    assert side.min() >= 0.02 and side.max() <= 0.1
    assert (cam.width, cam.height) == (512, 512)


def test_config2_sizes():
    sc, cam = configs.config2()
    assert sc.num_triangles == 2 * 511 * 511 + 2000 * 256 == 1034242
    assert len(sc.lights) == 10000 and len(sc.instances) == 2001
    assert (cam.width, cam.height) == (1920, 1080)
    assert len(sc.meshes[1].indices) == 256


def test_generators_are_deterministic():
    a, _ = configs.config1(32, 32, n_lights=16)
    b, _ = configs.config1(32, 32, n_lights=16)
    assert all(np.array_equal(x.points, y.points) for x, y in zip(a.meshes, b.meshes))
    assert [m.diffuse_color for m in a.materials] == [m.diffuse_color for m in b.materials]


def test_blackbody_normalised():
    rgb = configs.blackbody_rgb(np.array([2000.0, 6500.0, 9000.0]))
    lum = rgb @ np.array([0.2126, 0.7152, 0.0722])
    np.testing.assert_allclose(lum, 1.0, rtol=1e-12)
    assert rgb[0, 0] > rgb[0, 2] and rgb[2, 2] > rgb[2, 0]  # warm vs cool


def test_textured_variant_descriptor():
    """Texture arrays reach hdr_material_desc: pointer, width and height per slot (HDR_TEX_*),
    untextured slots NULL; the descriptor keeps the texel arrays alive."""
    import ctypes as C

    from hdrestir_b200 import abi
    from hdrestir_b200.scene import TEXTURE_FIELDS

    sc, _ = configs.textured_variant(16, 16)
    desc = sc.c_desc()
    seen = 0
    for k, m in enumerate(sc.materials):
        d = desc.materials[k]
        for slot, f in enumerate(TEXTURE_FIELDS):
            tex = getattr(m, f)
            if tex is None:
                assert not d.textures[slot]
                continue
            seen += 1
            assert (d.tex_height[slot], d.tex_width[slot]) == tex.shape[:2]
            got = np.ctypeslib.as_array(d.textures[slot], shape=(tex.size,))
            assert np.array_equal(got, np.ascontiguousarray(tex, np.float32).reshape(-1))
    assert seen >= 8
    assert C.sizeof(abi.MaterialDesc) % 8 == 0
