"""hdr_material_from_network (HdRestirMaterial::Sync's network walk,
hydra/hd_restir_material.cpp:22-424) on the host, through the C ABI.

The reference's walk needs Hydra's material network and the Sdr registry, so it
is not compiled here; these are known answers read off that source: each shader
family's parameter names and the PreviewSurface field each sets, the typed
lookups (a parameter holding another type is skipped), name order within a node
(a later name wins, e.g. "specular_roughness" over "roughness", "coat_ior" over
"coat_IOR"), diffuse = base colour x base weight with defaults 0.8 and 1, image
nodes mapped by the surface input their chain starts from, the emission chain
filling the diffuse slot only while it is empty, the terminal priority and
visiting each node once.
"""
import numpy as np
import pytest

from hdrestir_b200.material_network import Asset, material_from_network, to_material

DEFAULTS = dict(diffuse_color=(1.0, 1.0, 1.0), metallic=0.0, roughness=0.5, specular_color=(1.0, 1.0, 1.0),
                specular=1.0, opacity=1.0, ior=1.5, transmission=0.0, transmission_color=(1.0, 1.0, 1.0),
                transmission_depth=0.0, transmission_scatter=(0.0, 0.0, 0.0), emission_color=(1.0, 1.0, 1.0),
                emission=0.0, coat=0.0, coat_color=(1.0, 1.0, 1.0), coat_roughness=0.1, coat_ior=1.5, sheen=0.0,
                sheen_color=(1.0, 1.0, 1.0), sheen_roughness=0.3, subsurface=0.0, subsurface_color=(1.0, 1.0, 1.0),
                subsurface_radius=(1.0, 1.0, 1.0), subsurface_scale=1.0, subsurface_anisotropy=0.0, thin_walled=0,
                diffuse_roughness=0.0)


def _f32(v):
    return tuple(np.float32(x) for x in v) if isinstance(v, tuple) else np.float32(v)


def _check(fields, **want):
    exp = dict(DEFAULTS, **want)
    for k, v in exp.items():
        got = fields[k]
        if isinstance(v, tuple):
            assert tuple(np.float32(g) for g in got) == _f32(v), k
        else:
            assert np.float32(got) == _f32(v), k


def _net(node_id, params, inputs=None, extra=None, terminal="surface"):
    nodes = {"/mat/surf": {"id": node_id, "params": params, "inputs": inputs or {}}}
    nodes.update(extra or {})
    return {"nodes": nodes, "terminals": {terminal: "/mat/surf"}}


def test_defaults_without_terminal():
    fields, tex = material_from_network({"nodes": {}, "terminals": {}})
    _check(fields)
    assert tex == {}


def test_preview_surface():
    fields, _ = material_from_network(_net("UsdPreviewSurface", {
        "diffuseColor": (0.2, 0.4, 0.6), "metallic": 0.7, "roughness": 0.25, "specularColor": (0.9, 0.8, 0.7),
        "opacity": 0.5, "ior": 1.33, "emissiveColor": (2.0, 1.0, 0.5),
        "clearcoat": 0.9,                 # not a parameter the reference reads
        "useSpecularWorkflow": 1.0}))
    _check(fields, diffuse_color=(0.2, 0.4, 0.6), metallic=0.7, roughness=0.25, specular_color=(0.9, 0.8, 0.7),
           opacity=0.5, ior=1.33, emission_color=(2.0, 1.0, 0.5), emission=1.0)


def test_standard_surface_fields_and_name_order():
    fields, _ = material_from_network(_net("ND_standard_surface_surfaceshader", {
        "base": 0.5, "base_color": (0.8, 0.4, 0.2), "metalness": 0.3, "specular": 0.6,
        "specular_color": (0.5, 0.6, 0.7),
        "roughness": 0.7, "specular_roughness": 0.2,     # "specular_roughness" sorts later and wins
        "coat_IOR": 1.6, "coat_ior": 1.4,                # "coat_ior" sorts later ('i' > 'I') and wins
        "ior": 1.45, "opacity": 0.75, "transmission": 0.3, "transmission_color": (0.1, 0.2, 0.3),
        "transmission_depth": 2.0, "transmission_scatter": (0.3, 0.2, 0.1), "subsurface": 0.4,
        "subsurface_color": (0.9, 0.5, 0.4), "subsurface_radius": (1.0, 0.5, 0.25), "subsurface_scale": 0.1,
        "subsurface_anisotropy": 0.2, "sheen": 0.35, "sheen_color": (0.2, 0.3, 0.4), "sheen_roughness": 0.6,
        "coat": 0.8, "coat_color": (0.7, 0.7, 0.9), "coat_roughness": 0.05, "thin_walled": True,
        "diffuse_roughness": 0.15, "emission": 3.0, "emission_color": (1.0, 0.5, 0.25)}))
    _check(fields, diffuse_color=(np.float32(0.8) * np.float32(0.5), np.float32(0.4) * np.float32(0.5),
                                  np.float32(0.2) * np.float32(0.5)),
           metallic=0.3, specular=0.6, specular_color=(0.5, 0.6, 0.7), roughness=0.2, coat_ior=1.4, ior=1.45,
           opacity=0.75, transmission=0.3, transmission_color=(0.1, 0.2, 0.3), transmission_depth=2.0,
           transmission_scatter=(0.3, 0.2, 0.1), subsurface=0.4, subsurface_color=(0.9, 0.5, 0.4),
           subsurface_radius=(1.0, 0.5, 0.25), subsurface_scale=0.1, subsurface_anisotropy=0.2, sheen=0.35,
           sheen_color=(0.2, 0.3, 0.4), sheen_roughness=0.6, coat=0.8, coat_color=(0.7, 0.7, 0.9),
           coat_roughness=0.05, thin_walled=1, diffuse_roughness=0.15, emission=3.0,
           emission_color=(1.0, 0.5, 0.25))


@pytest.mark.parametrize("sid", ["standard_surface", "StandardSurface"])
def test_standard_surface_weights_and_types(sid):
    fields, _ = material_from_network(_net(sid, {
        "base_weight": 0.25, "specular_weight": 0.4, "transmission_weight": 0.6, "subsurface_weight": 0.1,
        "sheen_weight": 0.2, "coat_weight": 0.9, "emission_weight": 5.0,
        "metalness": (1.0, 1.0, 1.0),   # wrong type: skipped
        "thin_walled": 1.0}))           # a float where a bool is read: skipped
    _check(fields, diffuse_color=(np.float32(0.8) * np.float32(0.25),) * 3, specular=0.4, transmission=0.6,
           subsurface=0.1, sheen=0.2, coat=0.9, emission=5.0)


@pytest.mark.parametrize("sid", ["ND_open_pbr_surface_surfaceshader", "open_pbr_surface"])
def test_open_pbr_surface(sid):
    fields, _ = material_from_network(_net(sid, {
        "base_weight": 0.5, "base_color": (0.2, 0.4, 0.8), "base_metalness": 0.9, "specular_weight": 0.7,
        "specular_color": (0.9, 0.9, 0.8), "specular_roughness": 0.3, "geometry_opacity": 0.6,
        "specular_ior": 1.7, "transmission_weight": 0.2, "transmission_color": (0.5, 0.6, 0.7),
        "transmission_depth": 1.5, "transmission_scatter": (0.1, 0.1, 0.2), "subsurface_weight": 0.3,
        "subsurface_color": (0.8, 0.3, 0.2), "subsurface_radius": (0.5, 0.25, 0.125),
        "subsurface_radius_scale": 0.05, "subsurface_anisotropy": -0.2, "fuzz_weight": 0.4,
        "fuzz_color": (0.3, 0.2, 0.1), "fuzz_roughness": 0.8, "coat_weight": 0.6, "coat_color": (0.6, 0.7, 0.8),
        "coat_roughness": 0.02, "coat_ior": 1.55, "geometry_thin_walled": True, "emission_luminance": 12.0,
        "emission_color": (1.0, 0.9, 0.8),
        "base": 0.1, "metalness": 0.5, "specular": 0.1}))  # standard_surface names: not read here
    _check(fields, diffuse_color=(np.float32(0.2) * np.float32(0.5), np.float32(0.4) * np.float32(0.5),
                                  np.float32(0.8) * np.float32(0.5)),
           metallic=0.9, specular=0.7, specular_color=(0.9, 0.9, 0.8), roughness=0.3, opacity=0.6, ior=1.7,
           transmission=0.2, transmission_color=(0.5, 0.6, 0.7), transmission_depth=1.5,
           transmission_scatter=(0.1, 0.1, 0.2), subsurface=0.3, subsurface_color=(0.8, 0.3, 0.2),
           subsurface_radius=(0.5, 0.25, 0.125), subsurface_scale=0.05, subsurface_anisotropy=-0.2, sheen=0.4,
           sheen_color=(0.3, 0.2, 0.1), sheen_roughness=0.8, coat=0.6, coat_color=(0.6, 0.7, 0.8),
           coat_roughness=0.02, coat_ior=1.55, thin_walled=1, emission=12.0, emission_color=(1.0, 0.9, 0.8))


def test_texture_slots_follow_the_surface_input():
    img = lambda f, node_id="ND_image_color3": {"id": node_id, "params": {"file": Asset(f)}}  # noqa: E731
    net = _net("ND_standard_surface_surfaceshader", {"base_color": (0.5, 0.5, 0.5)}, inputs={
        "base_color": ["/mat/albedo"], "emission_color": ["/mat/glow"], "metalness": ["/mat/metal"],
        "normal": ["/mat/nmap"], "specular_roughness": ["/mat/mul"]}, extra={
        "/mat/albedo": img("albedo.png"), "/mat/glow": img("glow.png"), "/mat/metal": img("metal.png", "ND_image_float"),
        "/mat/nmap": {"id": "ND_normalmap", "params": {}, "inputs": {"in": ["/mat/ntex"]}},
        "/mat/ntex": img("normal.png", "ND_image_vector3"),
        "/mat/mul": {"id": "ND_multiply_float", "params": {}, "inputs": {"in1": ["/mat/rough"], "in2": ["/mat/albedo"]}},
        "/mat/rough": img("rough.png", "ND_image_float"),
        "/mat/unused": img("unused.png")})
    fields, tex = material_from_network(net)
    # base_color sorts before emission_color: the albedo fills the diffuse slot first, the emission
    # image only fills it while it is empty; the roughness chain keeps its starting input through the
    # multiply node; /mat/albedo is visited once (through base_color), not again under the multiply
    assert tex == {"diffuse": "albedo.png", "metallic": "metal.png", "roughness": "rough.png",
                   "normal": "normal.png"}
    _check(fields, diffuse_color=(np.float32(0.5) * np.float32(1.0),) * 3)
    # without the albedo, the emission image takes the diffuse slot
    del net["nodes"]["/mat/surf"]["inputs"]["base_color"]
    _, tex = material_from_network(net)
    assert tex["diffuse"] == "glow.png"


def test_usd_uv_texture_and_terminal_priority():
    nodes = {"/m/preview": {"id": "UsdPreviewSurface", "params": {"metallic": 0.25},
                            "inputs": {"diffuseColor": ["/m/tex"]}},
             "/m/tex": {"id": "UsdUVTexture", "params": {"file": Asset("wood.jpg"), "texcoord": 3.0}},
             "/m/mtlx": {"id": "ND_standard_surface_surfaceshader", "params": {"metalness": 0.75}}}
    fields, tex = material_from_network({"nodes": nodes, "terminals": {"surface": "/m/preview",
                                                                       "mtlx:surface": "/m/mtlx"}})
    assert np.float32(fields["metallic"]) == np.float32(0.75) and tex == {}
    fields, tex = material_from_network({"nodes": nodes, "terminals": {"surface": "/m/preview",
                                                                       "outputs:surface": "/m/mtlx"}})
    assert np.float32(fields["metallic"]) == np.float32(0.25) and tex == {"diffuse": "wood.jpg"}
    # no priority terminal: the first by name
    fields, _ = material_from_network({"nodes": nodes, "terminals": {"zz": "/m/preview", "displacement": "/m/mtlx"}})
    assert np.float32(fields["metallic"]) == np.float32(0.75)


def test_to_material_roundtrip():
    fields, _ = material_from_network(_net("standard_surface", {"coat": 0.5, "thin_walled": True}))
    m = to_material(fields)
    assert m.coat == pytest.approx(0.5) and m.thin_walled is True
