"""Python binding of hdr_material_from_network: a Hydra material network
(HdMaterialNetwork2) given as plain data, mapped to PreviewSurface parameters as
HdRestirMaterial::Sync does (hydra/hd_restir_material.cpp:22-424).

A network is ``{"nodes": {path: {"id": shader id, "params": {name: value},
"inputs": {input: [upstream path, ...]}}}, "terminals": {name: node path}}``.
Parameter values: a float, a 3-tuple of floats, a bool, or ``Asset(path)``.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

from . import abi
from .scene import Material


@dataclasses.dataclass(frozen=True)
class Asset:
    path: str


def _param(name: str, value) -> abi.MtlParam:
    p = abi.MtlParam()
    p.name = name.encode()
    if isinstance(value, Asset):
        p.type, p.asset = abi.MTL_ASSET, value.path.encode()
    elif isinstance(value, bool):
        p.type = abi.MTL_BOOL
        p.value[0] = 1.0 if value else 0.0
    elif isinstance(value, (tuple, list)):
        p.type = abi.MTL_FLOAT3
        for k in range(3):
            p.value[k] = float(value[k])
    else:
        p.type = abi.MTL_FLOAT
        p.value[0] = float(value)
    return p


def material_from_network(network: dict) -> tuple[dict, dict]:
    """Returns ({hdr_material_desc field: value}, {texture slot: asset path}) for a
    network: every numeric PreviewSurface field (3-tuples for colours), and the asset
    path of each texture slot ("diffuse", "metallic", "roughness", "normal") set."""
    keep = []
    nodes = []
    for path, node in network.get("nodes", {}).items():
        params = (abi.MtlParam * max(1, len(node.get("params", {}))))(
            *[_param(k, v) for k, v in node.get("params", {}).items()])
        conns = [(i, u) for i, ups in node.get("inputs", {}).items() for u in ups]
        inputs = (abi.MtlConnection * max(1, len(conns)))(
            *[abi.MtlConnection(i.encode(), u.encode()) for i, u in conns])
        keep += [params, inputs]
        nodes.append(abi.MtlNode(path.encode(), node["id"].encode(), params, len(node.get("params", {})), inputs,
                                 len(conns)))
    terms = [abi.MtlTerminal(k.encode(), v.encode()) for k, v in network.get("terminals", {}).items()]
    net = abi.MtlNetwork((abi.MtlNode * max(1, len(nodes)))(*nodes), len(nodes),
                         (abi.MtlTerminal * max(1, len(terms)))(*terms), len(terms))
    out, tex = abi.MaterialDesc(), abi.MtlTextures()
    abi.check(abi.lib().hdr_material_from_network(C.byref(net), C.byref(out), C.byref(tex)))
    fields = {}
    for name, _ in abi.MaterialDesc._fields_:
        if name in ("textures", "tex_width", "tex_height"):
            continue
        v = getattr(out, name)
        fields[name] = tuple(v) if isinstance(v, C.Array) else v
    slots = ("diffuse", "metallic", "roughness", "normal")
    textures = {slots[k]: tex.path[k].value.decode() for k in range(4) if tex.path[k].value}
    return fields, textures


def to_material(fields: dict) -> Material:
    """The scene description's Material with the fields it carries."""
    names = {f.name for f in dataclasses.fields(Material)}
    kw = {k: v for k, v in fields.items() if k in names}
    kw["thin_walled"] = bool(fields["thin_walled"])
    return Material(**kw)
