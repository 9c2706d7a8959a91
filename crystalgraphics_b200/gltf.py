"""glTF 2.0 export of scene descriptions, for LoadScene(path).

``write(scene, path)`` stores a :class:`crystalgraphics_b200.scenes.Scene` as
``path`` (.gltf JSON) plus ``path[:-5] + '.bin'``, such that the reference's
loading conventions (src/scene.cpp:829-1003) give back the same world:

  - every instance becomes a root node whose matrix is Rx(-90 deg) @ W, so
    the loader's y-up -> z-up rotation Rx(+90 deg) restores W exactly;
  - scene material k is written as glTF material k, which the loader places
    at k + 1 behind the default material;
  - a (mesh, material) pair is one glTF mesh whose primitive shares the
    mesh's accessors.

Loading is native (cg_scene_load_gltf in libcg_cuda.so).
"""
from __future__ import annotations

import json
import os

import numpy as np

from . import png

_RX_NEG90 = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, -1, 0, 0], [0, 0, 0, 1]], np.float64)


def write(scene, path: str) -> str:
    assert path.endswith(".gltf")
    bin_path = path[:-5] + ".bin"
    blobs = []
    offset = 0
    views, accessors = [], []

    def add(arr: np.ndarray, target=None):
        nonlocal offset
        data = np.ascontiguousarray(arr).tobytes()
        pad = (-len(data)) % 4
        views.append({"buffer": 0, "byteOffset": offset, "byteLength": len(data),
                      **({"target": target} if target else {})})
        blobs.append(data + b"\0" * pad)
        offset += len(data) + pad
        return len(views) - 1

    mesh_acc = []
    for m in scene.meshes:
        vo, vc, io, ic = int(m["vertex_offset"]), int(m["vertex_count"]), int(m["index_offset"]), \
            int(m["index_count"])
        v = scene.vertices[vo:vo + vc]
        pos = np.ascontiguousarray(v["position"], np.float32)
        nrm = np.ascontiguousarray(v["normal"], np.float32)
        idx = (scene.indices[io:io + ic].astype(np.int64) - vo)
        assert idx.min(initial=0) >= 0 and idx.max(initial=0) < max(vc, 1), \
            "mesh indices must address the mesh's own vertex range"
        pv = add(pos, 34962)
        accessors.append({"bufferView": pv, "componentType": 5126, "count": vc, "type": "VEC3",
                          "min": pos.min(0).tolist() if vc else [0, 0, 0],
                          "max": pos.max(0).tolist() if vc else [0, 0, 0]})
        pa = len(accessors) - 1
        nv = add(nrm, 34962)
        accessors.append({"bufferView": nv, "componentType": 5126, "count": vc, "type": "VEC3"})
        na = len(accessors) - 1
        uv_acc = []
        for key in ("tex_coord0", "tex_coord1"):
            uv = np.ascontiguousarray(v[key], np.float32)
            if vc and np.any(uv != 0):
                uvv = add(uv, 34962)
                accessors.append({"bufferView": uvv, "componentType": 5126, "count": vc,
                                  "type": "VEC2"})
                uv_acc.append(len(accessors) - 1)
            else:
                uv_acc.append(None)
        iv = add(idx.astype(np.uint32), 34963)
        accessors.append({"bufferView": iv, "componentType": 5125, "count": ic, "type": "SCALAR"})
        mesh_acc.append((pa, na, len(accessors) - 1, uv_acc))

    # textures: one PNG image (in the binary buffer), one sampler per texture
    images, samplers, textures = [], [], []
    for img, wrap_s, wrap_t in getattr(scene, "textures", []) or []:
        bv = add(np.frombuffer(png.encode_rgba8(img), np.uint8))
        images.append({"bufferView": bv, "mimeType": "image/png"})
        samplers.append({"wrapS": int(wrap_s), "wrapT": int(wrap_t)})
        textures.append({"source": len(images) - 1, "sampler": len(samplers) - 1})

    def tex_info(m, field, slot):
        t = int(m[field])
        if t < 0:
            return None
        return {"index": t, "texCoord": int((int(m["texcoord_sets"]) >> slot) & 1)}

    materials = []
    for m in scene.materials:
        mat = {"pbrMetallicRoughness": {
            "baseColorFactor": [float(x) for x in m["base_color_factor"]],
            "metallicFactor": float(m["metallic_factor"]),
            "roughnessFactor": float(m["roughness_factor"])},
            "emissiveFactor": [float(x) for x in m["emissive_factor"]]}
        pbr = mat["pbrMetallicRoughness"]
        if tex_info(m, "base_color_texture", 0):
            pbr["baseColorTexture"] = tex_info(m, "base_color_texture", 0)
        if tex_info(m, "metallic_roughness_texture", 1):
            pbr["metallicRoughnessTexture"] = tex_info(m, "metallic_roughness_texture", 1)
        if tex_info(m, "emissive_texture", 2):
            mat["emissiveTexture"] = tex_info(m, "emissive_texture", 2)
        ext = {}
        if float(m["emissive_strength"]) != 1.0:
            ext["KHR_materials_emissive_strength"] = {"emissiveStrength": float(m["emissive_strength"])}
        ext["KHR_materials_ior"] = {"ior": float(m["ior"])}
        if float(m["dispersion"]):
            ext["KHR_materials_dispersion"] = {"dispersion": float(m["dispersion"])}
        if float(m["transmission_factor"]) or int(m["transmission_texture"]) >= 0:
            ext["KHR_materials_transmission"] = {"transmissionFactor": float(m["transmission_factor"])}
            if tex_info(m, "transmission_texture", 3):
                ext["KHR_materials_transmission"]["transmissionTexture"] = \
                    tex_info(m, "transmission_texture", 3)
        if float(m["thickness_factor"]):
            ext["KHR_materials_volume"] = {"thicknessFactor": float(m["thickness_factor"])}
        mat["extensions"] = ext
        materials.append(mat)

    gl_meshes, mesh_of = [], {}
    nodes = []
    for inst in scene.instances:
        key = (int(inst["mesh"]), int(inst["material"]))
        if key not in mesh_of:
            pa, na, ia, uv_acc = mesh_acc[key[0]]
            attrs = {"POSITION": pa, "NORMAL": na}
            for k, a in enumerate(uv_acc):
                if a is not None:
                    attrs[f"TEXCOORD_{k}"] = a
            gl_meshes.append({"primitives": [{"attributes": attrs,
                                              "indices": ia, "material": key[1], "mode": 4}]})
            mesh_of[key] = len(gl_meshes) - 1
        W = np.eye(4)
        W[:3, :4] = inst["world_from_local"].reshape(3, 4).astype(np.float64)
        M = _RX_NEG90 @ W
        nodes.append({"mesh": mesh_of[key],
                      "matrix": [float(np.float32(x)) for x in M.T.reshape(-1)]})
    doc = {
        "asset": {"version": "2.0", "generator": "crystalgraphics_b200.gltf"},
        "extensionsUsed": ["KHR_materials_emissive_strength", "KHR_materials_ior",
                           "KHR_materials_dispersion", "KHR_materials_transmission",
                           "KHR_materials_volume"],
        "buffers": [{"uri": os.path.basename(bin_path), "byteLength": offset}],
        "bufferViews": views, "accessors": accessors, "materials": materials,
        "meshes": gl_meshes, "nodes": nodes, "scenes": [{"nodes": list(range(len(nodes)))}],
        "scene": 0,
    }
    if textures:
        doc.update(images=images, samplers=samplers, textures=textures)
    with open(bin_path, "wb") as f:
        for b in blobs:
            f.write(b)
    with open(path, "w") as f:
        json.dump(doc, f)
    return path
