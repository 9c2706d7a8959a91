"""LoadScene(path): the native glTF loader with the reference's conventions
(default material first, glTF material i -> i + 1, y-up -> z-up root
rotation), checked on the host against the in-memory descriptions it was
written from, and the C++23 crystal::graphics layer's error path."""
import base64
import json
import os
import struct
import subprocess

import numpy as np
import pytest

import oracle as O
from crystalgraphics_b200 import backend as B
from crystalgraphics_b200 import gltf, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("make", [lambda: scenes.cornell(),
                                  lambda: scenes.icosphere_scene(subdiv=3)])
def test_gltf_round_trip_is_exact(tmp_path, make):
    s = make()
    path = gltf.write(s, str(tmp_path / "scene.gltf"))
    p = B.parse_gltf(path)
    # default material first, then the written ones
    assert len(p.materials) == len(s.materials) + 1
    assert p.materials[0]["metallic_factor"] == 1.0 and p.materials[0]["ior"] == np.float32(1.5)
    for f in ("base_color_factor", "emissive_factor", "emissive_strength", "metallic_factor",
              "roughness_factor", "ior", "dispersion", "transmission_factor", "thickness_factor"):
        np.testing.assert_array_equal(p.materials[f][1:], s.materials[f], err_msg=f)
    # instances: same order, same world matrix bits, material shifted by one
    assert len(p.instances) == len(s.instances)
    assert p.instances["world_from_local"].tobytes() == s.instances["world_from_local"].tobytes()
    np.testing.assert_array_equal(p.instances["material"], s.instances["material"] + 1)
    # geometry of every instance identical (shared geometry stays shared)
    assert len(p.meshes) == len(s.meshes)
    for k in range(len(s.instances)):
        a, b = s.meshes[s.instances[k]["mesh"]], p.meshes[p.instances[k]["mesh"]]
        va = s.vertices[a["vertex_offset"]:a["vertex_offset"] + a["vertex_count"]]
        vb = p.vertices[b["vertex_offset"]:b["vertex_offset"] + b["vertex_count"]]
        assert va["position"].tobytes() == vb["position"].tobytes()
        assert va["normal"].tobytes() == vb["normal"].tobytes()
        ia = s.indices[a["index_offset"]:a["index_offset"] + a["index_count"]] - a["vertex_offset"]
        ib = p.indices[b["index_offset"]:b["index_offset"] + b["index_count"]] - b["vertex_offset"]
        np.testing.assert_array_equal(ia, ib)


def test_gltf_scene_packs_identically_in_the_oracle(tmp_path):
    s = scenes.icosphere_scene(subdiv=3)
    p = B.parse_gltf(gltf.write(s, str(tmp_path / "s.gltf")))
    a, aa, _ = O.OracleScene(s).emissive()
    b, ba, _ = O.OracleScene(p).emissive()
    assert a.tobytes() == b.tobytes() and aa.tobytes() == ba.tobytes()


def test_glb_container(tmp_path):
    s = scenes.cornell()
    path = gltf.write(s, str(tmp_path / "c.gltf"))
    doc = json.load(open(path))
    binary = open(path[:-5] + ".bin", "rb").read()
    del doc["buffers"][0]["uri"]
    js = json.dumps(doc).encode()
    js += b" " * ((-len(js)) % 4)
    binary += b"\0" * ((-len(binary)) % 4)
    glb = struct.pack("<4sII", b"glTF", 2, 12 + 8 + len(js) + 8 + len(binary))
    glb += struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(binary), 0x004E4942) + binary
    gp = tmp_path / "c.glb"
    gp.write_bytes(glb)
    p = B.parse_gltf(str(gp))
    assert p.instances["world_from_local"].tobytes() == s.instances["world_from_local"].tobytes()


def test_gltf_errors(tmp_path):
    with pytest.raises(B.Error, match="cannot open"):
        B.parse_gltf(str(tmp_path / "missing.gltf"))
    bad = tmp_path / "bad.gltf"
    bad.write_text("{ this is not json")
    with pytest.raises(B.Error, match="invalid JSON"):
        B.parse_gltf(str(bad))
    lines = tmp_path / "lines.gltf"
    lines.write_text(json.dumps({"asset": {"version": "2.0"},
                                 "meshes": [{"primitives": [{"attributes": {"POSITION": 0},
                                                             "mode": 1}]}]}))
    with pytest.raises(B.Error, match="triangle"):
        B.parse_gltf(str(lines))


def test_cxx_layer_reports_errors_through_expected(tmp_path):
    exe = os.path.join(ROOT, "crystalgraphics_b200", "cg_view")
    if not os.path.exists(exe):
        pytest.skip("C++ layer not built")
    r = subprocess.run([exe, str(tmp_path / "missing.gltf"), str(tmp_path / "o.ppm")],
                       capture_output=True, text=True)
    assert r.returncode == 1
    assert ("EnvInit" in r.stderr) or ("LoadScene" in r.stderr)


def test_gltf_textures_round_trip(tmp_path):
    """Images (PNG in the binary buffer), samplers' wrap modes, textures, the
    materials' texture references and TEXCOORD_0/1 survive write -> parse; the
    parsed scene packs the same light buffer in the oracle."""
    s = scenes.textured_cornell()
    p = B.parse_gltf(gltf.write(s, str(tmp_path / "t.gltf")))
    assert len(p.textures) == len(s.textures) == 4
    for (a, ws, wt), (b, ws2, wt2) in zip(s.textures, p.textures):
        assert np.array_equal(a, b) and (ws, wt) == (ws2, wt2)
    for f in ("base_color_texture", "metallic_roughness_texture", "emissive_texture",
              "transmission_texture", "texcoord_sets"):
        np.testing.assert_array_equal(p.materials[f][1:], s.materials[f], err_msg=f)
    for k in range(len(s.instances)):
        a, b = s.meshes[s.instances[k]["mesh"]], p.meshes[p.instances[k]["mesh"]]
        va = s.vertices[a["vertex_offset"]:a["vertex_offset"] + a["vertex_count"]]
        vb = p.vertices[b["vertex_offset"]:b["vertex_offset"] + b["vertex_count"]]
        assert va["tex_coord0"].tobytes() == vb["tex_coord0"].tobytes()
        assert va["tex_coord1"].tobytes() == vb["tex_coord1"].tobytes()
    a, aa, _ = O.OracleScene(s).emissive()
    b, ba, _ = O.OracleScene(p).emissive()
    assert a.tobytes() == b.tobytes() and aa.tobytes() == ba.tobytes()


def _one_triangle_doc(pos_accessor, extra_views=(), blob=b""):
    """A glTF with one indexed triangle whose POSITION accessor is given."""
    idx = np.array([0, 1, 2], np.uint16).tobytes() + b"\0\0"
    uv = np.array([[0, 255], [128, 7], [255, 0]], np.uint8).tobytes() + b"\0\0"
    data = idx + uv + blob
    views = [{"buffer": 0, "byteOffset": 0, "byteLength": 6},
             {"buffer": 0, "byteOffset": 8, "byteLength": 6}] + list(extra_views)
    accs = [{"bufferView": 0, "componentType": 5123, "count": 3, "type": "SCALAR"},
            {"bufferView": 1, "componentType": 5121, "normalized": True, "count": 3, "type": "VEC2"},
            pos_accessor]
    return {"asset": {"version": "2.0"},
            "buffers": [{"byteLength": len(data),
                         "uri": "data:application/octet-stream;base64," + base64.b64encode(data).decode()}],
            "bufferViews": views, "accessors": accs,
            "meshes": [{"primitives": [{"attributes": {"POSITION": 2, "TEXCOORD_0": 1}, "indices": 0}]}],
            "nodes": [{"mesh": 0}], "scenes": [{"nodes": [0]}], "scene": 0}


def _load(tmp_path, doc):
    p = tmp_path / "t.gltf"
    p.write_text(json.dumps(doc))
    return B.parse_gltf(str(p))


def test_normalized_and_sparse_accessors(tmp_path):
    # normalized u8 texture coordinates: c / 255 divided in float (cgltf)
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32).tobytes()
    dense = {"bufferView": 2, "componentType": 5126, "count": 3, "type": "VEC3"}
    p = _load(tmp_path, _one_triangle_doc(dense, [{"buffer": 0, "byteOffset": 16, "byteLength": 36}], pos))
    uv = np.array([[0, 255], [128, 7], [255, 0]], np.float32) / np.float32(255)
    assert p.vertices["tex_coord0"].tobytes() == uv.astype(np.float32).tobytes()
    assert p.vertices["position"].reshape(-1).tobytes() == pos
    # a sparse POSITION accessor: cgltf's element reader does not apply it, so
    # the reference's vertices keep the zero they were resized to
    sp_idx = np.array([1], np.uint8).tobytes() + b"\0\0\0"
    sp_val = np.array([5, 6, 7], np.float32).tobytes()
    views = [{"buffer": 0, "byteOffset": 16, "byteLength": 36},
             {"buffer": 0, "byteOffset": 52, "byteLength": 1},
             {"buffer": 0, "byteOffset": 56, "byteLength": 12}]
    sparse = dict(dense, sparse={"count": 1, "indices": {"bufferView": 3, "componentType": 5121},
                                 "values": {"bufferView": 4}})
    p = _load(tmp_path, _one_triangle_doc(sparse, views, pos + sp_idx + sp_val))
    assert len(p.vertices) == 3 and not p.vertices["position"].any()
    np.testing.assert_array_equal(p.indices, [0, 1, 2])
    # the usual form, a sparse accessor with no bufferView, reads as zeros too
    no_view = {k: v for k, v in sparse.items() if k != "bufferView"}
    p = _load(tmp_path, _one_triangle_doc(no_view, views, pos + sp_idx + sp_val))
    assert len(p.vertices) == 3 and not p.vertices["position"].any()
    # cgltf_validate's checks of the sparse block
    bad_index = np.array([3], np.uint8).tobytes() + b"\0\0\0"
    with pytest.raises(B.Error, match="sparse accessor index"):
        _load(tmp_path, _one_triangle_doc(sparse, views, pos + bad_index + sp_val))
    short = [views[0], views[1], dict(views[2], byteLength=8)]
    with pytest.raises(B.Error, match="exceeds its buffer view"):
        _load(tmp_path, _one_triangle_doc(sparse, short, pos + sp_idx + sp_val))


def test_damaged_documents_fail_cleanly(tmp_path):
    """Damage found by fuzzing the loader: each fails the load with an error
    instead of exhausting the stack, allocating for an absurd count, reading
    outside a buffer or throwing across the C ABI."""
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32).tobytes()
    view = [{"buffer": 0, "byteOffset": 16, "byteLength": 36}]
    dense = {"bufferView": 2, "componentType": 5126, "count": 3, "type": "VEC3"}
    _load(tmp_path, _one_triangle_doc(dense, view, pos))  # the undamaged document loads
    cases = [
        (dict(dense, count=-1), view, "invalid accessor count"),
        (dict(dense, count=2 ** 31), view, "exceeds its buffer"),
        ({"componentType": 5126, "count": 2 ** 31, "type": "VEC3"}, view, "too many elements"),
        (dict(dense, byteOffset=-8), view, "exceeds its buffer"),
        (dense, [dict(view[0], byteOffset=-16)], "bufferView exceeds its buffer"),
        (dense, [dict(view[0], byteLength=2 ** 63)], "bufferView exceeds its buffer"),
        (dense, [dict(view[0], byteLength=24)], "exceeds its buffer"),
        (dense, [dict(view[0], byteStride=-4)], "invalid byteStride"),
    ]
    for acc, views, msg in cases:
        with pytest.raises(B.Error, match=msg):
            _load(tmp_path, _one_triangle_doc(acc, views, pos))
    doc = _one_triangle_doc(dense, view, pos)
    doc["scenes"][0]["nodes"] = [1e30]
    with pytest.raises(B.Error, match="bad node index"):
        _load(tmp_path, doc)
    p = tmp_path / "deep.gltf"
    for text in ("[" * 100000 + "]" * 100000, '{"a":' * 50000 + "1" + "}" * 50000):
        p.write_text(text)
        with pytest.raises(B.Error, match="nested too deeply"):
            B.parse_gltf(str(p))
    p.write_text('{"asset": {"version": "2.0"}, "s": "\\uZZZZ"}')
    with pytest.raises(B.Error, match="bad unicode escape"):
        B.parse_gltf(str(p))


def test_node_hierarchy_must_be_a_forest(tmp_path):
    """A node listed as the child of two nodes, or parent links that loop, fail
    the load (cgltf rejects both while parsing and validating).  A diamond
    chain 40 levels deep, each node naming the next one twice, would otherwise
    have 2^40 paths from the root."""
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32).tobytes()
    view = [{"buffer": 0, "byteOffset": 16, "byteLength": 36}]
    dense = {"bufferView": 2, "componentType": 5126, "count": 3, "type": "VEC3"}
    doc = _one_triangle_doc(dense, view, pos)
    doc["nodes"] = [{"mesh": 0, "children": [k + 1, k + 1]} for k in range(40)] + [{"mesh": 0}]
    with pytest.raises(B.Error, match="has two parents"):
        _load(tmp_path, doc)
    doc["nodes"] = [{"mesh": 0}, {"children": [2]}, {"children": [1]}]
    with pytest.raises(B.Error, match="cycle"):
        _load(tmp_path, doc)
    doc["nodes"] = [{"mesh": 0, "children": [0]}]
    with pytest.raises(B.Error, match="cycle"):
        _load(tmp_path, doc)
    # a proper tree still loads: one instance per node that holds the mesh
    doc["nodes"] = [{"mesh": 0, "children": [1, 2]}, {"mesh": 0}, {"mesh": 0, "children": [3]},
                    {"mesh": 0}]
    assert len(_load(tmp_path, doc).instances) == 4
