"""Material textures: validation of the scene description (no GPU needed) and
the oracle's texture restatement (array resize, bilinear clamp-to-edge
sampling, the light buffer's nearest-texel factor with glTF wrap modes)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from crystalgraphics_b200 import _abi, scenes
from crystalgraphics_b200 import backend as B


def _scene_with(material_textures, textures):
    s = scenes.textured_cornell()
    s.materials = s.materials.copy()
    s.materials[0]["base_color_texture"] = material_textures
    s.textures = textures
    return s


def test_missing_texture_index_is_rejected():
    s = _scene_with(7, scenes.textured_cornell().textures)  # only 4 textures
    with pytest.raises(B.Error) as e:
        B.LoadScene(s)
    assert e.value.code == _abi.CG_E_INVALID
    assert "texture" in str(e.value)


def test_empty_texture_is_rejected():
    tex = list(scenes.textured_cornell().textures)
    tex[0] = (np.zeros((0, 4, 4), np.uint8), 10497, 10497)
    with pytest.raises(B.Error) as e:
        B.LoadScene(_scene_with(0, tex))
    assert e.value.code == _abi.CG_E_INVALID


def test_oracle_light_buffer_uses_the_emissive_texel():
    """The two light triangles take the nearest texel of the emissive texture
    at their mean UV (mirrored repeat in s, repeat in t)."""
    s = scenes.textured_cornell()
    prims, _, _ = O.OracleScene(s).emissive()
    assert len(prims) == 2
    img = s.textures[2][0]
    # mean UVs of the two triangles of the light quad, corners at
    # (-0.7, -0.7), (1.8, -0.7), (1.8, 1.8), (-0.7, 1.8)
    c = np.array([(-0.7, -0.7), (1.8, -0.7), (1.8, 1.8), (-0.7, 1.8)], np.float32)
    for tri, prim in zip([(0, 1, 2), (0, 2, 3)], prims):
        u = np.float32((c[tri[0], 0] + c[tri[1], 0]) + c[tri[2], 0]) / np.float32(3)
        v = np.float32((c[tri[0], 1] + c[tri[1], 1]) + c[tri[2], 1]) / np.float32(3)
        fu = u - np.floor(u)
        if int(np.floor(u)) % 2 != 0:
            fu = 1 - fu
        fv = v - np.floor(v)
        x = min(7, int(np.float32(fu) * 8))
        y = min(7, int(np.float32(fv) * 8))
        texel = img[y, x, :3].astype(np.float32) / np.float32(255)
        np.testing.assert_allclose(prim["emission"], 15.0 * texel, rtol=1e-6)


def test_oracle_renders_textures():
    """Textures change the oracle's image (and leave it finite)."""
    s = scenes.textured_cornell()
    conf = _abi.make_conf(32, 32, 2, 3)
    a, _, _ = O.OracleScene(s).render(conf, s.camera, rng=O.RNG_KEYED, prune=True)
    s2 = scenes.textured_cornell()
    s2.materials = s2.materials.copy()
    for k in ("base_color_texture", "metallic_roughness_texture", "emissive_texture",
              "transmission_texture"):
        s2.materials[k] = -1
    b, _, _ = O.OracleScene(s2).render(conf, s2.camera, rng=O.RNG_KEYED, prune=True)
    assert np.isfinite(a).all() and np.isfinite(b).all()
    assert np.abs(a - b).mean() > 1e-3 * np.abs(b).mean()


@pytest.mark.gpu
def test_gltf_textured_scene_renders_like_the_in_memory_scene(tmp_path):
    from crystalgraphics_b200 import gltf
    s = scenes.textured_cornell()
    path = gltf.write(s, str(tmp_path / "t.gltf"))
    B.EnvInit(B.PathTraceConf(render_width=48, render_height=48, sample_count=2, trace_depth=3))
    cam = B.Camera.from_c(s.camera)
    g = B.LoadScene(s)
    B.View(g, cam)
    a = B.ReadFilm()
    gl = B.LoadScene(path)
    B.View(gl, cam)
    b = B.ReadFilm()
    scale = max(float(np.abs(a).mean()), 1e-6)
    assert float(np.abs(a - b).max()) / scale < 1e-4
    B.EnvTerm()
