"""The C ABI: the library loads, exports every declared entry point, and its
host-side logic (argument checks, scene validation, alias tables) works
without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from crystalgraphics_b200 import _abi, scenes
from crystalgraphics_b200 import backend as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"CG_API\s+[\w\s\*]+?\b(cg_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_symbols()
    for required in ("cg_init", "cg_term", "cg_scene_create", "cg_scene_destroy", "cg_view",
                     "cg_film_read", "cg_last_error", "cg_batch_render", "cg_server_submit",
                     "cg_trace_closest"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(B.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_reference_sizes():
    # Camera 48 B (camera.h), Vertex 48 B (vertex.h), EmissivePrim 80 B and
    # AliasTableEntry 8 B (emissive_buffer.h, alias_table.h)
    assert C.sizeof(_abi.CgCamera) == 48
    assert _abi.VERTEX_DTYPE.itemsize == 48
    assert _abi.EMISSIVE_DTYPE.itemsize == 80
    assert _abi.ALIAS_DTYPE.itemsize == 8


# ctypes mirror -> C struct of include/cg_cuda.h
_MIRRORS = {"CgConf": "cg_conf", "CgCamera": "cg_camera", "CgSceneDesc": "cg_scene_desc",
            "CgTexture": "cg_texture", "CgSceneInfo": "cg_scene_info", "CgHit": "cg_hit",
            "CgStats": "cg_stats", "CgProfile": "cg_profile", "CgViewDesc": "cg_view_desc",
            "CgTuning": "cg_tuning", "CgRequest": "cg_request",
            "CgRequestResult": "cg_request_result", "CgServerStats": "cg_server_stats"}


def test_ctypes_mirrors_match_the_header(tmp_path):
    """Every ctypes structure has the size and field offsets of its C struct
    (compiled against include/cg_cuda.h with the host C compiler)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    inc = os.path.join(ROOT, "include")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cg_cuda.h"', 'int main(void) {']
    for py, c in _MIRRORS.items():
        lines.append(f'  printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in getattr(_abi, py)._fields_:
            lines.append(f'  printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "sizes.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "sizes"
    subprocess.run([cc, "-std=c11", "-I", inc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    bad = []
    for line in out.splitlines():
        py, field, value = line.split()
        cls = getattr(_abi, py)
        got = C.sizeof(cls) if field == "size" else getattr(cls, field).offset
        if got != int(value):
            bad.append((py, field, got, int(value)))
    assert not bad, bad


def test_calls_without_init_fail_with_reference_message():
    if B.EnvStatus():
        pytest.skip("environment initialised by another test")
    cam = _abi.make_camera((0, 0, 0), (1, 0, 0), (0.5, 0.5))
    rc = B.lib.cg_view(C.c_void_p(1), C.byref(cam))
    assert rc == _abi.CG_E_NOT_INIT
    assert B.lib.cg_last_error().decode() == "Environment not initialized."
    with pytest.raises(B.Error):
        B.ReadFilm()


def test_null_arguments_are_rejected():
    assert B.lib.cg_init(None, 0) == _abi.CG_E_INVALID
    assert B.lib.cg_scene_create(None, None) == _abi.CG_E_INVALID
    assert B.lib.cg_alias_build(None, 3, None) == _abi.CG_E_INVALID
    assert B.lib.cg_term() == _abi.CG_OK  # safe when not initialised


def _desc_of(scene):
    return scene.desc()


def test_scene_validation_runs_on_the_host():
    s = scenes.cornell()
    bad = scenes.Scene(**{k: getattr(s, k) for k in ("name", "vertices", "indices", "meshes",
                                                      "instances", "materials")})
    bad.instances = bad.instances.copy()
    bad.instances["mesh"][0] = 999
    with pytest.raises(B.Error, match="missing mesh"):
        B.LoadScene(bad)
    tex = scenes.Scene(**{k: getattr(s, k) for k in ("name", "vertices", "indices", "meshes",
                                                      "instances", "materials")})
    tex.materials = tex.materials.copy()
    tex.materials["base_color_texture"][0] = 0
    with pytest.raises(B.Error, match="texture"):
        B.LoadScene(tex)
    idx = scenes.Scene(**{k: getattr(s, k) for k in ("name", "vertices", "indices", "meshes",
                                                      "instances", "materials")})
    idx.indices = idx.indices.copy()
    idx.indices[0] = 10_000_000
    with pytest.raises(B.Error, match="index beyond"):
        B.LoadScene(idx)


def test_alias_build_matches_reference_golden():
    g = np.load(os.path.join(ROOT, "tests", "golden", "alias_tables.npz"))
    names = sorted({k.split("__")[0] for k in g.files})
    assert len(names) >= 8
    for name in names:
        w = g[f"{name}__w"]
        out = B.alias_build(w)
        np.testing.assert_array_equal(out["alias"], g[f"{name}__alias"], err_msg=name)
        assert out["prob"].tobytes() == g[f"{name}__prob"].tobytes(), name


def test_version_string():
    assert b"sm_100a" in B.lib.cg_version()


def test_spectral_and_roulette_settings_check_their_arguments():
    """Hero-wavelength mode and Russian roulette are environment settings:
    an unknown mode or a start depth beyond the depth cap is rejected, and
    without an environment the calls report it (no device is needed)."""
    assert B.lib.cg_set_spectral(7) == _abi.CG_E_INVALID
    assert B.lib.cg_set_roulette(65) == _abi.CG_E_INVALID
    if not B.EnvStatus():
        assert B.lib.cg_set_spectral(_abi.CG_SPECTRAL_HERO) == _abi.CG_E_NOT_INIT
        assert B.lib.cg_set_roulette(3) == _abi.CG_E_NOT_INIT
