"""ctypes wrapper of the CPU oracle (oracle/_build/libcg_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, bench.py's CPU arms and
__graft_entry__.smoke() as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libcg_oracle.so")
REF_ALIAS_PATH = os.path.join(HERE, "_ref", "libref_alias.so")

RNG_REFERENCE = 0
RNG_KEYED = 1
SPECTRAL_REFERENCE = 0
SPECTRAL_HERO = 1


def reference_dir() -> str | None:
    """The reference source tree: $CG_REFERENCE when set, else a `reference`
    directory beside this repository's; None when neither holds its
    src/pathtracing/."""
    for d in (os.environ.get("CG_REFERENCE"),
              os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")):
        if d and os.path.isdir(os.path.join(d, "src", "pathtracing")):
            return os.path.abspath(d)
    return None


def build(reference: bool = True) -> None:
    """Compiles the oracle (and, when the reference tree is present, the
    reference's own alias_table.h into _ref/)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref = reference_dir() if reference else None
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE={ref}"], check=True)


def use_native() -> bool:
    """Switches this process to the oracle built for its own CPU
    (-march=native, `make native`), building it if needed; for the timed CPU
    baselines.  Must come before the first oracle call.  Returns False (and
    keeps the portable build) if the native build fails."""
    global LIB_PATH, _lib
    native = os.path.join(HERE, "_build", "libcg_oracle_native.so")
    try:
        subprocess.run(["make", "-s", "-C", HERE, "native"], check=True, timeout=300,
                       capture_output=True)
    except (subprocess.SubprocessError, OSError):
        return False
    if _lib is None and os.path.exists(native):
        LIB_PATH = native
        return True
    return LIB_PATH == native


def _abi():
    import sys
    root = os.path.dirname(HERE)
    if root not in sys.path:
        sys.path.insert(0, root)
    from crystalgraphics_b200 import _abi as abi
    return abi


class RenderArgs(C.Structure):
    pass


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build(reference=False)
    abi = _abi()
    RenderArgs._fields_ = [("conf", abi.CgConf), ("camera", abi.CgCamera),
                           ("iter_count", C.c_uint32), ("rng_mode", C.c_uint32),
                           ("seed", C.c_uint32), ("threads", C.c_uint32), ("prune", C.c_uint32),
                           ("pixel_begin", C.c_uint32), ("pixel_end", C.c_uint32),
                           ("spectral", C.c_uint32), ("roulette", C.c_uint32),
                           ("_pad", C.c_uint32)]
    L = C.CDLL(LIB_PATH)
    L.oracle_scene_create.restype = C.c_void_p
    L.oracle_scene_create.argtypes = [C.POINTER(abi.CgSceneDesc)]
    L.oracle_scene_destroy.argtypes = [C.c_void_p]
    L.oracle_scene_pack_seconds.argtypes = [C.c_void_p, C.c_void_p]
    L.oracle_emissive_count.restype = C.c_uint32
    L.oracle_emissive_count.argtypes = [C.c_void_p]
    L.oracle_emissive.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_float)]
    L.oracle_alias_build.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    L.oracle_trace_closest.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                       C.c_void_p, C.c_int]
    L.oracle_render.argtypes = [C.c_void_p, C.POINTER(RenderArgs), C.c_void_p, C.c_void_p,
                                C.c_void_p]
    L.oracle_sample_wavelength.restype = C.c_float
    L.oracle_sample_wavelength.argtypes = [C.c_float, C.POINTER(C.c_float)]
    L.oracle_xyz_match.argtypes = [C.c_float, C.c_void_p]
    L.oracle_rgb_to_reflectance.restype = C.c_float
    L.oracle_rgb_to_reflectance.argtypes = [C.c_void_p, C.c_float]
    L.oracle_rgb_to_radiance.restype = C.c_float
    L.oracle_rgb_to_radiance.argtypes = [C.c_void_p, C.c_float]
    L.oracle_xyz_to_srgb.argtypes = [C.c_void_p, C.c_void_p]
    L.oracle_rng_sequence.restype = C.c_uint32
    L.oracle_rng_sequence.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p]
    L.oracle_sample_key.restype = C.c_uint32
    L.oracle_sample_key.argtypes = [C.c_uint32] * 4
    _lib = L
    return L


class OracleScene:
    def __init__(self, scene):
        self.scene = scene
        self._desc = scene.desc()
        self.h = lib().oracle_scene_create(C.byref(self._desc))
        if not self.h:
            raise RuntimeError("oracle_scene_create failed")

    def close(self):
        if self.h:
            lib().oracle_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pack_seconds(self) -> dict:
        """Single-threaded seconds of the host packing stages the create call
        ran, as the reference runs them on the host: median-split BLAS builds,
        TLAS build, emissive buffer, alias table."""
        out = np.zeros(4, np.float64)
        assert lib().oracle_scene_pack_seconds(self.h, out.ctypes.data) == 0
        return dict(zip(("blas", "tlas", "emissive", "alias"), map(float, out)))

    def emissive(self):
        abi = _abi()
        n = lib().oracle_emissive_count(self.h)
        prims = np.zeros(n, abi.EMISSIVE_DTYPE)
        alias = np.zeros(n, abi.ALIAS_DTYPE)
        total = C.c_float()
        lib().oracle_emissive(self.h, prims.ctypes.data, alias.ctypes.data, C.byref(total))
        return prims, alias, total.value

    def trace_closest(self, rays: np.ndarray, threads: int = 0):
        abi = _abi()
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hits = np.zeros(len(rays), abi.HIT_DTYPE)
        t2 = np.zeros(len(rays), np.float32)
        rc = lib().oracle_trace_closest(self.h, rays.ctypes.data, len(rays), hits.ctypes.data,
                                        t2.ctypes.data, threads)
        assert rc == 0
        return hits, t2

    def render(self, conf, camera, film=None, seeds=None, iter_count=0, rng=RNG_KEYED, seed=0,
               threads=0, prune=False, pixel_range=None, spectral=SPECTRAL_REFERENCE,
               roulette=0):
        W, H = conf.render_width, conf.render_height
        if film is None:
            film = np.zeros((H, W, 3), np.float32)
        if seeds is None:
            seeds = np.zeros((H, W), np.uint32)
        a = RenderArgs()
        a.conf = conf
        a.camera = camera
        a.iter_count = iter_count
        a.rng_mode = rng
        a.seed = seed
        a.threads = threads
        a.prune = 1 if prune else 0
        a.spectral = spectral
        a.roulette = roulette
        if pixel_range is not None:
            a.pixel_begin, a.pixel_end = pixel_range
        stats = np.zeros(5, np.uint64)
        rc = lib().oracle_render(self.h, C.byref(a), film.ctypes.data, seeds.ctypes.data,
                                 stats.ctypes.data)
        assert rc == 0
        return film, seeds, stats


def alias_build(weights):
    abi = _abi()
    w = np.ascontiguousarray(weights, np.float64)
    out = np.zeros(len(w), abi.ALIAS_DTYPE)
    assert lib().oracle_alias_build(w.ctypes.data, len(w), out.ctypes.data) == 0
    return out


def ref_alias_available() -> bool:
    return os.path.exists(REF_ALIAS_PATH)


def ref_alias_build(weights):
    """The reference's own AliasTable (alias_table.h), compiled unmodified."""
    abi = _abi()
    L = C.CDLL(REF_ALIAS_PATH)
    L.ref_alias_build_raw.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    w = np.ascontiguousarray(weights, np.float64)
    out = np.zeros(len(w), abi.ALIAS_DTYPE)
    n = L.ref_alias_build_raw(w.ctypes.data, len(w), out.ctypes.data)
    assert n == len(w)
    return out


def xyz_to_srgb8(xyz: np.ndarray) -> np.ndarray:
    """luminanceToSrgb + rgba8unorm store (physics/srgb.wesl:5-27)."""
    flat = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    out = np.zeros_like(flat)
    L = lib()
    for i in range(len(flat)):
        L.oracle_xyz_to_srgb(flat[i].ctypes.data, out[i].ctypes.data)
    return np.rint(out * 255.0).astype(np.uint8).reshape(xyz.shape)
