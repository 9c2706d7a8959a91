"""Python mirror of the reference's ``crystal::graphics`` API over libcg_cuda.so.

The reference's public API (include/CrystalGraphics/*.h) returns
``std::expected<..., Error>`` with ``Error = std::string``; here the same
calls raise :class:`Error` with that message.  Names, argument meaning and
defaults follow the reference:

  EnvInit(conf=PathTraceConf())   environment.h:20     (CUDA context, film)
  EnvTerm(), EnvPoll(), EnvPresent(), EnvStatus()      (Poll/Present are
                                  headless no-ops: there is no window)
  LoadScene(scene)                scene.h:37           (uploads once)
  View(scene, camera=Camera())    api.h:13             (one progressive frame)

plus what the headless backend adds: ``ReadFilm`` (explicit readback instead
of EnvPresent), ``batch_render`` (the batched form), ``Server`` (the served
form), ``trace_closest`` (the closest-hit query the parity tests use).

There is no CPU fallback: if libcg_cuda.so is missing this module raises on
import, and every call that needs a GPU raises when there is none.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import _abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libcg_cuda.so")


class Error(RuntimeError):
    """The reference's ``Error`` (a string), raised instead of returned."""

    def __init__(self, message: str, code: int = 0):
        super().__init__(message)
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m crystalgraphics_b200.build` "
                          "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    i, u32, vp = C.c_int, C.c_uint32, C.c_void_p
    sig = {
        "cg_init": (i, [C.POINTER(_abi.CgConf), i]),
        "cg_term": (i, []),
        "cg_status": (i, []),
        "cg_last_error": (C.c_char_p, []),
        "cg_get_conf": (i, [C.POINTER(_abi.CgConf)]),
        "cg_scene_create": (i, [C.POINTER(_abi.CgSceneDesc), C.POINTER(vp)]),
        "cg_scene_destroy": (i, [vp]),
        "cg_scene_load_gltf": (i, [C.c_char_p, C.POINTER(vp)]),
        "cg_gltf_parse": (i, [C.c_char_p, C.POINTER(_abi.CgSceneDesc), C.POINTER(vp)]),
        "cg_gltf_free": (i, [vp]),
        "cg_scene_get_info": (i, [vp, C.POINTER(_abi.CgSceneInfo)]),
        "cg_scene_read_emissive": (i, [vp, vp, vp, u32, C.POINTER(u32)]),
        "cg_alias_build": (i, [vp, u32, vp]),
        "cg_view": (i, [vp, C.POINTER(_abi.CgCamera)]),
        "cg_film_read": (i, [vp, C.c_size_t, i]),
        "cg_view_samples": (i, [vp, C.POINTER(_abi.CgCamera), u32, u32]),
        "cg_film_device": (i, [C.POINTER(vp), C.POINTER(C.c_size_t)]),
        "cg_film_update_rgba8": (i, []),
        "cg_film_frames": (i, [C.POINTER(u32)]),
        "cg_last_stats": (i, [C.POINTER(_abi.CgStats)]),
        "cg_set_counting": (i, [i]),
        "cg_set_seed": (i, [u32]),
        "cg_set_spectral": (i, [i]),
        "cg_set_roulette": (i, [u32]),
        "cg_get_spectral": (i, [C.POINTER(C.c_int)]),
        "cg_set_profiling": (i, [i]),
        "cg_profile_read": (i, [C.POINTER(_abi.CgProfile)]),
        "cg_trace_closest": (i, [vp, vp, u32, vp]),
        "cg_batch_render": (i, [vp, vp, u32, vp, vp]),
        "cg_set_tuning": (i, [C.POINTER(_abi.CgTuning)]),
        "cg_get_tuning": (i, [C.POINTER(_abi.CgTuning)]),
        "cg_autotune": (i, [vp, C.POINTER(_abi.CgViewDesc), C.POINTER(_abi.CgTuning)]),
        "cg_autotune_views": (i, [vp, vp, u32, C.POINTER(_abi.CgTuning)]),
        "cg_set_bvh_build": (i, [i]),
        "cg_png_decode": (i, [vp, C.c_size_t, C.POINTER(u32), C.POINTER(u32), vp]),
        "cg_hdr_decode": (i, [vp, C.c_size_t, C.POINTER(u32), C.POINTER(u32), vp]),
        "cg_jpeg_decode": (i, [vp, C.c_size_t, C.POINTER(u32), C.POINTER(u32), vp]),
        "cg_env_from_cube": (i, [vp, u32, u32, vp, vp]),
        "cg_bvh_build": (i, [vp, u32, i, vp, u32, C.POINTER(u32), vp]),
        "cg_server_create": (i, [vp, u32, C.c_uint64, C.POINTER(vp)]),
        "cg_server_destroy": (i, [vp]),
        "cg_server_submit": (i, [vp, C.POINTER(_abi.CgRequest), vp, C.POINTER(C.c_uint64)]),
        "cg_server_wait": (i, [vp, C.c_uint64, i, C.POINTER(_abi.CgRequestResult)]),
        "cg_server_cancel": (i, [vp, C.c_uint64]),
        "cg_server_get_stats": (i, [vp, C.POINTER(_abi.CgServerStats)]),
        "cg_version": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


lib = _load()


def _check(rc: int):
    if rc != _abi.CG_OK:
        raise Error(lib.cg_last_error().decode(errors="replace"), rc)


# ---- configuration / camera -------------------------------------------------------
@dataclass
class PathTraceConf:
    """include/CrystalGraphics/environment.h:11-18 (same defaults)."""
    window_width: int = 1920
    window_height: int = 1080
    render_width: int = 1280
    render_height: int = 720
    sample_count: int = 1
    trace_depth: int = 2
    max_transport_sample_count: int = 3
    max_diffuse_sample_count: int = 1
    max_rough_sample_count: int = 1
    max_emission_sample_count: int = 1

    def to_c(self) -> _abi.CgConf:
        return _abi.CgConf(self.window_width, self.window_height, self.render_width,
                           self.render_height, self.sample_count, self.trace_depth,
                           self.max_transport_sample_count, self.max_diffuse_sample_count,
                           self.max_rough_sample_count, self.max_emission_sample_count)


@dataclass
class Camera:
    """include/CrystalGraphics/camera.h:9-13 (same defaults)."""
    position: tuple = (0.0, 0.0, 0.0)
    direction: tuple = (1.0, 0.0, 0.0)
    viewport: tuple = (0.5, 0.5)

    def to_c(self) -> _abi.CgCamera:
        return _abi.make_camera(self.position, self.direction, self.viewport)

    @staticmethod
    def from_c(c: _abi.CgCamera) -> "Camera":
        return Camera(tuple(c.position), tuple(c.direction), tuple(c.viewport))


# ---- environment ------------------------------------------------------------------------
def EnvInit(conf: PathTraceConf | None = None, device: int = 0) -> None:
    conf = conf or PathTraceConf()
    c = conf.to_c()
    _check(lib.cg_init(C.byref(c), device))


def EnvTerm() -> None:
    _check(lib.cg_term())


def EnvPoll() -> None:
    """Headless: there is no window event loop to poll."""
    if not EnvStatus():
        raise Error("Environment not initialized.", _abi.CG_E_NOT_INIT)


def EnvPresent() -> None:
    """Headless: there is no swap chain; read the film with ReadFilm()."""
    if not EnvStatus():
        raise Error("Environment not initialized.", _abi.CG_E_NOT_INIT)


def EnvStatus() -> bool:
    return lib.cg_status() == 1


def GetConf() -> PathTraceConf:
    c = _abi.CgConf()
    _check(lib.cg_get_conf(C.byref(c)))
    return PathTraceConf(*[getattr(c, f) for f, _ in _abi.CgConf._fields_])


# ---- scenes -------------------------------------------------------------------------------
class Scene:
    """An uploaded scene (crystal::graphics::Scene, move-only in the reference)."""

    def __init__(self, handle: int, source):
        self._h = handle
        self.source = source

    def FilePath(self):
        if isinstance(self.source, str):
            return self.source
        return getattr(self.source, "name", "")

    @property
    def handle(self) -> int:
        if not self._h:
            raise Error("scene was destroyed", _abi.CG_E_INVALID)
        return self._h

    def info(self) -> _abi.CgSceneInfo:
        out = _abi.CgSceneInfo()
        _check(lib.cg_scene_get_info(self.handle, C.byref(out)))
        return out

    def emissive(self):
        n = C.c_uint32()
        _check(lib.cg_scene_read_emissive(self.handle, None, None, 0, C.byref(n)))
        prims = np.zeros(n.value, _abi.EMISSIVE_DTYPE)
        alias = np.zeros(n.value, _abi.ALIAS_DTYPE)
        if n.value:
            _check(lib.cg_scene_read_emissive(self.handle, prims.ctypes.data, alias.ctypes.data,
                                              n.value, C.byref(n)))
        return prims, alias

    def close(self):
        if self._h:
            lib.cg_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def LoadScene(scene) -> Scene:
    """Uploads a scene.  `scene` is an in-memory description
    (crystalgraphics_b200.scenes.Scene) or a path to a .gltf file."""
    if isinstance(scene, (str, os.PathLike)):
        h = C.c_void_p()
        _check(lib.cg_scene_load_gltf(os.fspath(scene).encode(), C.byref(h)))
        return Scene(h.value, os.fspath(scene))
    desc = scene.desc()
    h = C.c_void_p()
    _check(lib.cg_scene_create(C.byref(desc), C.byref(h)))
    return Scene(h.value, scene)


def jpeg_decode(data: bytes) -> np.ndarray:
    """A JPEG image as (height, width, 4) uint8 RGBA (alpha 255)."""
    buf = np.frombuffer(data, np.uint8)
    w, h = C.c_uint32(), C.c_uint32()
    _check(lib.cg_jpeg_decode(buf.ctypes.data, buf.size, C.byref(w), C.byref(h), None))
    out = np.empty((h.value, w.value, 4), np.uint8)
    _check(lib.cg_jpeg_decode(buf.ctypes.data, buf.size, C.byref(w), C.byref(h), out.ctypes.data))
    return out


def hdr_decode(data: bytes) -> np.ndarray:
    """A Radiance .hdr image as (height, width, 4) float32 RGBA (alpha 1)."""
    buf = np.frombuffer(data, np.uint8)
    w, h = C.c_uint32(), C.c_uint32()
    _check(lib.cg_hdr_decode(buf.ctypes.data, buf.size, C.byref(w), C.byref(h), None))
    out = np.empty((h.value, w.value, 4), np.float32)
    _check(lib.cg_hdr_decode(buf.ctypes.data, buf.size, C.byref(w), C.byref(h), out.ctypes.data))
    return out


def env_from_cube(faces: np.ndarray, rotation=(0.0, 0.0, 0.0, 1.0)) -> np.ndarray:
    """The lat-long environment (2h, 4w, 4) of six (h, w, 4) float32 cube faces
    (+X, -X, +Y, -Y, +Z, -Z) seen through the quaternion `rotation` (x, y, z, w)."""
    f = np.ascontiguousarray(faces, np.float32)
    assert f.ndim == 4 and f.shape[0] == 6 and f.shape[3] == 4
    h, w = f.shape[1], f.shape[2]
    q = np.ascontiguousarray(rotation, np.float32)
    out = np.empty((2 * h, 4 * w, 4), np.float32)
    _check(lib.cg_env_from_cube(f.ctypes.data, w, h, q.ctypes.data, out.ctypes.data))
    return out


def parse_gltf(path) -> "scenes.Scene":
    """Parses a glTF file with the native loader (no device needed) into an
    in-memory scene description (copies)."""
    from . import scenes
    d = _abi.CgSceneDesc()
    st = C.c_void_p()
    _check(lib.cg_gltf_parse(os.fspath(path).encode(), C.byref(d), C.byref(st)))
    try:
        def arr(ptr, n, dtype):
            if n == 0:
                return np.zeros(0, dtype)
            buf = (C.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr)
            return np.frombuffer(buf, dtype=dtype, count=n).copy()
        textures = []
        if d.texture_count:
            tex = (_abi.CgTexture * d.texture_count).from_address(d.textures)
            for t in tex:
                img = arr(t.rgba8, t.width * t.height * 4, np.uint8).reshape(t.height, t.width, 4)
                textures.append((img, int(t.wrap_s), int(t.wrap_t)))
        env = None
        if d.env_rgba32f:
            env = arr(d.env_rgba32f, d.env_width * d.env_height * 4,
                      np.float32).reshape(d.env_height, d.env_width, 4)
        return scenes.Scene(name=os.fspath(path),
                            vertices=arr(d.vertices, d.vertex_count, _abi.VERTEX_DTYPE),
                            indices=arr(d.indices, d.index_count, np.uint32),
                            meshes=arr(d.meshes, d.mesh_count, _abi.MESH_DTYPE),
                            instances=arr(d.instances, d.instance_count, _abi.INSTANCE_DTYPE),
                            materials=arr(d.materials, d.material_count, _abi.MATERIAL_DTYPE),
                            env=env, textures=textures)
    finally:
        lib.cg_gltf_free(st)


def View(scene: Scene, camera: Camera | _abi.CgCamera | None = None) -> None:
    cam = camera if isinstance(camera, _abi.CgCamera) else (camera or Camera()).to_c()
    _check(lib.cg_view(scene.handle, C.byref(cam)))


def ViewSamples(scene: Scene, camera: Camera | _abi.CgCamera | None, sample_begin: int,
                sample_count: int) -> None:
    """Renders samples [sample_begin, sample_begin + sample_count) of every
    pixel (out of the conf's sample_count) as that range's share of the full
    frame's mean (cg_view_samples)."""
    cam = camera if isinstance(camera, _abi.CgCamera) else (camera or Camera()).to_c()
    _check(lib.cg_view_samples(scene.handle, C.byref(cam), int(sample_begin), int(sample_count)))


class _DeviceFilm:
    """The environment's float4 device film as a CUDA array interface."""

    def __init__(self):
        ptr, nbytes = C.c_void_p(), C.c_size_t()
        _check(lib.cg_film_device(C.byref(ptr), C.byref(nbytes)))
        conf = _abi.CgConf()
        _check(lib.cg_get_conf(C.byref(conf)))
        shape = (conf.render_height, conf.render_width, 4)
        assert nbytes.value == 16 * shape[0] * shape[1]
        # the film is complete when a call of this library returns, so the
        # consumer needs no stream synchronisation
        self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f4",
                                         "data": (ptr.value, False), "version": 3,
                                         "strides": None, "stream": None}


def FilmDevice():
    """A torch CUDA tensor (height, width, 4) aliasing the environment's film
    (X, Y, Z, 0 per pixel); valid until the next EnvInit or EnvTerm."""
    import torch
    return torch.as_tensor(_DeviceFilm(), device="cuda")


def UpdateRgba8() -> None:
    """Recomputes the rgba8 film from the (changed) float film."""
    _check(lib.cg_film_update_rgba8())


def sample_range(spp: int, rank: int, world: int) -> tuple[int, int]:
    """(first sample, count) of rank `rank` when `world` ranks split `spp`
    samples per pixel in contiguous, near-equal ranges."""
    begin = spp * rank // world
    return begin, spp * (rank + 1) // world - begin


def sum_films(film, group=None) -> None:
    """Sums a film tensor over the ranks of `group` in place (all-reduce; NCCL
    over NVLink for CUDA tensors) and waits for the result."""
    import torch
    import torch.distributed as dist
    dist.all_reduce(film, op=dist.ReduceOp.SUM, group=group)
    if film.is_cuda:
        torch.cuda.synchronize(film.device)


def ViewSplit(scene: Scene, camera: Camera | _abi.CgCamera | None = None, group=None) -> None:
    """One View() frame (frame 0) spread over the ranks of a torch.distributed
    group, one GPU per rank: each rank renders its range of every pixel's
    samples, then the device films are summed across the ranks, so every rank
    ends with the full frame's film (equal to a one-GPU cg_view frame 0 up to
    float summation order).  The film's running mean restarts."""
    import torch.distributed as dist
    conf = _abi.CgConf()
    _check(lib.cg_get_conf(C.byref(conf)))
    begin, count = sample_range(conf.sample_count, dist.get_rank(group),
                                dist.get_world_size(group))
    ViewSamples(scene, camera, begin, count)
    sum_films(FilmDevice(), group)
    UpdateRgba8()


def partition_views(views, world: int) -> list[list[int]]:
    """Indices of the views each of `world` GPUs renders: longest first, each
    view to the rank with the fewest samples (width * height * spp) so far,
    the lower rank on ties.  Deterministic, so every rank computes the same
    assignment from the same view list with no communication; a view's film
    does not depend on the views it is batched with (its sample streams are
    keyed by its seed, pixel and sample), so each rank's films equal a one-GPU
    batch's."""
    arr = views if isinstance(views, C.Array) else make_views(views)
    work = [int(arr[k].width) * int(arr[k].height) * int(arr[k].spp) for k in range(len(arr))]
    load = [0] * world
    parts = [[] for _ in range(world)]
    for k in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(k)
        load[r] += work[k]
    return [sorted(p) for p in parts]


def BatchSplit(scene: Scene, views, group=None):
    """A batch of views spread over the ranks of a torch.distributed group, one
    GPU per rank, with no collective: this rank renders its share
    (partition_views) in one wavefront.  Returns (view indices, films) of this
    rank's share; the shares of all ranks cover every view exactly once."""
    import torch.distributed as dist
    arr = views if isinstance(views, C.Array) else make_views(views)
    mine = partition_views(arr, dist.get_world_size(group))[dist.get_rank(group)]
    if not mine:
        return [], []
    sub = (_abi.CgViewDesc * len(mine))(*[arr[k] for k in mine])
    return mine, batch_render(scene, sub)


class RequestRouter:
    """Routes a request stream over `world` GPUs, each running its own Server,
    with no communication: every rank sees the same stream and routes request
    k to the rank with the fewest samples routed so far (the lower rank on
    ties), so all ranks agree on every request's owner and the work stays
    balanced to within one request."""

    def __init__(self, world: int):
        self.world = world
        self.load = [0] * world

    def route(self, width: int, height: int, spp: int) -> int:
        r = min(range(self.world), key=lambda r: (self.load[r], r))
        self.load[r] += int(width) * int(height) * int(spp)
        return r


def ReadFilm(fmt: int = _abi.CG_FILM_XYZ32F, out: np.ndarray | None = None) -> np.ndarray:
    conf = _abi.CgConf()
    _check(lib.cg_get_conf(C.byref(conf)))
    W, H = conf.render_width, conf.render_height
    if fmt == _abi.CG_FILM_RGBA8:
        shape, dtype = (H, W, 4), np.uint8
    else:
        shape, dtype = (H, W, 3), np.float32
    if out is None:
        out = np.empty(shape, dtype)
    assert out.shape == shape and out.dtype == dtype and out.flags["C_CONTIGUOUS"]
    _check(lib.cg_film_read(out.ctypes.data, out.nbytes, fmt))
    return out


def FilmFrames() -> int:
    n = C.c_uint32()
    _check(lib.cg_film_frames(C.byref(n)))
    return n.value


def LastStats() -> _abi.CgStats:
    s = _abi.CgStats()
    _check(lib.cg_last_stats(C.byref(s)))
    return s


def SetCounting(enable: bool) -> None:
    _check(lib.cg_set_counting(1 if enable else 0))


def SetProfiling(enable: bool) -> None:
    _check(lib.cg_set_profiling(1 if enable else 0))


def ReadProfile() -> dict:
    """Per-kernel device time (ms) and launch counts since the last read."""
    p = _abi.CgProfile()
    _check(lib.cg_profile_read(C.byref(p)))
    names = ("gen", "extend", "shade", "shadow", "resolve")
    return {n: (p.ms[k], p.launches[k]) for k, n in enumerate(names)}


def SetSeed(seed: int) -> None:
    _check(lib.cg_set_seed(seed))


def SetSpectral(mode: int) -> None:
    """_abi.CG_SPECTRAL_REFERENCE (the reference's one wavelength per sample)
    or _abi.CG_SPECTRAL_HERO (four wavelengths per sample)."""
    _check(lib.cg_set_spectral(mode))


def SetRoulette(start_depth: int) -> None:
    """Russian roulette for child rays spawned at hits of depth >= start_depth
    (0 = off, as the reference)."""
    _check(lib.cg_set_roulette(start_depth))


def GetSpectral() -> int:
    m = C.c_int()
    _check(lib.cg_get_spectral(C.byref(m)))
    return m.value


def SetTuning(queue_capacity=0, extend_block=0, shade_block=0, use_graph=1, bvh_width=0,
              persistent=None, shade_sort=None, box_bits=0, pipelines=0,
              traversal_threads=0) -> None:
    """0 (or None for the two switches) keeps the current value.  shade_sort:
    True / "global" (level-wide sort by material kind), "block" (per block),
    False / "none".  persistent: True (persistent warps), False (one ray per
    thread) or "postponed" (persistent, with postponed leaves)."""
    if shade_sort is None:
        sort = 0
    elif isinstance(shade_sort, str):
        sort = {"global": 1, "none": 2, "block": 3}[shade_sort]
    else:
        sort = 1 if shade_sort else 2
    t = _abi.CgTuning(queue_capacity, extend_block, shade_block, use_graph, bvh_width,
                      0 if persistent is None else
                      (3 if persistent == "postponed" else 1 if persistent else 2), sort, box_bits,
                      pipelines, traversal_threads)
    _check(lib.cg_set_tuning(C.byref(t)))


def SetBvhBuild(mode: int) -> None:
    """Where LoadScene builds BVHs: _abi.CG_BVH_BUILD_AUTO (GPU for large trees),
    CG_BVH_BUILD_HOST or CG_BVH_BUILD_DEVICE."""
    _check(lib.cg_set_bvh_build(mode))


def png_decode(data: bytes) -> np.ndarray:
    """A PNG file image as an (h, w, 4) uint8 RGBA array."""
    buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
    w, h = C.c_uint32(), C.c_uint32()
    _check(lib.cg_png_decode(buf, len(data), C.byref(w), C.byref(h), None))
    out = np.empty((h.value, w.value, 4), np.uint8)
    _check(lib.cg_png_decode(buf, len(data), C.byref(w), C.byref(h), out.ctypes.data))
    return out


def bvh_build(boxes: np.ndarray, mode: int):
    """One BVH over (n, 6) float32 boxes built on the host (1) or the GPU (2):
    returns (nodes as (m, 16) uint32 words of the 64-byte records, order)."""
    boxes = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
    n = boxes.shape[0]
    order = np.empty(n, np.uint32)
    cnt = C.c_uint32()
    _check(lib.cg_bvh_build(boxes.ctypes.data, n, mode, None, 0, C.byref(cnt), order.ctypes.data))
    nodes = np.empty((cnt.value, 16), np.uint32)
    _check(lib.cg_bvh_build(boxes.ctypes.data, n, mode, nodes.ctypes.data, cnt.value, C.byref(cnt),
                            order.ctypes.data))
    return nodes, order


def GetTuning() -> _abi.CgTuning:
    t = _abi.CgTuning()
    _check(lib.cg_get_tuning(C.byref(t)))
    return t


def trace_closest(scene: Scene, rays: np.ndarray) -> np.ndarray:
    """Closest hits of world rays (n x 8 floats: o, _, d, _)."""
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    hits = np.zeros(len(rays), _abi.HIT_DTYPE)
    _check(lib.cg_trace_closest(scene.handle, rays.ctypes.data, len(rays), hits.ctypes.data))
    return hits


def alias_build(weights) -> np.ndarray:
    w = np.ascontiguousarray(weights, np.float64)
    out = np.zeros(len(w), _abi.ALIAS_DTYPE)
    _check(lib.cg_alias_build(w.ctypes.data, len(w), out.ctypes.data))
    return out


# ---- batched form -----------------------------------------------------------------------
def make_views(views) -> "C.Array":
    """views: iterable of (position, direction, width, height, spp, seed[, viewport])."""
    views = list(views)
    arr = (_abi.CgViewDesc * len(views))()
    for k, v in enumerate(views):
        pos, d, w, h, spp, seed = v[:6]
        vp = v[6] if len(v) > 6 else (0.5 * w / h, 0.5)
        arr[k].camera = _abi.make_camera(pos, d, vp)
        arr[k].width, arr[k].height, arr[k].spp, arr[k].seed = w, h, spp, seed
    return arr


def batch_render(scene: Scene, views, rgba: bool = False):
    """Renders many views in one wavefront.  Returns a list of (h, w, 3) XYZ
    films (and rgba8 films if asked)."""
    arr = views if isinstance(views, C.Array) else make_views(views)
    n = len(arr)
    sizes = [(arr[k].height, arr[k].width) for k in range(n)]
    total = sum(h * w for h, w in sizes)
    xyz = np.empty(total * 3, np.float32)
    rgb8 = np.empty(total * 4, np.uint8) if rgba else None
    _check(lib.cg_batch_render(scene.handle, arr, n, xyz.ctypes.data,
                               rgb8.ctypes.data if rgba else None))
    films, films8, off = [], [], 0
    for h, w in sizes:
        films.append(xyz[off * 3:(off + h * w) * 3].reshape(h, w, 3))
        if rgba:
            films8.append(rgb8[off * 4:(off + h * w) * 4].reshape(h, w, 4))
        off += h * w
    return (films, films8) if rgba else films


def autotune(scene: Scene, view) -> _abi.CgTuning:
    arr = make_views([view])
    best = _abi.CgTuning()
    _check(lib.cg_autotune(scene.handle, C.byref(arr[0]), C.byref(best)))
    return best


def autotune_views(scene: Scene, views) -> _abi.CgTuning:
    """The autotuner timed on several probe views (e.g. a sample of a batch)."""
    arr = views if isinstance(views, C.Array) else make_views(views)
    best = _abi.CgTuning()
    _check(lib.cg_autotune_views(scene.handle, arr, len(arr), C.byref(best)))
    return best


# ---- served form ------------------------------------------------------------------------------
class Server:
    """Continuous-batching request loop over resident scenes."""

    def __init__(self, scenes, hbm_budget_bytes: int):
        self.scenes = list(scenes)
        arr = (C.c_void_p * len(self.scenes))(*[s.handle for s in self.scenes])
        h = C.c_void_p()
        _check(lib.cg_server_create(arr, len(self.scenes), hbm_budget_bytes, C.byref(h)))
        self._h = h.value
        self._films = {}

    def submit(self, scene_index, position, direction, width, height, spp, seed=0, viewport=None,
               out: np.ndarray | None = None):
        """Queues a request; its XYZ film lands in `out` (a C-contiguous
        (height, width, 3) float32 array that a caller may reuse across
        requests) or in a new array.  Returns the request id."""
        req = _abi.CgRequest()
        req.scene = scene_index
        vp = viewport or (0.5 * width / height, 0.5)
        req.view.camera = _abi.make_camera(position, direction, vp)
        req.view.width, req.view.height, req.view.spp, req.view.seed = width, height, spp, seed
        if out is None:
            film = np.empty((height, width, 3), np.float32)
        else:
            assert out.shape == (height, width, 3) and out.dtype == np.float32 \
                and out.flags["C_CONTIGUOUS"]
            film = out
        rid = C.c_uint64()
        _check(lib.cg_server_submit(self._h, C.byref(req), film.ctypes.data, C.byref(rid)))
        self._films[rid.value] = film
        return rid.value

    def wait(self, rid, timeout_ms=-1):
        res = _abi.CgRequestResult()
        rc = lib.cg_server_wait(self._h, rid, timeout_ms, C.byref(res))
        if rc == _abi.CG_E_TIMEOUT:
            raise Error(lib.cg_last_error().decode(), rc)
        film = self._films.pop(rid, None)
        _check(rc)
        return film, res

    def cancel(self, rid):
        _check(lib.cg_server_cancel(self._h, rid))

    def stats(self) -> _abi.CgServerStats:
        s = _abi.CgServerStats()
        _check(lib.cg_server_get_stats(self._h, C.byref(s)))
        return s

    def close(self):
        if self._h:
            lib.cg_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
