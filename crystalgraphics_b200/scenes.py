"""Seeded synthetic scenes: the benchmark workloads of the View() path.

The reference validates on Khronos glTF sample scenes that are not available
here; these generators stand in for them with the shapes, sizes and value
distributions of the benchmark configurations:

  cornell()        256^2, 1 spp, depth 2: five walls, a diffuse box, a
                   conductor box, a 0.25 x 0.25 ceiling light of radiance 15.
  icosphere_scene() 1280x720, 16 spp, depth 8: icosphere subdivided 8 times
                   (1,310,720 triangles) displaced by 3-octave value noise,
                   a dispersive rough dielectric, a diffuse ground, 64
                   emissive triangles of log-uniform radiance in [1, 100].
  instanced_scene() 1920x1080, 64 spp, depth 12: 8 noise-displaced sphere /
                   torus meshes (10k-200k triangles), 4096 instances, a
                   40/30/20/10 material mix, 10,000 emissive triangles with
                   log-normal(0, 2) radiance.
  batch_views(), request_stream(): the 256-view batch and the serving mix.

Material conventions follow glTF (the reference's loader,
src/scene.cpp:711-815): a "diffuse" material is metallic 0, roughness 1,
ior 1.5; roughness is glTF roughness (alpha = roughness^2).  Materials are
per instance (src/pathtracing/instance.h:15), so every emissive triangle with
its own radiance is its own one-triangle instance.

All arrays use the record layouts of include/cg_cuda.h.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi

# Cauchy A = 1.5, B = 0.0042 um^2 expressed as the glTF ior/dispersion pair the
# reference's dispersedIor (shading/material.wesl:80-97) consumes.
CAUCHY_IOR = 1.5121656
CAUCHY_DISPERSION = 0.313201


@dataclass
class Scene:
    """A scene description in host memory (the input of LoadScene)."""
    name: str
    vertices: np.ndarray
    indices: np.ndarray
    meshes: np.ndarray
    instances: np.ndarray
    materials: np.ndarray
    env: np.ndarray | None = None
    camera: object = None
    conf: dict = field(default_factory=dict)
    # material textures: (rgba8 uint8 array (h, w, 4), wrap_s, wrap_t) per glTF texture
    textures: list = field(default_factory=list)
    _desc: object = None
    _tex: object = None

    def desc(self) -> _abi.CgSceneDesc:
        """A cg_scene_desc pointing into this object's arrays (keep self alive)."""
        for a in (self.vertices, self.indices, self.meshes, self.instances, self.materials):
            assert a.flags["C_CONTIGUOUS"]
        d = _abi.CgSceneDesc()
        d.vertices = self.vertices.ctypes.data
        d.vertex_count = len(self.vertices)
        d.indices = self.indices.ctypes.data
        d.index_count = len(self.indices)
        d.meshes = self.meshes.ctypes.data
        d.mesh_count = len(self.meshes)
        d.instances = self.instances.ctypes.data
        d.instance_count = len(self.instances)
        d.materials = self.materials.ctypes.data
        d.material_count = len(self.materials)
        if self.env is not None:
            assert self.env.dtype == np.float32 and self.env.ndim == 3 and self.env.shape[2] == 4
            d.env_rgba32f = self.env.ctypes.data
            d.env_height, d.env_width = self.env.shape[0], self.env.shape[1]
        if self.textures:
            arr = (_abi.CgTexture * len(self.textures))()
            for k, (img, ws, wt) in enumerate(self.textures):
                assert img.dtype == np.uint8 and img.ndim == 3 and img.shape[2] == 4
                assert img.flags["C_CONTIGUOUS"]
                arr[k].height, arr[k].width = img.shape[0], img.shape[1]
                arr[k].rgba8 = img.ctypes.data
                arr[k].wrap_s, arr[k].wrap_t = ws, wt
            d.textures = C.cast(arr, C.c_void_p)
            d.texture_count = len(self.textures)
            self._tex = arr
        self._desc = d
        return d

    @property
    def triangle_count(self) -> int:
        return int(sum(int(self.meshes[m]["index_count"]) // 3 for m in self.instances["mesh"]))


class _Builder:
    def __init__(self):
        self.verts = []
        self.idx = []
        self.meshes = []
        self.instances = []
        self.materials = []
        self.textures = []
        self.nv = 0
        self.ni = 0

    def add_mesh(self, positions, normals, tris, uv0=None, uv1=None) -> int:
        positions = np.asarray(positions, np.float32)
        normals = np.asarray(normals, np.float32)
        tris = np.asarray(tris, np.uint32).reshape(-1)
        v = np.zeros(len(positions), _abi.VERTEX_DTYPE)
        v["position"] = positions
        v["normal"] = normals
        if uv0 is not None:
            v["tex_coord0"] = np.asarray(uv0, np.float32)
        if uv1 is not None:
            v["tex_coord1"] = np.asarray(uv1, np.float32)
        self.verts.append(v)
        self.idx.append(tris + np.uint32(self.nv))
        self.meshes.append((self.nv, len(positions), self.ni, len(tris)))
        self.nv += len(positions)
        self.ni += len(tris)
        return len(self.meshes) - 1

    def add_material(self, base=(1, 1, 1), metallic=0.0, roughness=1.0, ior=1.5, dispersion=0.0,
                     transmission=0.0, thickness=0.0, emissive=(0, 0, 0), strength=1.0,
                     textures=None, texcoord_sets=0) -> int:
        """textures: optional dict of base_color / metallic_roughness / emissive /
        transmission -> texture index; texcoord_sets: bit k selects TEXCOORD_1."""
        m = np.zeros(1, _abi.MATERIAL_DTYPE)
        m["base_color_factor"] = [base[0], base[1], base[2], 1.0]
        m["emissive_factor"] = emissive
        m["emissive_strength"] = strength
        m["metallic_factor"] = metallic
        m["roughness_factor"] = roughness
        m["ior"] = ior
        m["dispersion"] = dispersion
        m["transmission_factor"] = transmission
        m["thickness_factor"] = thickness
        for k in ("base_color_texture", "metallic_roughness_texture", "emissive_texture",
                  "transmission_texture"):
            m[k] = (textures or {}).get(k.replace("_texture", ""), -1)
        m["texcoord_sets"] = texcoord_sets
        self.materials.append(m)
        return len(self.materials) - 1

    def add_instance(self, mesh, material, matrix=None):
        inst = np.zeros(1, _abi.INSTANCE_DTYPE)
        if matrix is None:
            matrix = np.eye(3, 4)
        inst["world_from_local"] = np.asarray(matrix, np.float32).reshape(12)
        inst["mesh"] = mesh
        inst["material"] = material
        self.instances.append(inst)

    def add_texture(self, rgba8, wrap_s=10497, wrap_t=10497) -> int:
        """An RGBA8 image (h, w, 4) as a material texture (glTF wrap modes)."""
        self.textures.append((np.ascontiguousarray(rgba8, np.uint8), int(wrap_s), int(wrap_t)))
        return len(self.textures) - 1

    def build(self, name, camera, conf, env=None) -> Scene:
        """The scene (empty arrays where nothing was added: a scene without
        geometry renders the environment alone)."""
        def cat(parts, dtype):
            return np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(0, dtype))
        meshes = np.array(self.meshes, np.uint32).reshape(-1, 4).copy().view(_abi.MESH_DTYPE).reshape(-1)
        return Scene(name=name,
                     vertices=cat(self.verts, _abi.VERTEX_DTYPE),
                     indices=cat(self.idx, np.uint32),
                     meshes=np.ascontiguousarray(meshes),
                     instances=cat(self.instances, _abi.INSTANCE_DTYPE),
                     materials=cat(self.materials, _abi.MATERIAL_DTYPE),
                     env=env, camera=camera, conf=conf, textures=list(self.textures))


def _quad(p0, p1, p2, p3):
    """Two triangles (p0 p1 p2), (p0 p2 p3) with the flat normal of the winding."""
    pos = np.array([p0, p1, p2, p3], np.float32)
    n = np.cross(pos[1] - pos[0], pos[2] - pos[0])
    n = n / np.linalg.norm(n)
    return pos, np.repeat(n[None], 4, 0), np.array([0, 1, 2, 0, 2, 3], np.uint32)


def _cube():
    """Unit cube [-0.5, 0.5]^3, 12 triangles, flat normals (24 vertices)."""
    P, N, T = [], [], []
    faces = [((0, 0, -1), 2), ((0, 0, 1), 2), ((0, -1, 0), 1), ((0, 1, 0), 1), ((-1, 0, 0), 0),
             ((1, 0, 0), 0)]
    for n, ax in faces:
        n = np.array(n, np.float32)
        u = np.roll(np.array([1, 0, 0], np.float32), (ax + 1) % 3)
        v = np.cross(n, u)
        c = n * 0.5
        corners = [c - 0.5 * u - 0.5 * v, c + 0.5 * u - 0.5 * v, c + 0.5 * u + 0.5 * v,
                   c - 0.5 * u + 0.5 * v]
        base = len(P)
        P += corners
        N += [n] * 4
        T += [base, base + 1, base + 2, base, base + 2, base + 3]
    return np.array(P, np.float32), np.array(N, np.float32), np.array(T, np.uint32)


def _trs(scale=(1, 1, 1), rot_z=0.0, translate=(0, 0, 0), rot=None):
    """Row-major 3x4 world_from_local = T * R * S."""
    if rot is None:
        c, s = math.cos(rot_z), math.sin(rot_z)
        rot = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]], np.float64)
    m = np.zeros((3, 4), np.float64)
    m[:, :3] = rot @ np.diag(np.asarray(scale, np.float64))
    m[:, 3] = translate
    return m


def camera_viewport(width, height, half_height=0.5):
    return (half_height * width / height, half_height)


# ---------------------------------------------------------------------------
# Config 0: Cornell box
# ---------------------------------------------------------------------------
def cornell(width=256, height=256, spp=1, depth=2) -> Scene:
    b = _Builder()
    white = b.add_material(base=(0.75, 0.75, 0.75))
    red = b.add_material(base=(0.63, 0.06, 0.05))
    green = b.add_material(base=(0.14, 0.45, 0.09))
    metal = b.add_material(base=(0.95, 0.95, 0.95), metallic=1.0, roughness=0.0)
    light = b.add_material(base=(0, 0, 0), emissive=(1, 1, 1), strength=15.0)
    # room: x in [-1, 1], y in [-1, 1], z in [0, 2]; open at y = -1
    walls = [_quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0)),      # floor
             _quad((-1, -1, 2), (-1, 1, 2), (1, 1, 2), (1, -1, 2)),      # ceiling
             _quad((-1, 1, 0), (1, 1, 0), (1, 1, 2), (-1, 1, 2))]        # back
    P = np.concatenate([w[0] for w in walls])
    N = np.concatenate([w[1] for w in walls])
    T = np.concatenate([w[2] + 4 * i for i, w in enumerate(walls)])
    b.add_instance(b.add_mesh(P, N, T), white)
    b.add_instance(b.add_mesh(*_quad((-1, -1, 0), (-1, 1, 0), (-1, 1, 2), (-1, -1, 2))), red)
    b.add_instance(b.add_mesh(*_quad((1, -1, 0), (1, -1, 2), (1, 1, 2), (1, 1, 0))), green)
    cube = b.add_mesh(*_cube())
    b.add_instance(cube, white, _trs((0.6, 0.6, 1.2), 0.3, (-0.35, 0.3, 0.6)))
    b.add_instance(cube, metal, _trs((0.6, 0.6, 0.6), -0.3, (0.4, -0.3, 0.3)))
    h = 0.125
    b.add_instance(b.add_mesh(*_quad((-h, -h, 1.999), (-h, h, 1.999), (h, h, 1.999), (h, -h, 1.999))),
                   light)
    cam = _abi.make_camera((0.0, -3.4, 1.0), (0.0, 1.0, 0.0), camera_viewport(width, height, 0.42))
    return b.build("cornell", cam, dict(width=width, height=height, spp=spp, depth=depth))


def _quad_uv(scale=1.0, offset=0.0):
    """UVs of _quad's four corners."""
    return np.array([(0, 0), (1, 0), (1, 1), (0, 1)], np.float32) * scale + offset


def _texture(rng, h, w, kind):
    """Seeded procedural RGBA8 images for the textured scene."""
    y, x = np.mgrid[0:h, 0:w]
    img = np.zeros((h, w, 4), np.uint8)
    img[..., 3] = 255
    if kind == "checker":
        c = ((x // 8 + y // 8) % 2).astype(bool)
        img[..., 0] = np.where(c, 230, 40)
        img[..., 1] = np.where(c, 200, 90)
        img[..., 2] = np.where(c, 60, 210)
    elif kind == "gradient":   # g: roughness, b: metallic (glTF metallicRoughness)
        img[..., 1] = (255 * x / max(w - 1, 1)).astype(np.uint8)
        img[..., 2] = (255 * y / max(h - 1, 1)).astype(np.uint8)
    else:                      # random texels
        img[..., :3] = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
    return img


def textured_cornell(width=96, height=96, spp=2, depth=4) -> Scene:
    """The Cornell room with material textures of different sizes (resized to
    the largest into one array): a checkered base color on the floor and back
    wall with UVs reaching past [0, 1] (clamp to edge when shading, wrap modes
    in the light buffer), a metallic-roughness gradient on the metal box read
    through TEXCOORD_1, a random-texel emissive texture on the ceiling light
    and a transmission texture on a glass box."""
    rng = np.random.default_rng(7)
    b = _Builder()
    checker = b.add_texture(_texture(rng, 64, 64, "checker"))
    mr = b.add_texture(_texture(rng, 16, 32, "gradient"), 33071, 33071)
    emis = b.add_texture(_texture(rng, 8, 8, "random"), 33648, 10497)
    trans = b.add_texture(_texture(rng, 24, 16, "random"))
    white_tex = b.add_material(base=(0.9, 0.9, 0.9), textures={"base_color": checker})
    red = b.add_material(base=(0.63, 0.06, 0.05))
    green = b.add_material(base=(0.14, 0.45, 0.09))
    metal = b.add_material(base=(0.95, 0.95, 0.95), metallic=1.0, roughness=0.8,
                           textures={"metallic_roughness": mr}, texcoord_sets=0b10)
    glass = b.add_material(base=(1, 1, 1), roughness=0.0, ior=1.5, transmission=1.0, thickness=1.0,
                           textures={"transmission": trans})
    light = b.add_material(base=(0, 0, 0), emissive=(1, 1, 1), strength=15.0,
                           textures={"emissive": emis})
    floor = _quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0))
    back = _quad((-1, 1, 0), (1, 1, 0), (1, 1, 2), (-1, 1, 2))
    b.add_instance(b.add_mesh(*floor, uv0=_quad_uv(1.6, -0.3)), white_tex)
    b.add_instance(b.add_mesh(*back, uv0=_quad_uv(1.0)), white_tex)
    b.add_instance(b.add_mesh(*_quad((-1, -1, 2), (-1, 1, 2), (1, 1, 2), (1, -1, 2))), red)
    b.add_instance(b.add_mesh(*_quad((-1, -1, 0), (-1, 1, 0), (-1, 1, 2), (-1, -1, 2))), red)
    b.add_instance(b.add_mesh(*_quad((1, -1, 0), (1, -1, 2), (1, 1, 2), (1, 1, 0))), green)
    P, N, T = _cube()
    uv = np.tile(_quad_uv(1.0), (6, 1))
    cube_uv = b.add_mesh(P, N, T, uv0=uv, uv1=uv[:, ::-1].copy())
    b.add_instance(cube_uv, metal, _trs((0.6, 0.6, 0.6), -0.3, (0.4, -0.3, 0.3)))
    b.add_instance(cube_uv, glass, _trs((0.5, 0.5, 0.9), 0.4, (-0.4, 0.2, 0.45)))
    h = 0.3
    b.add_instance(b.add_mesh(*_quad((-h, -h, 1.999), (-h, h, 1.999), (h, h, 1.999), (h, -h, 1.999)),
                              uv0=_quad_uv(2.5, -0.7)), light)
    cam = _abi.make_camera((0.0, -3.4, 1.0), (0.0, 1.0, 0.0), camera_viewport(width, height, 0.42))
    return b.build("textured_cornell", cam, dict(width=width, height=height, spp=spp, depth=depth))


# ---------------------------------------------------------------------------
# Procedural meshes
# ---------------------------------------------------------------------------
def _value_noise3(p, seed, octaves=3):
    """Seeded 3-octave value noise in [-1, 1] at points p (n, 3)."""
    p = np.asarray(p, np.float64)
    total = np.zeros(len(p))
    amp_sum = 0.0
    for o in range(octaves):
        freq = 2.0 * (2 ** o)
        amp = 0.5 ** o
        q = p * freq
        i0 = np.floor(q).astype(np.int64)
        f = q - i0
        f = f * f * (3.0 - 2.0 * f)

        def h(ix, iy, iz):
            x = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791) ^ (seed * 2654435761 + o * 97)
            x = (x ^ (x >> 13)) * 1274126177
            x = x ^ (x >> 16)
            return (x & 0xFFFF).astype(np.float64) / 32767.5 - 1.0

        acc = 0.0
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    w = (np.where(dx, f[:, 0], 1 - f[:, 0]) * np.where(dy, f[:, 1], 1 - f[:, 1]) *
                         np.where(dz, f[:, 2], 1 - f[:, 2]))
                    acc = acc + w * h(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz)
        total += amp * acc
        amp_sum += amp
    return total / amp_sum


def _vertex_normals(P, T):
    T = T.reshape(-1, 3)
    fn = np.cross(P[T[:, 1]] - P[T[:, 0]], P[T[:, 2]] - P[T[:, 0]])
    N = np.zeros_like(P, dtype=np.float64)
    for k in range(3):
        np.add.at(N, T[:, k], fn)
    N /= np.maximum(np.linalg.norm(N, axis=1, keepdims=True), 1e-30)
    return N.astype(np.float32)


def icosphere(subdiv):
    t = (1.0 + 5 ** 0.5) / 2.0
    V = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                 np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                  [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                  [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                  [8, 6, 7], [9, 8, 1]], np.int64)
    for _ in range(subdiv):
        a, b_, c = F[:, 0], F[:, 1], F[:, 2]
        edges = np.concatenate([np.stack([a, b_], 1), np.stack([b_, c], 1), np.stack([c, a], 1)])
        edges.sort(axis=1)
        uniq, inv = np.unique(edges, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mids = V[uniq[:, 0]] + V[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = len(V)
        V = np.concatenate([V, mids])
        nf = len(F)
        ab, bc, ca = inv[:nf] + base, inv[nf:2 * nf] + base, inv[2 * nf:] + base
        F = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b_, bc, ab], 1),
                            np.stack([c, ca, bc], 1), np.stack([ab, bc, ca], 1)])
    return V, F


def _displaced(V, F, amp, seed):
    r = 1.0 + amp * _value_noise3(V, seed)
    P = (V * r[:, None]).astype(np.float32)
    T = F.astype(np.uint32).reshape(-1)
    return P, _vertex_normals(P.astype(np.float64), T), T


def _uv_sphere(target_tris, amp, seed):
    stacks = max(4, int(round(math.sqrt(target_tris / 4.0))))
    slices = max(6, int(round(target_tris / (2.0 * stacks))))
    th = np.linspace(0, math.pi, stacks + 1)
    ph = np.linspace(0, 2 * math.pi, slices, endpoint=False)
    TH, PH = np.meshgrid(th, ph, indexing="ij")
    V = np.stack([np.sin(TH) * np.cos(PH), np.sin(TH) * np.sin(PH), np.cos(TH)], -1).reshape(-1, 3)
    i = np.arange(stacks)[:, None]
    j = np.arange(slices)[None, :]
    a = i * slices + j
    b_ = i * slices + (j + 1) % slices
    c = (i + 1) * slices + j
    d = (i + 1) * slices + (j + 1) % slices
    F = np.concatenate([np.stack([a, c, b_], -1).reshape(-1, 3), np.stack([b_, c, d], -1).reshape(-1, 3)])
    # drop the degenerate triangles at the poles
    P = V[F]
    area = np.linalg.norm(np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]), axis=1)
    F = F[area > 1e-12]
    return _displaced(V, F, amp, seed)


def _torus(target_tris, amp, seed, R=1.0, r=0.35):
    nu = max(8, int(round(math.sqrt(target_tris / 2.0 * 3.0))))
    nv = max(6, int(round(target_tris / (2.0 * nu))))
    u = np.linspace(0, 2 * math.pi, nu, endpoint=False)
    v = np.linspace(0, 2 * math.pi, nv, endpoint=False)
    U, Vv = np.meshgrid(u, v, indexing="ij")
    rr = r * (1.0 + amp * _value_noise3(np.stack([np.cos(U), np.sin(U), np.cos(Vv)], -1).reshape(-1, 3),
                                        seed).reshape(U.shape))
    P = np.stack([(R + rr * np.cos(Vv)) * np.cos(U), (R + rr * np.cos(Vv)) * np.sin(U), rr * np.sin(Vv)],
                 -1).reshape(-1, 3)
    i = np.arange(nu)[:, None]
    j = np.arange(nv)[None, :]
    a = i * nv + j
    b_ = ((i + 1) % nu) * nv + j
    c = i * nv + (j + 1) % nv
    d = ((i + 1) % nu) * nv + (j + 1) % nv
    F = np.concatenate([np.stack([a, b_, c], -1).reshape(-1, 3), np.stack([c, b_, d], -1).reshape(-1, 3)])
    P = P.astype(np.float32)
    T = F.astype(np.uint32).reshape(-1)
    return P, _vertex_normals(P.astype(np.float64), T), T


def _emissive_triangles(b, rng, count, radiance, centers, size):
    """count one-triangle emissive instances of white emission x radiance."""
    tri_mesh = b.add_mesh(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32),
                          np.array([[0, 0, 1]] * 3, np.float32), np.array([0, 1, 2], np.uint32))
    for k in range(count):
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        mat = b.add_material(base=(0, 0, 0), emissive=(1, 1, 1), strength=float(radiance[k]))
        b.add_instance(tri_mesh, mat, _trs((size, size, size), translate=centers[k], rot=q))


# ---------------------------------------------------------------------------
# Config 1: displaced dispersive icosphere
# ---------------------------------------------------------------------------
def icosphere_scene(width=1280, height=720, spp=16, depth=8, subdiv=8, seed=1) -> Scene:
    rng = np.random.default_rng(seed)
    b = _Builder()
    glass = b.add_material(base=(1, 1, 1), metallic=0.0, roughness=0.1, ior=CAUCHY_IOR,
                           dispersion=CAUCHY_DISPERSION, transmission=1.0, thickness=1.0)
    ground = b.add_material(base=(0.5, 0.5, 0.5))
    V, F = icosphere(subdiv)
    b.add_instance(b.add_mesh(*_displaced(V, F, 0.05, seed)), glass)
    g = 50.0
    b.add_instance(b.add_mesh(*_quad((-g, -g, -1.1), (g, -g, -1.1), (g, g, -1.1), (-g, g, -1.1))),
                   ground)
    n = 64
    ang = rng.uniform(0, 2 * math.pi, n)
    rad = rng.uniform(1.6, 3.0, n)
    centers = np.stack([rad * np.cos(ang), rad * np.sin(ang), rng.uniform(1.5, 3.0, n)], 1)
    radiance = np.exp(rng.uniform(math.log(1.0), math.log(100.0), n))
    _emissive_triangles(b, rng, n, radiance, centers, 0.3)
    cam = _abi.make_camera((0.0, -4.2, 0.6), (0.0, 1.0, -0.15), camera_viewport(width, height))
    return b.build("icosphere", cam, dict(width=width, height=height, spp=spp, depth=depth))


# ---------------------------------------------------------------------------
# Config 2: instanced two-level scene
# ---------------------------------------------------------------------------
def _random_rotation(rng):
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def instanced_scene(width=1920, height=1080, spp=64, depth=12, instances=4096, lights=10000,
                    seed=2, mesh_scale=1.0, extent=50.0, camera_distance=150.0,
                    radiance_sigma=2.0) -> Scene:
    rng = np.random.default_rng(seed)
    b = _Builder()
    meshes = []
    sizes = np.exp(rng.uniform(math.log(10_000), math.log(200_000), 8)) * mesh_scale
    for k in range(8):
        if k % 2 == 0:
            meshes.append(b.add_mesh(*_uv_sphere(int(sizes[k]), 0.08, seed * 100 + k)))
        else:
            meshes.append(b.add_mesh(*_torus(int(sizes[k]), 0.08, seed * 100 + k)))
    kinds = rng.choice(4, size=instances, p=[0.4, 0.3, 0.2, 0.1])
    for i in range(instances):
        kind = kinds[i]
        if kind == 0:
            a = rng.uniform(0.1, 0.9, 3)
            mat = b.add_material(base=tuple(a))
        elif kind == 1:
            mat = b.add_material(base=tuple(rng.uniform(0.5, 1.0, 3)), metallic=1.0,
                                 roughness=float(rng.uniform(0.05, 0.6)))
        elif kind == 2:
            mat = b.add_material(base=(0.95, 0.95, 0.95), metallic=1.0, roughness=0.0)
        else:
            mat = b.add_material(base=(1, 1, 1), roughness=0.0, ior=float(rng.uniform(1.3, 1.8)),
                                 transmission=1.0, thickness=1.0)
        s = rng.uniform(0.5, 3.0)
        b.add_instance(meshes[rng.integers(8)], mat,
                       _trs((s, s, s), translate=rng.uniform(-extent, extent, 3),
                            rot=_random_rotation(rng)))
    radiance = np.exp(rng.normal(0.0, radiance_sigma, lights))
    centers = rng.uniform(-extent, extent, (lights, 3))
    _emissive_triangles(b, rng, lights, radiance, centers, 0.5)
    cam = _abi.make_camera((0.0, -camera_distance, 0.13 * camera_distance), (0.0, 1.0, -0.13),
                           camera_viewport(width, height))
    return b.build(f"instanced{instances}", cam,
                   dict(width=width, height=height, spp=spp, depth=depth))


# ---------------------------------------------------------------------------
# Config 3 / 4: view batches and request streams
# ---------------------------------------------------------------------------
def sphere_pose(rng, radius=150.0):
    """A camera on a sphere of `radius` looking at the origin; poses whose
    direction is within 0.999 of +-z are rejected (cameraRay's fixed +z up
    vector degenerates there, compute.wesl:68-74)."""
    while True:
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        d = -v
        if abs(d[2]) <= 0.999:
            return v * radius, d


def batch_views(count=256, seed=3, min_side=64, max_side=1024, spp_choices=(1, 4, 16, 64)):
    """[(position, direction, side, spp, seed)] for the 256-view batch."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        side = int(round(math.exp(rng.uniform(math.log(min_side), math.log(max_side)))))
        spp = int(rng.choice(spp_choices))
        p, d = sphere_pose(rng)
        out.append((p, d, side, side, spp, i))
    return out


def request_stream(count, rate_hz, scenes=4, seed=4,
                   resolutions=((256, 256), (512, 512), (1280, 720), (1920, 1080)),
                   spp_choices=(1, 4, 16)):
    """Poisson arrivals: [(arrival_s, scene, position, direction, w, h, spp, seed)]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate_hz)
        w, h = resolutions[rng.integers(len(resolutions))]
        p, d = sphere_pose(rng)
        out.append((t, int(rng.integers(scenes)), p, d, w, h, int(rng.choice(spp_choices)), i))
    return out
