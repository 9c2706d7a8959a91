"""ctypes mirror of include/cg_cuda.h (the C ABI of libcg_cuda.so).

Only layouts and constants live here; the loaded library and its calls are in
``crystalgraphics_b200.backend``.
"""
import ctypes as C

import numpy as np

CG_OK = 0
CG_E_INVALID = -1
CG_E_NOT_INIT = -2
CG_E_CUDA = -3
CG_E_OOM = -4
CG_E_TIMEOUT = -5
CG_E_DEVICE = -6
CG_E_CANCELLED = -7
CG_E_BUSY = -8

CG_SPECTRAL_REFERENCE, CG_SPECTRAL_HERO = 0, 1
CG_FILM_XYZ32F = 0
CG_FILM_RGBA8 = 1
CG_FILM_RGB32F = 2

u32 = C.c_uint32
f32 = C.c_float


class CgConf(C.Structure):
    """PathTraceConf (include/CrystalGraphics/environment.h:11-18)."""
    _fields_ = [
        ("window_width", u32), ("window_height", u32),
        ("render_width", u32), ("render_height", u32),
        ("sample_count", u32), ("trace_depth", u32),
        ("max_transport_sample_count", u32), ("max_diffuse_sample_count", u32),
        ("max_rough_sample_count", u32), ("max_emission_sample_count", u32),
    ]


class CgCamera(C.Structure):
    """Camera (include/CrystalGraphics/camera.h:9-13), 48 bytes."""
    _fields_ = [
        ("position", f32 * 3), ("_pad0", f32),
        ("direction", f32 * 3), ("_pad1", f32),
        ("viewport", f32 * 2), ("_pad2", f32 * 2),
    ]


class CgSceneDesc(C.Structure):
    _fields_ = [
        ("vertices", C.c_void_p), ("vertex_count", u32),
        ("indices", C.c_void_p), ("index_count", u32),
        ("meshes", C.c_void_p), ("mesh_count", u32),
        ("instances", C.c_void_p), ("instance_count", u32),
        ("materials", C.c_void_p), ("material_count", u32),
        ("env_rgba32f", C.c_void_p), ("env_width", u32), ("env_height", u32),
        ("textures", C.c_void_p), ("texture_count", u32),
    ]


class CgTexture(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("rgba8", C.c_void_p), ("wrap_s", C.c_int32),
                ("wrap_t", C.c_int32), ("_pad", u32 * 2)]


class CgSceneInfo(C.Structure):
    _fields_ = [
        ("instance_count", u32), ("mesh_count", u32), ("triangle_count", u32),
        ("material_count", u32), ("emissive_count", u32),
        ("blas_node_count", u32), ("tlas_node_count", u32), ("light_node_count", u32),
        ("device_bytes", C.c_uint64), ("tag", C.c_uint64),
        ("bvh_build_seconds", C.c_double), ("bvh_host_builds", u32),
        ("bvh_device_builds", u32),
    ]


class CgHit(C.Structure):
    _fields_ = [("t", f32), ("u", f32), ("v", f32), ("instance", C.c_int32),
                ("triangle", C.c_int32), ("_pad", C.c_int32 * 3)]


class CgStats(C.Structure):
    _fields_ = [
        ("samples", C.c_uint64), ("extend_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
        ("node_visits", C.c_uint64), ("tri_tests", C.c_uint64), ("inst_visits", C.c_uint64),
        ("chunks", u32), ("kernel_launches", u32), ("device_ms", f32), ("_pad", u32),
        ("nonfinite_samples", C.c_uint64),
    ]


class CgProfile(C.Structure):
    _fields_ = [("ms", C.c_double * 5), ("launches", C.c_uint64 * 5)]


class CgViewDesc(C.Structure):
    _fields_ = [("camera", CgCamera), ("width", u32), ("height", u32), ("spp", u32),
                ("seed", u32)]


class CgTuning(C.Structure):
    _fields_ = [("queue_capacity", u32), ("extend_block", u32), ("shade_block", u32),
                ("use_graph", u32), ("bvh_width", u32), ("persistent", u32), ("shade_sort", u32),
                ("box_bits", u32), ("pipelines", u32), ("traversal_threads", u32)]


class CgRequest(C.Structure):
    _fields_ = [("scene", u32), ("view", CgViewDesc)]


class CgRequestResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("_pad", u32), ("submit_s", C.c_double),
                ("start_s", C.c_double), ("finish_s", C.c_double)]


class CgServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64),
                ("cancelled", C.c_uint64), ("rejected", C.c_uint64),
                ("samples", C.c_uint64), ("active", u32), ("pending", u32),
                ("bytes_in_use", C.c_uint64), ("peak_bytes", C.c_uint64),
                ("chunks", C.c_uint64), ("busy_s", C.c_double), ("all_busy_s", C.c_double),
                ("copy_out_s", C.c_double)]


# numpy record layouts of the scene arrays (must match include/cg_cuda.h)
VERTEX_DTYPE = np.dtype([("position", "<f4", 3), ("_pad0", "<f4"), ("normal", "<f4", 3),
                         ("_pad1", "<f4"), ("tex_coord0", "<f4", 2), ("tex_coord1", "<f4", 2)])
MESH_DTYPE = np.dtype([("vertex_offset", "<u4"), ("vertex_count", "<u4"),
                       ("index_offset", "<u4"), ("index_count", "<u4")])
INSTANCE_DTYPE = np.dtype([("world_from_local", "<f4", 12), ("mesh", "<u4"),
                           ("material", "<u4"), ("_pad", "<u4", 2)])
MATERIAL_DTYPE = np.dtype([
    ("base_color_factor", "<f4", 4), ("emissive_factor", "<f4", 3), ("emissive_strength", "<f4"),
    ("metallic_factor", "<f4"), ("roughness_factor", "<f4"), ("ior", "<f4"),
    ("dispersion", "<f4"), ("transmission_factor", "<f4"), ("thickness_factor", "<f4"),
    ("base_color_texture", "<i4"), ("metallic_roughness_texture", "<i4"),
    ("emissive_texture", "<i4"), ("transmission_texture", "<i4"), ("texcoord_sets", "<u4"),
    ("_pad", "<u4")])
EMISSIVE_DTYPE = np.dtype([("v0", "<f4", 3), ("_p0", "<f4"), ("v1", "<f4", 3), ("_p1", "<f4"),
                           ("v2", "<f4", 3), ("_p2", "<f4"), ("emission", "<f4", 3),
                           ("area", "<f4"), ("weight", "<f4"), ("_pad", "<f4", 3)])
ALIAS_DTYPE = np.dtype([("alias", "<u4"), ("prob", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("u", "<f4"), ("v", "<f4"), ("instance", "<i4"),
                      ("triangle", "<i4"), ("_pad", "<i4", 3)])

assert C.sizeof(CgCamera) == 48
assert C.sizeof(CgConf) == 40
assert VERTEX_DTYPE.itemsize == 48
assert INSTANCE_DTYPE.itemsize == 64
assert MATERIAL_DTYPE.itemsize == 80
assert EMISSIVE_DTYPE.itemsize == 80
assert ALIAS_DTYPE.itemsize == 8
assert HIT_DTYPE.itemsize == C.sizeof(CgHit) == 32


def make_conf(width, height, spp, depth, max_transport=3, max_diffuse=1, max_rough=1,
              max_emission=1):
    """PathTraceConf with the reference defaults for the sample caps."""
    return CgConf(1920, 1080, width, height, spp, depth, max_transport, max_diffuse,
                  max_rough, max_emission)


def make_camera(position, direction, viewport):
    cam = CgCamera()
    cam.position[:] = [float(x) for x in position]
    cam.direction[:] = [float(x) for x in direction]
    cam.viewport[:] = [float(x) for x in viewport]
    return cam

CG_BVH_BUILD_AUTO, CG_BVH_BUILD_HOST, CG_BVH_BUILD_DEVICE = 0, 1, 2
