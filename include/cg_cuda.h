/*
 * cg_cuda.h — C ABI of the B200 spectral path-tracing backend (libcg_cuda.so).
 *
 * This is the drop-in boundary for the View() hot path of
 * ray847/CrystalGraphics.  The reference renders through WebGPU:
 *   View(scene, camera)                    src/view.cpp:12-16
 *   └ Env::View → SceneData (host packing) src/environment.cpp:69-74
 *     └ wgpu::Env::View (upload, dispatch) src/wgpu/view.cpp:16-88
 *       └ compute.wesl main (per pixel)    src/wgpu/shader/compute.wesl:32-62
 * Here the same work is a set of plain C entry points over plain pointers and
 * sizes.  The C++23 layer (include/CrystalGraphics/) keeps the reference's
 * public signatures and calls these; Python reaches them through ctypes.
 *
 * Conventions
 *   - Every function returns an int status: CG_OK (0) or a negative CG_E_*
 *     code.  cg_last_error() returns a thread-local message for the last
 *     failure on the calling thread.  No C++ exception crosses this ABI.
 *   - Host pointers are plain host memory.  The library owns every device
 *     allocation it makes; handles are opaque.
 *   - There is no CPU fallback: with no CUDA device every call that needs
 *     one fails with CG_E_CUDA.
 */
#ifndef CG_CUDA_H_
#define CG_CUDA_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CG_API __attribute__((visibility("default")))

/* ---- status codes ------------------------------------------------------ */
enum {
  CG_OK = 0,
  CG_E_INVALID = -1,     /* bad argument, size or handle                     */
  CG_E_NOT_INIT = -2,    /* cg_init() not called ("Environment not initialized.") */
  CG_E_CUDA = -3,        /* a CUDA runtime call failed                       */
  CG_E_OOM = -4,         /* device allocation failed or over the HBM budget  */
  CG_E_TIMEOUT = -5,     /* a bounded device or host wait ran out            */
  CG_E_DEVICE = -6,      /* a kernel reported an error in its status word    */
  CG_E_CANCELLED = -7,   /* a served request was cancelled                   */
  CG_E_BUSY = -8         /* a queue is full; retry later                     */
};

/* ---- configuration ------------------------------------------------------
 * Mirrors PathTraceConf (include/CrystalGraphics/environment.h:11-18).
 * window_* are accepted and ignored: the backend is headless.  trace_depth is
 * clamped to [1, 64] as wgpu::CreateEnv does (src/wgpu/environment.cpp:20).
 * The max_*_sample_count fields become the override constants @id(5..8) of
 * shading/sample.wesl:102-105 and are further capped by its constants
 * (sample.wesl:98-101). */
typedef struct cg_conf {
  uint32_t window_width, window_height;
  uint32_t render_width, render_height;
  uint32_t sample_count;
  uint32_t trace_depth;
  uint32_t max_transport_sample_count, max_diffuse_sample_count,
      max_rough_sample_count, max_emission_sample_count;
} cg_conf;

/* ---- camera --------------------------------------------------------------
 * Same 48-byte layout as crystal::graphics::Camera (camera.h:9-13):
 * alignas(16) vec3 position, alignas(16) vec3 direction, alignas(8) vec2 viewport. */
typedef struct cg_camera {
  float position[3];
  float _pad0;
  float direction[3];
  float _pad1;
  float viewport[2];
  float _pad2[2];
} cg_camera;

/* ---- scene description (the input of LoadScene) ---------------------------
 * cg_vertex has the layout of the reference Vertex (src/vertex.h:12-24). */
typedef struct cg_vertex {
  float position[3];
  float _pad0;
  float normal[3];
  float _pad1;
  float tex_coord0[2];
  float tex_coord1[2];
} cg_vertex;

/* A mesh is one glTF mesh primitive's geometry: a range of the global index
 * buffer whose entries are absolute vertex indices (Primitive,
 * src/scene_impl.h:24-30, without its material). */
typedef struct cg_mesh {
  uint32_t vertex_offset, vertex_count;
  uint32_t index_offset, index_count;
} cg_mesh;

/* An instance is one placed primitive: the reference builds one BLAS and one
 * Instance per (node, mesh primitive) (src/pathtracing/tlas.h:56-73,
 * src/pathtracing/instance.h:9-17).  Here instances that name the same mesh
 * share one BLAS on the device; the geometry and every hit are identical.
 * world_from_local is a row-major 3x4 affine matrix. */
typedef struct cg_instance {
  float world_from_local[12];
  uint32_t mesh;
  uint32_t material;
  uint32_t _pad[2];
} cg_instance;

/* The material fields the path tracer reads out of the reference's
 * PackedMaterial (src/material.h:30-87, shading/material.wesl:19-53).
 * Texture references index cg_scene_desc.textures (-1 = none), the four
 * textures decode() samples (material.wesl:181-262); bit k of texcoord_sets
 * selects TEXCOORD_1 instead of TEXCOORD_0 for texture k in this order:
 * base color, metallic-roughness, emissive, transmission. */
typedef struct cg_material {
  float base_color_factor[4];
  float emissive_factor[3];
  float emissive_strength;
  float metallic_factor;
  float roughness_factor;
  float ior;
  float dispersion;
  float transmission_factor;
  float thickness_factor;
  int32_t base_color_texture;
  int32_t metallic_roughness_texture;
  int32_t emissive_texture;
  int32_t transmission_texture;
  uint32_t texcoord_sets;
  uint32_t _pad;
} cg_material;

/* A decoded material texture (the reference's TextureData after
 * DecodeImageRgba8, src/image_decode.h:27): RGBA8 rows, top row first.
 * wrap_s / wrap_t are the glTF sampler wrap modes (33071 clamp to edge,
 * 33648 mirrored repeat, other = repeat); the reference uses them only for
 * the emissive-texture factor of its light buffer (emissive_buffer.h:150-200)
 * and samples every texture with clamp to edge when shading
 * (src/wgpu/resource.cpp:133-142). */
typedef struct cg_texture {
  uint32_t width, height;
  const uint8_t* rgba8;
  int32_t wrap_s, wrap_t;
  uint32_t _pad[2];
} cg_texture;

/* env_rgba32f == NULL selects the reference's fallback sky: a 512x256
 * vertical gradient (src/pathtracing/scene_data.h:73-98). */
typedef struct cg_scene_desc {
  const cg_vertex* vertices;
  uint32_t vertex_count;
  const uint32_t* indices;
  uint32_t index_count;
  const cg_mesh* meshes;
  uint32_t mesh_count;
  const cg_instance* instances;
  uint32_t instance_count;
  const cg_material* materials;
  uint32_t material_count;
  const float* env_rgba32f;
  uint32_t env_width, env_height;
  const cg_texture* textures;  /* material textures (may be NULL when count is 0) */
  uint32_t texture_count;
} cg_scene_desc;

typedef struct cg_scene_s* cg_scene_t;

/* ---- environment (EnvInit / EnvTerm / EnvStatus) -------------------------
 * cg_init replaces EnvInit (environment.h:20, src/environment.cpp:12-17):
 * it selects the CUDA device, creates the stream, the wavelength tables and
 * the film of render_width x render_height.  Calling it again re-creates the
 * environment. */
CG_API int cg_init(const cg_conf* conf, int device);
/* EnvTerm (src/environment.cpp:18-23).  Safe to call when not initialised.
 * Also frees the pinned film staging buffers that served requests left for
 * reuse (those a live server still holds stay). */
CG_API int cg_term(void);
/* EnvStatus (src/environment.cpp:34-37): 1 when initialised. */
CG_API int cg_status(void);
/* Thread-local message of the last failure on this thread ("" if none). */
CG_API const char* cg_last_error(void);
/* Effective configuration after clamping. */
CG_API int cg_get_conf(cg_conf* out);

/* ---- scenes (LoadScene, ~Scene) ------------------------------------------
 * Builds the BVHs, the emissive buffer and its alias table on the host and
 * uploads them with the geometry, materials and environment into device
 * buffers, once.  The reference rebuilds these on every View()
 * (src/environment.cpp:70); the uploaded scene is immutable. */
CG_API int cg_scene_create(const cg_scene_desc* desc, cg_scene_t* out);
CG_API int cg_scene_destroy(cg_scene_t scene);
/* LoadScene(path) (src/scene.cpp:829-1003): reads a glTF 2.0 file (.gltf with
 * .bin or data-URI buffers, or .glb) with the reference's conventions —
 * material 0 is the default material and glTF material i becomes i + 1, one
 * instance per (node, mesh primitive), y-up rotated to z-up — and uploads it
 * as cg_scene_create does. */
CG_API int cg_scene_load_gltf(const char* path, cg_scene_t* out);
/* The parse step of cg_scene_load_gltf alone (no device needed): fills *out
 * with arrays owned by *storage, released by cg_gltf_free. */
CG_API int cg_gltf_parse(const char* path, cg_scene_desc* out, void** storage);
CG_API int cg_gltf_free(void* storage);
/* Decodes a PNG file image to RGBA8 (the reference decodes glTF images with
 * stb_image, src/image_decode.cpp:12-45; JPEG: cg_jpeg_decode).  With
 * rgba_out == NULL only *width and *height are set; otherwise rgba_out must
 * hold width * height * 4 bytes. */
CG_API int cg_png_decode(const uint8_t* data, size_t size, uint32_t* width, uint32_t* height,
                         uint8_t* rgba_out);
/* A JPEG image to RGBA8 (the JPEG half of the reference's DecodeImageRgba8,
 * src/image_decode.cpp:12-45, written from ITU-T T.81 since stb_image is not
 * available): baseline, extended sequential and progressive Huffman-coded
 * 8-bit images, grey or three components, any sampling factors, restart
 * intervals.  Values can differ from stb_image's by a level or two (IDCT and
 * colour-conversion rounding).  Same calling convention as cg_png_decode;
 * glTF images and image-based-light faces are decoded as PNG or JPEG by their
 * signatures. */
CG_API int cg_jpeg_decode(const uint8_t* data, size_t size, uint32_t* width, uint32_t* height,
                          uint8_t* rgba_out);
/* A Radiance RGBE (.hdr) image to linear RGBA32F, alpha 1 (stb_image's HDR
 * loader, which the reference's DecodeImageRgba32f uses for environment
 * faces, src/image_decode.cpp:51-88): "-Y height +X width" images, flat or
 * run-length-encoded scanlines.  With rgba_out == NULL only the size is set;
 * otherwise rgba_out holds width * height * 4 floats. */
CG_API int cg_hdr_decode(const uint8_t* data, size_t size, uint32_t* width, uint32_t* height,
                         float* rgba_out);
/* The lat-long environment of an image-based light's cube
 * (CubeToEnvironmentTexture, src/scene.cpp:541-575): `faces` holds six
 * face_width x face_height RGBA32F images (+X, -X, +Y, -Y, +Z, -Z as
 * EXT_lights_image_based lists them) one after another; `rotation` is the
 * light's quaternion (x, y, z, w); `env_out` receives (2 * face_height) rows
 * of (4 * face_width) RGBA32F texels.  cg_scene_load_gltf / cg_gltf_parse do
 * this for a file's first image-based light (PNG or HDR faces). */
CG_API int cg_env_from_cube(const float* faces, uint32_t face_width, uint32_t face_height,
                            const float* rotation, float* env_out);

typedef struct cg_scene_info {
  uint32_t instance_count, mesh_count, triangle_count, material_count;
  uint32_t emissive_count;      /* emissive triangles (EmissivePrim entries) */
  uint32_t blas_node_count, tlas_node_count, light_node_count;
  uint64_t device_bytes;        /* device memory held by the scene           */
  uint64_t tag;                 /* unique per cg_scene_create (Scene::Impl::tag_) */
  double bvh_build_seconds;     /* time spent building the BVHs              */
  uint32_t bvh_host_builds;     /* trees built on the host ...               */
  uint32_t bvh_device_builds;   /* ... and on the GPU                        */
} cg_scene_info;
CG_API int cg_scene_get_info(cg_scene_t scene, cg_scene_info* out);

/* Where LoadScene builds its BVHs (binned SAH, 16 bins, with the same split
 * rule either way): 0 = on the GPU for trees of at least 16384 primitives when
 * a device is present, else on the host (default); 1 = always on the host;
 * 2 = always on the GPU (a failed device build fails the load).  No
 * counterpart in the reference, which builds median-split trees on the host
 * (src/pathtracing/blas.h:112-194, tlas.h:98-140). */
#define CG_BVH_BUILD_AUTO 0
#define CG_BVH_BUILD_HOST 1
#define CG_BVH_BUILD_DEVICE 2
CG_API int cg_set_bvh_build(int mode);
/* Builds one BVH over `count` boxes (6 floats each: lo xyz, hi xyz) on the
 * host (mode 1) or the GPU (mode 2) and returns its 64-byte BvhNode records
 * (when node_capacity suffices; *node_count is always set) and the primitive
 * permutation its leaves index.  For tests of the two builders. */
CG_API int cg_bvh_build(const float* boxes, uint32_t count, int mode, void* nodes_out,
                        uint32_t node_capacity, uint32_t* node_count,
                        uint32_t* order_out);

/* EmissivePrim (src/pathtracing/emissive_buffer.h:27-40), 80 bytes. */
typedef struct cg_emissive_prim {
  float v0[3]; float _p0;
  float v1[3]; float _p1;
  float v2[3]; float _p2;
  float emission[3];
  float area;
  float weight;
  float _pad[3];
} cg_emissive_prim;
/* AliasTableEntry (src/pathtracing/alias_table.h:14-17), 8 bytes. */
typedef struct cg_alias_entry {
  uint32_t alias;
  float prob;
} cg_alias_entry;

/* Copies the scene's emissive buffer and alias table, read back from the
 * device buffers the kernels sample, into host arrays of `capacity`
 * entries.  *count receives the entry count; with both arrays NULL the call
 * only reports the count. */
CG_API int cg_scene_read_emissive(cg_scene_t scene, cg_emissive_prim* prims,
                                  cg_alias_entry* alias, uint32_t capacity,
                                  uint32_t* count);

/* Builds an alias table on the host from `count` weights, the way
 * AliasTable's constructor does (src/pathtracing/alias_table.h:24-70). */
CG_API int cg_alias_build(const double* weights, uint32_t count,
                          cg_alias_entry* out);

/* ---- View (the hot path) ---------------------------------------------------
 * One progressive frame of `scene` from `camera` into the environment's film:
 * conf.sample_count samples per pixel, the running mean of CIE XYZ kept while
 * the scene and the camera stay the same (src/wgpu/frame_history.h:12-23,
 * compute.wesl:41-56), then the sRGB resolve (physics/srgb.wesl:5-27).
 * Synchronous up to the film on the device; read it with cg_film_read. */
CG_API int cg_view(cg_scene_t scene, const cg_camera* camera);

enum {
  CG_FILM_XYZ32F = 0,   /* running-mean XYZ, 3 floats per pixel (12 B/px)   */
  CG_FILM_RGBA8 = 1,    /* sRGB rgba8unorm, what the reference blits (4 B/px) */
  CG_FILM_RGB32F = 2    /* linear sRGB before the transfer curve (12 B/px)   */
};
/* Copies the film into `host` (row-major, row y = pixel.y of cameraRay). */
CG_API int cg_film_read(void* host, size_t bytes, int format);

/* ---- one view split across GPUs -------------------------------------------
 * No counterpart in the reference (its View() renders on one adapter).  For
 * spreading one large frame over several GPUs: each process renders a share
 * of every pixel's samples and the films are summed across GPUs (NCCL
 * all-reduce of the device films; backend.ViewSplit does all of it).
 *
 * cg_view_samples renders samples [sample_begin, sample_begin + sample_count)
 * of each pixel out of the conf's sample_count, with the sample keys of a
 * full cg_view frame 0 of the same seed, into the film as that range's share
 * of the pixel mean (every sample's term divided by sample_count of the
 * conf).  Films of ranges that partition [0, sample_count) add up to the full
 * frame (up to float summation order).  The film's running mean restarts:
 * the next cg_view begins a fresh accumulation.  An empty range writes a zero
 * film.  Ranges beyond the conf's sample_count are rejected (CG_E_INVALID). */
CG_API int cg_view_samples(cg_scene_t scene, const cg_camera* camera,
                           uint32_t sample_begin, uint32_t sample_count);
/* The environment's device film: float4 (X, Y, Z, 0) per pixel, row-major,
 * `*bytes` long, owned by the environment (valid until cg_init or cg_term).
 * Work on it on another stream must be complete before the next call of
 * this library that touches the film. */
CG_API int cg_film_device(void** film_xyzw, size_t* bytes);
/* Recomputes the rgba8 film from the float film (after it was changed on the
 * device, e.g. summed across GPUs), with the resolve's sRGB step. */
CG_API int cg_film_update_rgba8(void);
/* Frames accumulated so far in the film (iter_count + 1 after a View). */
CG_API int cg_film_frames(uint32_t* frames);

/* Per-View statistics of the last cg_view / batch on this environment. */
typedef struct cg_stats {
  uint64_t samples;          /* camera-path samples (pixels x spp)            */
  uint64_t extend_rays;      /* closest-hit rays traced (all depths)          */
  uint64_t shadow_rays;      /* shadow rays traced                            */
  uint64_t node_visits;      /* BVH node visits (counting build only, else 0) */
  uint64_t tri_tests;        /* triangle tests (counting build only, else 0)  */
  uint64_t inst_visits;      /* instance entries (counting build only, else 0)*/
  uint32_t chunks;           /* wavefront chunks the work was split into      */
  uint32_t kernel_launches;  /* kernels this library launched                 */
  float device_ms;           /* CUDA-event time of the device work            */
  uint32_t _pad;
  uint64_t nonfinite_samples; /* samples whose estimate was NaN or infinite:
                                 they add nothing to the film, so one bad
                                 sample cannot stay in a pixel's running mean */
} cg_stats;
CG_API int cg_last_stats(cg_stats* out);
/* 1 = count node visits / triangle tests in the traversal kernels (slower;
 * for the roofline's algorithmic bytes), 0 = off (default). */
CG_API int cg_set_counting(int enable);

/* Selects the RNG seed of the keyed sample streams (default 0). */
CG_API int cg_set_seed(uint32_t seed);

/* ---- spectral sampling --------------------------------------------------------
 * CG_SPECTRAL_REFERENCE (the default after cg_init): one wavelength per
 * sample, importance-sampled on [380, 720] nm by the 16-step bisection of
 * physics/wavelength.wesl:20-45, weighted as render.wesl:7-18 does.
 * CG_SPECTRAL_HERO: hero-wavelength sampling (no counterpart in the
 * reference): four wavelengths per sample, a hero uniform on [380, 780] nm
 * from the same random number and three more 100 nm apart (wrapped), all
 * carried by one sample tree drawn at the hero; a sample's XYZ is the mean of
 * the four wavelengths' terms over their uniform pdf.  Where the four would
 * draw the tree differently (a lobe whose heuristic vanishes at some of
 * them, a transmission whose refraction index varies with the wavelength)
 * the subtree carries the hero alone, weighted by 4, so the estimate keeps the
 * reference estimator's expectation at every wavelength; the images of the
 * two modes agree up to the reference's wavelength range (720-780 nm adds a
 * little X and Y) and the hero mode's lower colour noise.  Applies to cg_view,
 * cg_view_samples, cg_batch_render and servers created afterwards (each keeps
 * the mode it was created with); cg_render_noalloc always uses the reference
 * sampler.  A change restarts the film's running mean.  cg_init resets the
 * mode to CG_SPECTRAL_REFERENCE. */
enum { CG_SPECTRAL_REFERENCE = 0, CG_SPECTRAL_HERO = 1 };
CG_API int cg_set_spectral(int mode);
CG_API int cg_get_spectral(int* mode);

/* ---- Russian roulette ------------------------------------------------------------
 * No counterpart in the reference, whose sample trees end only at the depth
 * cut (trace.wesl:41-49).  With start_depth S > 0, every child ray spawned at
 * a hit of depth >= S (depth 0 = the camera ray's hit; S = 3 is "after the
 * third bounce") survives with probability q = min(1, its path weight t, the
 * largest over the wavelengths it carries) and then carries t / q; one
 * number from a stream keyed by the child decides.  The estimate keeps its
 * expectation and traces fewer rays.  0 (the default after cg_init) turns it
 * off.  Applies like cg_set_spectral; a change restarts the film's running
 * mean; cg_render_noalloc never uses it. */
CG_API int cg_set_roulette(uint32_t start_depth);

/* Per-kernel device time of the environment's View() / batch launches,
 * recorded with CUDA events on the launching stream while profiling is on
 * (batches then run without graph capture).  Index: CG_K_* */
enum { CG_K_GEN = 0, CG_K_EXTEND = 1, CG_K_SHADE = 2, CG_K_SHADOW = 3, CG_K_RESOLVE = 4,
       CG_K_COUNT = 5 };
typedef struct cg_profile {
  double ms[CG_K_COUNT];
  uint64_t launches[CG_K_COUNT];
} cg_profile;
CG_API int cg_set_profiling(int enable);
/* Reads and clears the accumulated per-kernel times. */
CG_API int cg_profile_read(cg_profile* out);

/* ---- ray queries (parity) --------------------------------------------------
 * Closest hit of `n` world-space rays, each 8 floats (ox, oy, oz, _, dx, dy,
 * dz, _), against the scene, as rayTraverseTlas/rayTraverseBlas compute it
 * (structural/bvh.wesl:52-186): t is the smallest Möller–Trumbore distance
 * below 1e6.  instance = -1 marks a miss. */
typedef struct cg_hit {
  float t, u, v;
  int32_t instance;
  int32_t triangle;  /* triangle index within the instance's mesh (original order) */
  int32_t _pad[3];
} cg_hit;
CG_API int cg_trace_closest(cg_scene_t scene, const float* rays, uint32_t n,
                            cg_hit* hits);

/* ---- batched form ------------------------------------------------------------
 * Renders many views of one scene, of uneven resolution and spp, in one
 * wavefront over shared ray queues.  Each view writes a fresh film (one frame,
 * no history).  `films_xyz` receives, per view, width*height*3 floats
 * (running-mean XYZ) concatenated in view order; `films_rgba8` (may be NULL)
 * receives width*height*4 bytes per view.  The launch sequence is captured as
 * a CUDA graph per (scene, batch) and replayed. */
typedef struct cg_view_desc {
  cg_camera camera;
  uint32_t width, height;
  uint32_t spp;
  uint32_t seed;        /* stream seed of this view's samples               */
} cg_view_desc;
CG_API int cg_batch_render(cg_scene_t scene, const cg_view_desc* views,
                           uint32_t view_count, float* films_xyz,
                           uint8_t* films_rgba8);

/* Wavefront tuning: rays per level queue (capacity), threads per block of the
 * traversal and shading kernels, and kernel variants.  0 = keep.  cg_autotune
 * searches these for a scene and a representative view (cg_autotune_views:
 * several views) and keeps the best. */
typedef struct cg_tuning {
  uint32_t queue_capacity;  /* rays per level queue, in [4096, 2^28] (default
                               64M: ~11.1 GB of path state per pipeline) */
  uint32_t extend_block;  /* threads per block of the traversal launches: a
                             multiple of 32 in [32, 256] (default 128; 0 = keep) */
  uint32_t shade_block;   /* the same for the shading launch (larger values
                             run as 256) */
  uint32_t use_graph;   /* 1 (default) = capture the launch sequence as a CUDA
                           graph and replay it: per batch in cg_batch_render,
                           per scene in cg_view (not while profiling);
                           always written (0 = launch directly) */
  uint32_t bvh_width;   /* 4 (default) or 2: node width the traversal walks */
  uint32_t persistent;  /* 1 (default) = persistent traversal warps that refill
                           idle lanes, 2 = one ray per thread, 3 = persistent
                           with postponed leaves on four-wide trees (a lane
                           parks a BLAS leaf and goes on with inner nodes;
                           the warp tests the parked triangles together),
                           0 = keep */
  uint32_t shade_sort;  /* order of the rays the shading kernel takes: 1 (default)
                           = grouped by material kind with a level-wide counting
                           sort, 3 = sorted within each block's slice, 2 = as
                           queued, 0 = keep */
  uint32_t box_bits;    /* four-wide child boxes: 32 (default) = floats in
                           128-byte nodes, 8 = 8-bit offsets in 64-byte nodes */
  uint32_t pipelines;   /* chunk pipelines of View() and cg_batch_render, 1 to
                           4: chunk k runs on stream k mod pipelines with that
                           stream's own ray queues (2 = default); 0 = keep */
  uint32_t traversal_threads;  /* threads per SM of the persistent traversal
                           grids: a multiple of extend_block in [extend_block,
                           1024] (1024 = default: the register file's limit at
                           64 registers per thread); fewer leave SM room for
                           another pipeline's shading launches to run beside
                           them; 0 = keep */
} cg_tuning;
CG_API int cg_set_tuning(const cg_tuning* tuning);
CG_API int cg_get_tuning(cg_tuning* out);
CG_API int cg_autotune(cg_scene_t scene, const cg_view_desc* view,
                       cg_tuning* best);
/* The same search with the timed batch made of `count` probe views (for
 * example a sample of a batch to be rendered).  The search is a coordinate
 * descent from the current tuning: kernel variant (node width and box bits,
 * persistent traversal, shading sort), then chunk pipelines (1-4), then queue
 * capacity, then block sizes; the fastest tuning is kept. */
CG_API int cg_autotune_views(cg_scene_t scene, const cg_view_desc* views,
                             uint32_t count, cg_tuning* best);

/* ---- served form -----------------------------------------------------------
 * A request loop over several resident scenes.  Requests are admitted while
 * their film plus path-state bytes fit the HBM budget, batched with the work
 * already on the GPU at chunk granularity (continuous batching), and
 * completed independently: a copy-out thread writes each finished film into
 * the caller's buffer while the GPU goes on with other requests.  Admission
 * and dispatch go shortest first (fewest samples left), except that a request
 * that has waited more than one second since its submit goes before every
 * younger one (oldest first), so a stream of small requests cannot starve a
 * large one.  A chunk holds one scene: that of the first request in this
 * order, filled with the scene's requests in the same order.  Per-request
 * sample streams are keyed by (request seed, pixel, sample), so a request's
 * result does not depend on what it was batched with or when it ran. */
typedef struct cg_server_s* cg_server_t;
typedef struct cg_request {
  uint32_t scene;       /* index into the server's scene list */
  cg_view_desc view;
} cg_request;
typedef struct cg_request_result {
  int32_t status;       /* CG_OK, CG_E_CANCELLED, ...              */
  uint32_t _pad;
  double submit_s, start_s, finish_s;   /* host clock (seconds)     */
} cg_request_result;
CG_API int cg_server_create(const cg_scene_t* scenes, uint32_t scene_count,
                            uint64_t hbm_budget_bytes, cg_server_t* out);
CG_API int cg_server_destroy(cg_server_t server);
/* Queues a request; its XYZ film (width*height*3 floats) is written into
 * `film_xyz`, which must stay valid until the request completes. */
CG_API int cg_server_submit(cg_server_t server, const cg_request* request,
                            float* film_xyz, uint64_t* request_id);
/* Waits up to timeout_ms (-1 = forever) for the request to complete. */
CG_API int cg_server_wait(cg_server_t server, uint64_t request_id,
                          int timeout_ms, cg_request_result* result);
CG_API int cg_server_cancel(cg_server_t server, uint64_t request_id);
typedef struct cg_server_stats {
  uint64_t submitted, completed, cancelled, rejected;
  uint64_t samples;
  uint32_t active, pending;
  uint64_t bytes_in_use, peak_bytes;
  uint64_t chunks;     /* wavefront chunks dispatched */
  double busy_s;       /* seconds with at least one chunk in flight (host clock,
                          dispatch to retirement) */
  double all_busy_s;   /* seconds with a chunk in flight on every lane */
  double copy_out_s;   /* seconds the copy-out thread spent waiting for finished
                          films' device-to-host copies and writing them into
                          the callers' buffers (overlaps the rendering) */
} cg_server_stats;
CG_API int cg_server_get_stats(cg_server_t server, cg_server_stats* out);

/* ---- rendering without allocation -------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory while they render (a host application that owns the memory budget
 * and hands the renderer only its buffers, a pooled allocator that forbids
 * driver allocations during a frame, a real-time loop that cannot afford an
 * allocation's implicit synchronisation): renders one fresh frame of `view`
 * (frame 0, keyed sample streams of view->seed) of `scene` with the caps of
 * `conf` into the caller's device film — `film_xyzw` holds float4 (X, Y, Z, 0)
 * per pixel, `film_rgba8` (may be NULL) uchar4 sRGB — on `stream` (NULL = the
 * default stream) of the current device, and returns when it is done.
 * It calls no cudaMalloc or cudaFree: the ray queues and tables live in a
 * library-owned device array of about 21.9 MB (131072 queued rays) that every
 * GPU loading the library holds until the process exits.  A view whose spp
 * cannot fit that array in one chunk is rejected with CG_E_INVALID.  The call
 * runs on the caller's current device, which must be the device and CUDA
 * context the scene was uploaded in (a scene from another device, or from
 * before a device reset, is rejected with CG_E_INVALID); `stream` must belong
 * to that device.  Films must be device (or managed) memory of that device;
 * a host pointer, a film the driver reports as smaller than the view
 * (16 B / 4 B per pixel), or a view of more than 2^32 - 1 pixels is rejected
 * with CG_E_INVALID before anything runs.  The first call in a device's
 * context sets the array up (finds its device address, fills the wavelength
 * table), and so does the first call after that context changes (a device
 * reset); make that first call before any stream capture.  All calls share
 * the array: calls that overlap on the GPU (other threads, other streams of
 * the same device) race and must be serialised by the caller. */
CG_API int cg_render_noalloc(cg_scene_t scene, const cg_conf* conf, const cg_view_desc* view,
                             void* film_xyzw, void* film_rgba8, void* stream);

/* Library version string. */
CG_API const char* cg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CG_CUDA_H_ */
