/*
 * cg_oracle.h — CPU oracle for the View() path-tracing hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C++ restatement of the reference
 * ray847/CrystalGraphics (WGSL compute shader + host scene packing), used as
 * the checker for the CUDA backend and as the timed CPU baseline.  The
 * product (libcg_cuda.so, the crystal::graphics layer, the Python package)
 * never links, loads or calls it; only tests/, __graft_entry__.smoke() and
 * bench.py's CPU arms do.
 *
 * Parity status: the reference has no tests, golden vectors or CPU path
 * tracer.  Pins used here:
 *   - alias tables: checked bit-exactly against the reference's own
 *     src/pathtracing/alias_table.h compiled unmodified (oracle/_ref);
 *   - everything else is a restatement of the cited WGSL/C++ lines; its
 *     parity against the reference's own execution is unpinned (the WGSL
 *     cannot run without a graphics API).
 * Every function cites the reference file:line it follows.
 */
#ifndef CG_ORACLE_H_
#define CG_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#include "../include/cg_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_scene_s* oracle_scene_t;

/* Builds the restated SceneData (src/pathtracing/scene_data.h:38-54): BLAS
 * per mesh (blas.h), TLAS (tlas.h), emissive buffer (emissive_buffer.h),
 * alias table (alias_table.h), environment (scene_data.h:57-98). */
oracle_scene_t oracle_scene_create(const cg_scene_desc* desc);
void oracle_scene_destroy(oracle_scene_t scene);
/* Single-threaded seconds the create call spent in each host packing stage,
 * as the reference runs them on the host (src/environment.cpp:69-74): [0] the
 * median-split BLAS builds (blas.h:112-194, one per mesh), [1] the TLAS build
 * (tlas.h:98-140), [2] the emissive buffer (emissive_buffer.h:44-100), [3]
 * the alias table (alias_table.h:26-70). */
int oracle_scene_pack_seconds(oracle_scene_t scene, double* out);

uint32_t oracle_emissive_count(oracle_scene_t scene);
/* Copies the emissive prims, alias entries and the float total weight. */
int oracle_emissive(oracle_scene_t scene, cg_emissive_prim* prims,
                    cg_alias_entry* alias, float* total_weight);
/* Restated AliasTable constructor (alias_table.h:24-70). */
int oracle_alias_build(const double* weights, uint32_t count,
                       cg_alias_entry* out);

/* Closest hit per ray, restating rayTraverseTlas / rayTraverseBlas /
 * rayIntersectTriangle / rayIntersectAABB (structural/bvh.wesl:52-221,
 * math/geometric.wesl:5-26) op for op.  rays: n x 8 floats
 * (ox, oy, oz, _, dx, dy, dz, _).  t2 (may be NULL) receives, per ray, the
 * second-smallest hit distance over distinct (instance, triangle) pairs, or
 * 1e6 — used to exclude ulp-level ties from bit-exact comparisons. */
int oracle_trace_closest(oracle_scene_t scene, const float* rays, uint32_t n,
                         cg_hit* hits, float* t2, int threads);

enum {
  ORACLE_RNG_REFERENCE = 0, /* one PCG-hash stream per pixel, seeded with the
                               pixel index on frame 0 and persisted, consumed
                               depth-first (compute.wesl:41-56, rng.wesl) */
  ORACLE_RNG_KEYED = 1      /* one stream per sample-tree node, keyed by
                               (seed, frame, pixel, sample, child path): the
                               streams the CUDA kernels use */
};

enum {
  ORACLE_SPECTRAL_REFERENCE = 0, /* one wavelength per sample, importance-sampled
                                    by bisection of the CIE-sum CDF on
                                    [380, 720] (physics/wavelength.wesl:20-45) */
  ORACLE_SPECTRAL_HERO = 1       /* four wavelengths per sample: a hero uniform
                                    on [380, 780] and three rotated by 100 nm;
                                    directions follow the hero, the others
                                    weigh the same paths, and a refraction
                                    whose index varies across the four keeps
                                    the hero alone (weight x 4) below it     */
};

typedef struct oracle_render_args {
  cg_conf conf;            /* render size, spp, depth, sample caps          */
  cg_camera camera;
  uint32_t iter_count;     /* frame index (0 = fresh film)                  */
  uint32_t rng_mode;       /* ORACLE_RNG_*                                  */
  uint32_t seed;           /* keyed-mode stream seed                        */
  uint32_t threads;        /* host threads (0 = all)                        */
  uint32_t prune;          /* 1 = t-bounded traversal (same closest hit
                              except exact ties; faster), 0 = as reference  */
  uint32_t pixel_begin, pixel_end;  /* render only this pixel range
                              (end 0 = all); other pixels are left as is  */
  uint32_t spectral;       /* ORACLE_SPECTRAL_*                             */
  uint32_t roulette;       /* Russian roulette from this hit depth on (0 = off,
                              as the reference): a child survives with
                              q = min(1, its path weight) and carries weight / q */
  uint32_t _pad;
} oracle_render_args;

/* One View() frame: for every pixel, render() + film update + rng seed
 * update (compute.wesl:32-62).  film_xyz: W*H*3 floats (in/out running mean),
 * seeds: W*H u32 (in/out, reference mode), both may be updated in place.
 * stats (may be NULL): [0] extend rays, [1] shadow rays, [2] node visits,
 * [3] triangle tests, [4] samples whose estimate was not finite (they add
 * nothing to the film, as in the library). */
int oracle_render(oracle_scene_t scene, const oracle_render_args* args,
                  float* film_xyz, uint32_t* seeds, uint64_t* stats);

/* Spectral helpers, for unit tests. */
float oracle_sample_wavelength(float u, float* prob);
void oracle_xyz_match(float wavelength, float* xyz);
float oracle_rgb_to_reflectance(const float* rgb, float wavelength);
float oracle_rgb_to_radiance(const float* rgb, float wavelength);
void oracle_xyz_to_srgb(const float* xyz, float* rgb01);
uint32_t oracle_rng_sequence(uint32_t seed, uint32_t n, float* out);
uint32_t oracle_sample_key(uint32_t seed, uint32_t frame, uint32_t pixel,
                           uint32_t sample);

#ifdef __cplusplus
}
#endif

#endif
