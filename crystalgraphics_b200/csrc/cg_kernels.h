// cg_kernels.h — launch interface of the wavefront kernels (cg_kernels.cu).
//
// One View() frame is a sequence of chunks.  A chunk is a run of whole pixels
// (all their samples) from one or more views; per chunk the launches are
//   gen -> D x (extend -> shade -> shadow) -> resolve
// over ping-pong ray queues in HBM.  Every launch reads its work count from
// device memory, so the sequence needs no host synchronisation and can be
// captured as a CUDA graph.
#ifndef CG_KERNELS_H_
#define CG_KERNELS_H_

#include <cuda_runtime.h>

#include <cstdint>

#include "cg_types.h"

namespace cg {

// Per-view constants (device).  An entry covers image pixels
// [pixel_base, pixel_base + pixel_count) of a view, so a chunk can hold slices
// of several views.
struct ViewDev {
  float pos[3], dir[3], dx[3], dy[3];  // camera basis of cameraRay (compute.wesl:64-79)
  uint32_t width, height, spp, seed;
  uint32_t frame;              // iter_count: 0 starts a fresh running mean
  float sample_weight;         // 1 / (frame + 1)
  uint32_t pixel_base;         // first image pixel this entry covers
  uint32_t pixel_count;        // image pixels this entry covers
  uint32_t sample_base;        // per-pixel index of the first sample rendered (sample keys)
  uint32_t spp_total;          // divisor of the pixel mean: the full frame's spp (0: spp)
  uint64_t pixel_offset;       // first global pixel index of this entry
  uint64_t sample_offset;      // first global sample index of this entry
  float4* film;                // running-mean XYZ (w unused)
  uchar4* rgba;                // sRGB rgba8 (may be null)
};

// Sample caps of a frame (PathTraceConf, after clamping).
struct Caps {
  uint32_t trace_depth, transport_cap, emission_cap, diffuse_cap, rough_cap;
};

// Wavefront buffers (device).
struct WaveBuffers {
  float4* ray_o[2];      // origin.xyz, path weight
  float4* ray_d[2];      // dir.xyz, node key bits
  uint32_t* ray_slot[2];
  float4* hit;           // t, u, v, triangle slot bits
  int32_t* hit_inst;     // -1 = miss
  float4* sh_o;          // shadow origin.xyz, contribution
  float4* sh_d;          // shadow dir.xyz, tmax
  uint32_t* sh_slot;
  float* s_L;            // per sample slot: accumulated radiance
  float* s_lambda;
  float* s_prob;
  uint8_t* shade_key;    // per queued ray: its shading key (the global shading sort)
  uint32_t* shade_perm;  // queued rays in shading-key order
  uint32_t* counts;      // [0], [1] ray queues, [2] shadow queue, [3], [4] traversal work
                         // counters, [6] block ticket, [8..26] rays per shading key,
                         // [32..50] scatter cursors
  unsigned long long* stats;  // [0] extend rays [1] shadow rays [2] nodes [3] tris [4] insts
  uint32_t* status;      // bit 0: traversal stack overflow, bit 1: queue overflow
  uint32_t capacity;     // rays per queue (and shadow rays)
  uint32_t sample_capacity;
  // hero-wavelength mode (hero != 0): per queued ray the path weights of the
  // three other wavelengths (x, y, z) and flags (w: bit 0 = the hero alone
  // below a hit where the four wavelengths sample differently); per shadow ray
  // the other wavelengths' light-sample terms; per sample slot the four
  // wavelengths' radiance (s_lambda then holds the hero's offset above 380 nm)
  float4* ray_w[2];
  float4* sh_w;
  float4* s_L4;
  uint32_t hero;
  // per queued ray of a level that draws light samples: the hit position of
  // its parent (xyz) and its balance-heuristic denominator without the light
  // term (w; -1: the ray's weight is final), and the lobe value the weight is
  // still to be multiplied by (defer_dist; ray_o.w holds the parent's weight
  // meanwhile).  k_light_pdf adds the light-pdf term and completes the weight
  // after the shading launches.  Null (and with a per-block or no shading
  // order, or where roulette is active): shading completes the weights itself.
  float4* defer;
  float* defer_dist;
  // hero-wavelength mode: per deferred ray the other three wavelengths' lobe
  // values (xyz; ray_w.xyz holds the parent's weights meanwhile)
  float4* defer_w;
};

struct FrameConst {
  const ViewDev* views;
  uint32_t view_count;
  Caps caps;
  const float* wl_tree;  // 65535 cdf values (sampleWavelengthCdf bisection)
  const float* wl_const; // [0] total integral, [1] total / 3
  uint32_t roulette = 0; // Russian roulette from this hit depth on (0 = off, as the reference)
};

struct ChunkDesc {
  uint64_t sample_begin;
  uint64_t pixel_begin;
  uint32_t sample_count;
  uint32_t pixel_count;
};

// How the shading kernel orders a level's rays: as queued, by a counting
// sort of each block's slice, or by a counting sort of the whole level (the
// closest-hit kernel counts keys, a scatter kernel builds the permutation; no
// barriers in the shading kernel).
enum ShadeSort : int { kShadeSortNone = 0, kShadeSortBlock = 1, kShadeSortGlobal = 2 };

struct LaunchShape {
  uint32_t extend_block = 128;
  uint32_t shade_block = 128;
  uint32_t grid_extend = 0;  // 0: derived from the SM count
  uint32_t grid_shade = 0;
  int nodes = kNodesWide4;   // NodeFormat of the traversal
  bool persistent = true;    // persistent warps with lane refill
  bool spec = false;         // with persistent four-wide closest hits: postponed leaves
  uint32_t traversal_threads = 1024;  // threads per SM of the persistent traversal grids
  int shade_sort = kShadeSortGlobal;  // ShadeSort: order of the rays the shading kernel takes
};

void launchWavelengthTree(float* tree, float* consts, cudaStream_t s);
void launchGen(const FrameConst& fc, const WaveBuffers& wb, const ChunkDesc& ch, cudaStream_t s);
// With the level-wide shading order (ls.shade_sort == kShadeSortGlobal) the
// launch also writes the level's shading keys; `cut`: the level is shaded at
// or beyond the depth cut.
void launchExtend(const SceneView& sc, const WaveBuffers& wb, int parity, bool counting,
                  const LaunchShape& ls, bool cut, cudaStream_t s);
// Returns the number of kernels launched (one, or with the global sort the
// scatter and one shading launch per lobe group: four, and k_light_pdf after
// them on a light-sampling level with wb.defer set: five).
// `light`: the level can draw light samples (false leaves the light-sample code
// out of the level's global-order shading launches).
int launchShade(const SceneView& sc, const FrameConst& fc, const WaveBuffers& wb, int depth,
                int parity, const LaunchShape& ls, cudaStream_t s, bool light = true);
void launchShadow(const SceneView& sc, const WaveBuffers& wb, bool counting,
                  const LaunchShape& ls, cudaStream_t s);
void launchResolve(const FrameConst& fc, const WaveBuffers& wb, const ChunkDesc& ch,
                   cudaStream_t s);
// Packs a float4 film to three floats per pixel (XYZ, or linear sRGB).
void launchFilmPack(const float4* film, float* out, size_t npx, bool rgb, cudaStream_t s);
// Re-resolves the rgba8 film from the float4 XYZ film (the resolve's sRGB step).
void launchFilmRgba8(const float4* film, uchar4* rgba, size_t npx, cudaStream_t s);
void launchTraceClosest(const SceneView& sc, const float4* rays, uint32_t n, float4* out_tuv,
                        int4* out_ids, uint32_t* status, int nodes, cudaStream_t s);

int smCount();
// Sets kernel attributes on the current device (once per device, outside any
// stream capture).
void configureKernels();

}  // namespace cg

#endif
