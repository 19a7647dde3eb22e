// Launch interface of the wavefront path-tracing kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/anacapa_b200.h"
#include "layout.h"

namespace ana {

// Queues are structure-of-arrays of float4, indexed by queue position.
//   extend queue: o (xyz, global path id), d (xyz, meta), beta (xyz, scene)
//     meta bits: 0..7 bounce, 8 specular-bounce flag, 9 first-hit AOVs taken,
//     16..31 next sampler dimension
//   hit record:   (t, prim, u, v) and, for curve hits, (tangent xyz, strand v)
//     prim: leaf-order triangle index, 0x80000000 | segment index, or ~0 (miss)
//   shadow queue: o (xyz, path id), d (xyz, tmax), contribution (xyz, scene)
//   MIS queue:    o (xyz, path id), d (xyz, -), contribution without Li (xyz, scene)
struct Queues {
    float4* ext_o[2];
    float4* ext_d[2];
    float4* ext_b[2];
    float4* hit0;
    float4* hit1;
    float4* sh_o;
    float4* sh_d;
    float4* sh_c;
    float4* mis_o;
    float4* mis_d;
    float4* mis_c;
    float* L;  // 3 floats per path of the chunk
    float* aov;  // 6 floats per path of the chunk: first-hit albedo, shading normal
};

// Per-bounce device counters: [bounce][0] extend queue length, [1] shadow
// queue length, [2] MIS queue length, [3..5] the persistent kernels' fetch
// counters of extend, shadow and MIS. Zeroed per chunk.
constexpr int kCountersPerBounce = 8;

// A run of whole pixels of one scene inside a chunk. Chunks are cut in the
// global path space at pixel boundaries, so a chunk may span several scenes.
struct ChunkSeg {
    uint32_t scene;        // scene index
    uint32_t first_pixel;  // first pixel (within the scene's film)
    uint32_t num_pixels;
    uint32_t local_pixel;  // chunk-local index of the first pixel
    uint32_t local_path;   // chunk-local index of the first path
    uint32_t pad[3];
};

// Path-replay adjoint state (used only by the backward pass). Gradient
// accumulators: 8 floats per material (albedo rgb, roughness, emission rgb,
// -), then 4 per light (Le rgb, -). Material and light ids in the payloads
// are global indices; kNoKey marks an absent one.
//   ext_g0/1: pending continuation gradient of the vertex that spawned the
//             extend entry: d log f / d albedo (xyz), material (w bits);
//             d log f / d roughness (xyz)
//   sh_g0/1:  NEE term: delta * d contribution / d albedo (xyz), / d roughness
//             summed over channels (w); delta * d contribution / d Le (xyz),
//             material (low 16 bits) | light (high 16 bits) (w bits)
//   mis_g0/1: MIS term without Li: delta * dK / d albedo (xyz), material (w
//             bits); delta * dK / d roughness (xyz)
//   sh_vis:   1 when the shadow ray was unoccluded
//   mis_res:  Li of the MIS ray (xyz), material hit (w bits, kNoKey: none)
struct AdjQueues {
    float4* ext_g0[2];
    float4* ext_g1[2];
    float4* sh_g0;
    float4* sh_g1;
    float4* mis_g0;
    float4* mis_g1;
    uint32_t* sh_vis;
    float4* mis_res;
    const float* Lp;       // primal radiance of every path of the chunk (3 floats)
    float* dL;             // dLoss / dL of every path of the chunk (3 floats)
    const float* d_image;  // dLoss / d pixel, film layout (3 floats per pixel)
    float* grad;
    uint32_t num_materials;
};
constexpr uint32_t kNoKey = 0xFFFFFFFFu;

struct Params {
    DevScene S;
    Queues q;
    AdjQueues a;
    ana_film_pixel* film;      // batch film (all scenes)
    float* aov;                // AOV film, 8 floats per pixel: albedo (r, g, b, w),
                               // normal (x, y, z, w); null: no AOVs
    uint32_t* counters;        // this chunk's counters
    uint32_t* err;             // device error word (bit 0: traversal stack overflow)
    unsigned long long* work;  // [node fetches, triangle tests, segment tests] (count mode)
    const ChunkSeg* segs;      // this chunk's pixel runs
    uint32_t num_segs;
    uint32_t chunk_first_path; // global path id of the chunk's first path
    uint32_t chunk_paths, chunk_pixels;
    uint32_t bounce;
};

struct LaunchCfg {
    int block;       // threads per block for the stage kernels
    int grid_cap;    // blocks for grid-stride kernels over the chunk capacity
    int stage_grid;  // blocks for stage kernels whose item count is only known on
                     // the device (shade, adjoint resolution): four waves of
                     // the most blocks an SM can hold, so sparse late bounces do
                     // not pay for launching blocks sized for a full chunk
    int persistent;  // traversal schedule: 1 persistent warps with refill, 0 thread per ray
};

// Loads every kernel and caches its resident grid on the current device.
// Called when a context is created, so a later stream capture launches only.
void prime_kernels();

void launch_generate(const Params& p, const LaunchCfg& c, cudaStream_t s);
void launch_extend(const Params& p, const LaunchCfg& c, cudaStream_t s, bool count_work);
void launch_shade(const Params& p, const LaunchCfg& c, cudaStream_t s);
void launch_shadow(const Params& p, const LaunchCfg& c, cudaStream_t s);
void launch_mis(const Params& p, const LaunchCfg& c, cudaStream_t s);
void launch_film(const Params& p, const LaunchCfg& c, cudaStream_t s);

// Adjoint replay stages: the shade / shadow / MIS kernels of the forward pass
// with the gradient bookkeeping compiled in (identical sampling decisions),
// the per-path delta set-up, and the resolution of the NEE and MIS gradient
// payloads once their rays are traced.
void launch_adj_init(const Params& p, const LaunchCfg& c, cudaStream_t s);
void launch_shade_adj(const Params& p, const LaunchCfg& c, cudaStream_t s);
void launch_shadow_adj(const Params& p, const LaunchCfg& c, cudaStream_t s);
void launch_mis_adj(const Params& p, const LaunchCfg& c, cudaStream_t s);
void launch_adj_direct(const Params& p, const LaunchCfg& c, cudaStream_t s);
// times: one ray time per ray (motion-blurred meshes), or null (time 0)
void launch_trace_batch(const DevScene& S, uint32_t scene, const float* rays, const float* times, size_t n,
                        ana_hit* out, int occlusion, uint32_t* fetch, uint32_t* err, int persistent, cudaStream_t s);

// IMaterial::evaluate / sample of one material over n queries (ana_bsdf_batch).
void launch_bsdf_query(const DevMaterial& m, const ana_bsdf_query* q, uint32_t n, ana_bsdf_result* out,
                       cudaStream_t s);

// Fixed device scratch of the allocation-free trace entry point: a 256-byte
// header (the scene record at 0, the error word at kNoAllocErrOffset and the
// persistent schedule's work counter 4 bytes after it), then room for
// ANA_TRACE_NOALLOC_MAX_RAYS rays of 32 bytes, then as many 32-byte hits.
constexpr size_t kNoAllocHeader = 256;
constexpr size_t kNoAllocErrOffset = 240;
constexpr size_t kNoAllocRays = kNoAllocHeader;
constexpr size_t kNoAllocHits = kNoAllocRays + size_t(ANA_TRACE_NOALLOC_MAX_RAYS) * 32;
constexpr size_t kNoAllocBytes = kNoAllocHits + size_t(ANA_TRACE_NOALLOC_MAX_RAYS) * sizeof(ana_hit);
static_assert(sizeof(DevSceneRec) <= kNoAllocErrOffset, "scene record overlaps the error word");
static_assert(sizeof(ana_hit) == 32, "hit record size");

// Device address of that scratch on `device`, which must be the current
// device. The first call per device looks it up (cudaGetSymbolAddress) and
// caches it with the current context; later calls in the same context only
// read the cache (after a device reset the new context looks it up again).
cudaError_t noalloc_trace_scratch(int device, unsigned char** base);

}  // namespace ana
