// Wavefront path tracing on sm_100a: one kernel per stage of
// PathIntegrator::Li (src/integrator/PathIntegrator.cpp:71-265).
//
//   generate  camera rays for a chunk of paths      (renderTile, 33-38)
//   extend    closest hit of every live path         (Li, 81)
//   shade     emission, NEE light + BSDF samples, continuation, RR (Li 83-160,
//             estimateDirect 166-265); emits shadow, MIS and extend queues
//   shadow    any-hit of the NEE shadow rays         (shadowTransmittance)
//   mis       closest hit of the BSDF-sampled MIS rays; adds emitter Le / env
//   film      per-pixel reduction into the film      (renderTile 43-57)
//
// A render is a batch of scenes (a plain render is a batch of one): every
// path carries its scene index, and the scene record gives its BVH roots,
// slot and light ranges, camera, spp and depth. Chunks are cut in the global
// path space at pixel boundaries, so one chunk can hold paths of several
// scenes and the queues stay full across scene boundaries.
//
// Queues are SoA float4 arrays. Each stage kernel appends to the next queue
// with a block-level allocation: warp ballots give each lane its rank, one
// shared-memory scan over the block's warps and a single atomicAdd per block
// reserve a contiguous range, so every warp writes a contiguous, coalesced run.
#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "kernels.h"
#include "sampler.cuh"
#include "shade.cuh"
#include "traverse.cuh"

namespace ana {

constexpr uint32_t kMiss = 0xFFFFFFFFu;
constexpr int kMaxBlock = 1024;
constexpr int kPersistBlock = 256;    // traversal kernels: 8 warps per block
constexpr int kPersistMinBlocks = 5;  // persistent schedule: 5 resident blocks/SM (<= 51 registers)
// k_shade runs at most 256-thread blocks: three resident per SM (80 registers,
// spilling to L1) for the forward kernel without fiber code measured 5 % faster
// than two at 128 registers; the kernels compiled for a subset of the material
// and light classes fit four (64 registers: throughput frame's shade stage 77.4
// against 78.5 ms at three); the fiber and adjoint variants keep two
constexpr int kShadeBlock = 256;

// Reserves one slot per thread and queue where that thread's want flag is
// set, for three queues at once: warp ballots give each lane its rank, threads
// 0-2 scan the block's warp counts of one queue each and reserve the block's
// range with one atomicAdd. Must be reached by every thread of the block.
__device__ __forceinline__ void block_push3(bool w0, bool w1, bool w2, uint32_t* c0, uint32_t* c1, uint32_t* c2,
                                            uint32_t& k0, uint32_t& k1, uint32_t& k2) {
    __shared__ uint32_t s_cnt[3][kMaxBlock / 32];
    __shared__ uint32_t s_base[3];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nwarps = (blockDim.x + 31u) >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t m0 = __ballot_sync(0xFFFFFFFFu, w0), m1 = __ballot_sync(0xFFFFFFFFu, w1),
                   m2 = __ballot_sync(0xFFFFFFFFu, w2);
    if (lane == 0) {
        s_cnt[0][warp] = __popc(m0);
        s_cnt[1][warp] = __popc(m1);
        s_cnt[2][warp] = __popc(m2);
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        uint32_t* cnt = s_cnt[threadIdx.x];
        uint32_t run = 0;
        for (uint32_t w = 0; w < nwarps; ++w) {
            const uint32_t c = cnt[w];
            cnt[w] = run;
            run += c;
        }
        uint32_t* ctr = threadIdx.x == 0 ? c0 : (threadIdx.x == 1 ? c1 : c2);
        s_base[threadIdx.x] = run ? atomicAdd(ctr, run) : 0u;
    }
    __syncthreads();
    k0 = s_base[0] + s_cnt[0][warp] + __popc(m0 & lt);
    k1 = s_base[1] + s_cnt[1][warp] + __popc(m1 & lt);
    k2 = s_base[2] + s_cnt[2][warp] + __popc(m2 & lt);
    __syncthreads();  // s_cnt / s_base are reused by the next call
}

__device__ __forceinline__ float4 pack(float3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
__device__ __forceinline__ float4 pack_u(float3 v, uint32_t w) {
    return make_float4(v.x, v.y, v.z, __uint_as_float(w));
}

// Scene of a global path id: the last scene whose first path is <= gid.
__device__ __forceinline__ uint32_t scene_of(const DevScene& S, uint32_t gid) {
    uint32_t lo = 0, hi = S.num_scenes;  // invariant: offset[lo] <= gid < offset[hi]
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(S.scene_path_offset + mid) <= gid) lo = mid;
        else hi = mid;
    }
    return lo;
}

// floor(n / d) from m = ceil(2^64 / d) (0 encodes d = 1): m*d = 2^64 + e with
// e < d, so n*e < 2^64 for every 32-bit n and the high word of n*m is the
// quotient. The scene record carries m for its spp and rectangle width.
__device__ __forceinline__ uint32_t div_magic(uint32_t n, uint64_t m) {
    return m ? uint32_t(__umul64hi(uint64_t(n), m)) : n;
}

__device__ __forceinline__ void path_coords(const DevSceneRec& R, uint32_t gid, uint32_t& px, uint32_t& py,
                                            uint32_t& sidx) {
    uint32_t local = gid - R.path_offset;
    uint32_t pixel = div_magic(local, R.spp_div);
    sidx = R.sample_start + (local - pixel * R.spp);
    const uint32_t ly = div_magic(pixel, R.rect_w_div);
    px = R.rect_x0 + (pixel - ly * R.rect_w);
    py = R.rect_y0 + ly;
}

// The ray time of a path: Camera::generateRay's shutterOpen + timeU *
// (shutterClose - shutterOpen) with timeU its sample dimension 4; every ray of
// the path carries it (PathIntegrator.cpp:148-149, 185, 221).
__device__ __forceinline__ float path_time(const DevSceneRec& R, uint32_t gid) {
    uint32_t px, py, sidx;
    path_coords(R, gid, px, py, sidx);
    SampleStream ss{R.seed, px, py, sidx, 4};
    const float u = ss.next();
    return xadd(R.cam.shutter_open, xmul(u, xsub(R.cam.shutter_close, R.cam.shutter_open)));
}

// Film index of an item's pixel (its index within the item's rectangle).
__device__ __forceinline__ size_t film_index(const DevSceneRec& R, uint32_t pixel) {
    const uint32_t ly = div_magic(pixel, R.rect_w_div);
    return size_t(R.film_offset) + size_t(R.rect_y0 + ly) * R.film_w + R.rect_x0 + (pixel - ly * R.rect_w);
}

__device__ __forceinline__ void add_L(const Params& p, uint32_t gid, float3 v) {
    size_t li = size_t(gid - p.chunk_first_path) * 3;
    p.q.L[li + 0] += v.x;
    p.q.L[li + 1] += v.y;
    p.q.L[li + 2] += v.z;
}

// ---------------------------------------------------------------------------
// generate: Camera::generateRay (include/anacapa/integrator/IIntegrator.h:90-143)
// with jitter = dims 0,1, lens = dims 2,3, time = dim 4. The pinhole ray is
// computed with every operation rounded on its own (bit-identical origin and
// direction to the reference built without contraction).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_generate(const __grid_constant__ Params p) {
    const uint32_t n = p.chunk_paths;
    if (blockIdx.x == 0 && threadIdx.x == 0) p.counters[0] = n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t gid = p.chunk_first_path + i;
        const uint32_t sc = scene_of(p.S, gid);
        const DevSceneRec& R = p.S.scenes[sc];
        const DevCamera& cam = R.cam;
        uint32_t px, py, sidx;
        path_coords(R, gid, px, py, sidx);
        SampleStream ss{R.seed, px, py, sidx, 0};
        float jx = ss.next(), jy = ss.next();
        float lx = ss.next(), ly = ss.next();
        float tu = ss.next();
        (void)tu;  // shutter time: static scenes only
        float s = xdiv(xadd(__uint2float_rn(px), jx), __uint2float_rn(cam.width));
        float t = xdiv(xadd(__uint2float_rn(cam.height - 1u - py), jy), __uint2float_rn(cam.height));
        float3 target = xadd3(xadd3(cam.lower_left, xmul3(cam.horizontal, s)), xmul3(cam.vertical, t));
        float3 o = cam.origin, d;
        if (cam.aperture <= 0.f) {
            d = xnormalize(xsub3(target, o));
        } else {
            // thin lens, concentric disk mapping (IIntegrator.h:114-142)
            float ax = 2.f * lx - 1.f, ay = 2.f * ly - 1.f, dx, dy;
            if (ax == 0.f && ay == 0.f) {
                dx = dy = 0.f;
            } else if (fabsf(ax) >= fabsf(ay)) {
                float ph = (kPi / 4.f) * (ay / ax);
                dx = ax * cosf(ph);
                dy = ax * sinf(ph);
            } else {
                float ph = (kPi / 2.f) - (kPi / 4.f) * (ax / ay);
                dx = ay * cosf(ph);
                dy = ay * sinf(ph);
            }
            float3 lens = o + cam.basis_u * (dx * cam.aperture) + cam.basis_v * (dy * cam.aperture);
            float3 pd = normalize(target - o);
            float3 fp = o + pd * cam.focal_distance;
            o = lens;
            d = normalize(fp - lens);
        }
        uint32_t meta = (ss.dim << 16);  // bounce 0, not specular
        p.q.ext_o[0][i] = pack_u(o, gid);
        p.q.ext_d[0][i] = pack_u(d, meta);
        p.q.ext_b[0][i] = make_float4(1.f, 1.f, 1.f, __uint_as_float(sc));
        size_t li = size_t(i) * 3;
        p.q.L[li] = 0.f;
        p.q.L[li + 1] = 0.f;
        p.q.L[li + 2] = 0.f;
        if (p.aov)  // a camera ray that misses keeps black AOVs
            for (int k = 0; k < 6; ++k) p.q.aov[6 * size_t(i) + k] = 0.f;
    }
}

// ---------------------------------------------------------------------------
// Closest hit over triangles then curves (CurveBrute::trace, CurveBrute.cpp:398-440).
// ---------------------------------------------------------------------------
struct SceneHit {
    float t, u, v;
    uint32_t prim;  // leaf-order triangle, 0x80000000 | segment, or kMiss
    float3 tang;
    float tseg;
};

// Packs a finished traversal (triangles, then strictly closer ribbons when
// kCurves). kCurves = false compiles the curve code out of kernels for
// triangle-only batches.
template <bool kCurves>
__device__ __forceinline__ SceneHit finish_closest(const Traversal& T, float tmax) {
    SceneHit h;
    h.t = T.tri >= 0 ? T.closest : tmax;
    h.u = T.u;
    h.v = T.v;
    h.prim = T.tri >= 0 ? uint32_t(T.tri) : kMiss;
    h.tang = f3(0.f, 0.f, 0.f);
    h.tseg = 0.f;
    if (kCurves && T.seg >= 0) {
        h.t = T.closest;
        h.prim = 0x80000000u | uint32_t(T.seg);
        h.tang = T.tang;
        h.tseg = T.tseg;
        h.u = 0.f;
        h.v = T.tseg;
    }
    return h;
}

template <bool kCurves>
__device__ __forceinline__ bool finish_any(const Traversal& T) {
    return T.tri >= 0 || (kCurves && T.seg >= 0);
}

__device__ __forceinline__ void warp_add_work(unsigned long long* work, const Counters& cnt) {
    unsigned long long a = cnt.nodes, b = cnt.prims, c = cnt.segs, e = cnt.cnodes;
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_down_sync(0xFFFFFFFFu, a, off);
        b += __shfl_down_sync(0xFFFFFFFFu, b, off);
        c += __shfl_down_sync(0xFFFFFFFFu, c, off);
        e += __shfl_down_sync(0xFFFFFFFFu, e, off);
    }
    if ((threadIdx.x & 31u) == 0) {
        atomicAdd(work + 0, a);
        atomicAdd(work + 1, b);
        atomicAdd(work + 2, c);
        atomicAdd(work + 3, e);
    }
}

// Runs the traversal of queue entries [0, n) in one of two schedules:
//   kPersist: persistent warps with per-lane refill (persistent_traverse);
//   otherwise one thread per ray over a grid-stride loop.
// Both use the same interior/leaf steps, so results are identical.
template <bool kAny, bool kCount, bool kPersist, bool kCurves, bool kMotion = false, bool kPark = kAny,
          class Load, class Done>
__device__ __forceinline__ void run_traversal(const DevScene& S, uint32_t n, uint32_t* fetch, uint32_t* err,
                                              Counters* cnt, Load load, Done done) {
    if constexpr (kPersist) {
        persistent_traverse<kAny, kCount, kCurves, kMotion, kPark>(S, n, fetch, err, cnt, load, done);
    } else {
        uint2 stack[kMaxStack4];
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
            Ray ray;
            uint32_t root, segRoot;
            load(i, ray, root, segRoot);
            Traversal T;
            trav_init(T, ray, root);
            while (true) {
                while (true) {
                    while (!T.exhausted) {
                        if (!(T.cur & 0x80000000u)) {
                            node_step<kAny, kCount, kCurves>(T, S, stack, err, cnt);
                        } else if (leaf_step<kAny, kCount, kCurves, kMotion>(T, S, T.cur, cnt)) {
                            T.exhausted = true;
                        } else if (!trav_pop<kAny>(T, stack)) {
                            T.exhausted = true;
                        }
                    }
                    if (stage_done<kAny, kCurves>(T, ray.d, segRoot)) break;
                }
                Ray next;
                if (!trace_again(done, i, T, next)) break;
                trav_init(T, next, root);
            }
        }
    }
}

// Persistent triangle kernels fit 5 blocks per SM (48 registers, a few spills
// to L1; on the throughput frame 451 ms against 467 ms at 4 blocks and 64
// registers, and 520 ms at 6 blocks and 40); the motion variants (object-ray
// state) keep 4 and 64 registers; with the curve stage they take 3 (80
// registers with spills to L1: the ribbon test's state; the hair frame
// 1280x720x32 measured 1699 ms against 1813 ms at 2 blocks and 128).
#define ANA_TRAVERSAL_BOUNDS \
    __launch_bounds__(kPersistBlock, kPersist ? (kCurves ? 3 : (kMotion ? 4 : kPersistMinBlocks)) : 1)

__device__ __forceinline__ uint32_t scene_bits(float w) { return __float_as_uint(w); }

// extend: closest hit of every live path (PathIntegrator::Li, line 81).
// kCount: the same traversal, counting node fetches and primitive tests
// (warp-aggregated into p.work) to derive the stage's algorithmic bytes.
template <bool kCount, bool kCurves, bool kPersist, bool kMotion = false>
__global__ void ANA_TRAVERSAL_BOUNDS k_extend(const __grid_constant__ Params p) {
    const uint32_t cur = p.bounce & 1u;
    uint32_t* cb = p.counters + p.bounce * kCountersPerBounce;
    Counters cnt{0, 0, 0, 0};
    run_traversal<false, kCount, kPersist, kCurves, kMotion>(
        p.S, cb[0], cb + 3, p.err, &cnt,
        [&](uint32_t i, Ray& r, uint32_t& root, uint32_t& segRoot) {
            float4 o = p.q.ext_o[cur][i], d = p.q.ext_d[cur][i];
            r = Ray{f3(o), f3(d), 1e-4f, INFINITY};
            const DevSceneRec& R = p.S.scenes[scene_bits(p.q.ext_b[cur][i].w)];
            if constexpr (kMotion) r.time = path_time(R, __float_as_uint(o.w));
            root = R.tri_root;
            segRoot = kCurves ? R.seg_root : kNoRoot;
        },
        [&](uint32_t i, const Traversal& T) {
            SceneHit h = finish_closest<kCurves>(T, INFINITY);
            p.q.hit0[i] = make_float4(h.t, __uint_as_float(h.prim), h.u, h.v);
            if (kCurves && h.prim != kMiss && (h.prim & 0x80000000u)) p.q.hit1[i] = pack(h.tang, h.tseg);
        });
    if (kCount) warp_add_work(p.work, cnt);
}

// Surface interaction of a hit (BVHBackend::fillSurfaceInteraction,
// BVHBackend.cpp:285-317; CurveBrute intersectOneSegment, CurveBrute.cpp:209-233).
template <bool kCurves = true, bool kMotion = true>
__device__ __forceinline__ SurfInt surf_int(const DevScene& S, float3 o, float3 d, float t, uint32_t prim, float u,
                                            float v, float4 h1, float time = 0.f) {
    SurfInt si;
    if (!kCurves || !(prim & 0x80000000u)) {
        const float4* tp = S.tri_isect + 3 * size_t(prim);
        float4 a = ldg4(tp), e1 = ldg4(tp + 1), e2 = ldg4(tp + 2);
        const uint32_t ow = __float_as_uint(a.w), orig = ow & 0x01FFFFFFu;
        const float4* sp = S.tri_shade + 4 * size_t(orig);
        float4 s0 = ldg4(sp), s1 = ldg4(sp + 1), s2 = ldg4(sp + 2), s3 = ldg4(sp + 3);
        float w = 1.f - u - v;
        si.p = f3(a) + f3(e1) * u + f3(e2) * v;
        si.ng = f3(s0);
        float3 sn = safe_normalize(f3(s1) * w + f3(s2) * u + f3(s3) * v);
        si.dpdu = f3(e1);
        if (kMotion && (ow & 0x80000000u)) {
            // object-space triangle (fillSurfaceInteraction with worldXfm,
            // BVHBackend.cpp:290-300): objectToWorld at the ray's time
            M4 M;
            o2w_at(S, __float_as_uint(e1.w), time, M);
            si.p = m4_point(M, si.p);
            si.ng = xsafe_normalize(m4_normal(M, si.ng));
            sn = xsafe_normalize(m4_normal(M, sn));
            si.dpdu = m4_vector(M, si.dpdu);
        }
        if (dot(sn, si.ng) < 0.f) sn = -sn;
        si.n = sn;
        si.slot = __float_as_uint(s0.w);
        si.color = f3(1.f, 1.f, 1.f);
        si.is_curve = false;
    } else {
        uint32_t j = prim & 0x7FFFFFFFu;
        float4 rec = ldg4(S.segs + 5 * size_t(j) + 4);
        uint32_t strand = __float_as_uint(rec.x);
        float3 tang = f3(h1);
        si.p = o + d * t;
        float3 nd = -d;
        float3 nrm = nd - tang * dot(nd, tang);
        float3 fx, fy;
        onb(d, fx, fy);
        nrm = safe_normalize(nrm, fx);
        si.n = nrm;
        si.ng = nrm;
        si.dpdu = tang;
        si.slot = __float_as_uint(rec.z);
        si.color = f3(__ldg(S.strand_color + 3 * strand), __ldg(S.strand_color + 3 * strand + 1),
                      __ldg(S.strand_color + 3 * strand + 2));
        si.is_curve = true;
    }
    return si;
}

// SceneView::materials[meshID] of a scene (-1: no material).
__device__ __forceinline__ int slot_material(const DevScene& S, const DevSceneRec& R, uint32_t slot) {
    return slot < R.num_slots ? __ldg(S.slot_material + R.slot_base + slot) : -1;
}

// Mesh or strand slot (SurfaceInteraction::meshID) of a hit primitive.
__device__ __forceinline__ uint32_t hit_slot(const DevScene& S, uint32_t prim) {
    if (prim & 0x80000000u) return __float_as_uint(ldg4(S.segs + 5 * size_t(prim & 0x7FFFFFFFu) + 4).z);
    const uint32_t orig = __float_as_uint(ldg4(S.tri_isect + 3 * size_t(prim)).w) & 0x01FFFFFFu;
    return __float_as_uint(ldg4(S.tri_shade + 4 * size_t(orig)).w);
}

// Environment radiance seen along a direction that leaves the scene.
__device__ __forceinline__ float3 scene_env(const DevScene& S, const DevSceneRec& R, float3 d) {
    return R.has_dome ? env_eval(S.env, d) : R.env_radiance;
}

// Sums v over the lanes of the warp that share `key` and adds the sums to
// grad[key + j] with one atomic per distinct key (FP32 reduction before the
// atomics). Every lane of the warp must call it; kNoKey lanes add nothing.
template <int N>
__device__ __forceinline__ void warp_accum(float* grad, uint32_t key, const float (&v)[N]) {
    const uint32_t lane = threadIdx.x & 31u;
    bool ok = key != kNoKey;
#pragma unroll
    for (int j = 0; j < N; ++j) ok = ok && isfinite(v[j]);
    if (!ok) key = kNoKey;
    uint32_t pending = __ballot_sync(0xFFFFFFFFu, key != kNoKey);
    while (pending) {
        const int leader = __ffs(pending) - 1;
        const uint32_t k0 = __shfl_sync(0xFFFFFFFFu, key, leader);
        const bool mine = key == k0;
        pending &= ~__ballot_sync(0xFFFFFFFFu, mine);
#pragma unroll
        for (int j = 0; j < N; ++j) {
            float s = mine ? v[j] : 0.f;
            s += __shfl_xor_sync(0xFFFFFFFFu, s, 16);
            s += __shfl_xor_sync(0xFFFFFFFFu, s, 8);
            s += __shfl_xor_sync(0xFFFFFFFFu, s, 4);
            s += __shfl_xor_sync(0xFFFFFFFFu, s, 2);
            s += __shfl_xor_sync(0xFFFFFFFFu, s, 1);
            if (lane == uint32_t(leader) && s != 0.f) atomicAdd(grad + k0 + j, s);
        }
    }
}

__device__ __forceinline__ float3 load3(const float* a, size_t i) { return f3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
__device__ __forceinline__ float sum3(float3 v) { return v.x + v.y + v.z; }

// shade: one path vertex (PathIntegrator::Li, lines 81-176): emission,
// estimateDirect's light sample (shadow queue) and BSDF sample (MIS queue),
// and the continuation with Russian roulette (extend queue).
// kAdj (the adjoint replay) adds, with the sampling untouched:
//  - the pending continuation gradient of the previous vertex, now that its
//    remaining radiance L_rem = L - (radiance gathered so far) is known:
//    delta * (d log f / d theta) * L_rem;
//  - the emission gradient delta * beta of an emissive hit that counts;
//  - the NEE and MIS gradient payloads (resolved after their rays) and the
//    pending gradient of this vertex's continuation.
// kExtra: glass, alpha masks, motion blur and AOVs compiled in (batches
// without them take the smaller kernel).
// kFeat: the material and light classes compiled in (kFeat* bits); the host
// launches a kernel whose set covers the batch's (DevScene::features).
template <bool kAdj, bool kFiber, bool kExtra, uint32_t kFeat = kFeatAll>
__global__ void __launch_bounds__(kShadeBlock, (!kAdj && !kFiber) ? (kFeat == kFeatAll ? 3 : 4) : 2) k_shade(const __grid_constant__ Params p) {
    const uint32_t b = p.bounce;
    const uint32_t cur = b & 1u, nxt = cur ^ 1u;
    const uint32_t n = p.counters[b * kCountersPerBounce + 0];
    const DevScene& S = p.S;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t i = base + threadIdx.x;
        bool pushSh = false, pushMis = false, pushExt = false;
        float4 shO, shD, shC, mO, mD, mC, eO, eD, eB;
        // adjoint: payloads of the pushed entries and this vertex's direct sums
        float4 shG0, shG1, mG0, mG1, eG0, eG1;
        uint32_t keyPend = kNoKey, keyEmit = kNoKey;
        float vPend[4] = {0.f, 0.f, 0.f, 0.f}, vEmit[3] = {0.f, 0.f, 0.f};
        if (i < n) {
            float4 qo = p.q.ext_o[cur][i], qd = p.q.ext_d[cur][i], qb = p.q.ext_b[cur][i];
            float4 h0 = p.q.hit0[i];
            const uint32_t pid = __float_as_uint(qo.w), meta = __float_as_uint(qd.w);
            const uint32_t sc = scene_bits(qb.w);
            const DevSceneRec& R = S.scenes[sc];
            const uint32_t nL = R.num_lights;
            const uint32_t bounce = meta & 0xFFu;
            bool spec = (meta >> 8) & 1u;
            float3 o = f3(qo), d = f3(qd), beta = f3(qb);
            uint32_t prim = __float_as_uint(h0.y);
            float3 Ladd = f3(0.f, 0.f, 0.f);
            float3 delta = f3(0.f, 0.f, 0.f);
            bool adj = false;
            if constexpr (kAdj) {
                const size_t li = size_t(pid - p.chunk_first_path);
                delta = load3(p.a.dL, li);
                adj = !is_black(delta);
                const float4 g0 = p.a.ext_g0[cur][i];
                const uint32_t pm = __float_as_uint(g0.w);
                if (adj && pm != kNoKey) {
                    const float4 g1 = p.a.ext_g1[cur][i];
                    const float3 Lrem = load3(p.a.Lp, li) - load3(p.q.L, li);
                    const float3 wa = delta * Lrem * f3(g0), wr = delta * Lrem * f3(g1);
                    keyPend = 8u * pm;
                    vPend[0] = wa.x;
                    vPend[1] = wa.y;
                    vPend[2] = wa.z;
                    vPend[3] = sum3(wr);
                }
            }
            if (prim == kMiss) {
                if (bounce == 0 || spec) Ladd = beta * scene_env(S, R, d);
            } else {
                float4 h1 = (prim & 0x80000000u) ? p.q.hit1[i] : make_float4(0, 0, 0, 0);
                const float time = (kExtra && S.has_motion) ? path_time(R, pid) : 0.f;
                SurfInt si = surf_int<kFiber, kExtra>(S, o, d, h0.x, prim, h0.z, h0.w, h1, time);
                int mi = slot_material(S, R, si.slot);
                if (mi >= 0) {
                    const DevMaterial m = S.materials[mi];
                    uint32_t px, py, sidx;
                    path_coords(R, pid, px, py, sidx);
                    SampleStream ss{R.seed, px, py, sidx, meta >> 16};
                    // alpha test (PathIntegrator.cpp:103-118): a cut-out point
                    // continues the ray unshaded, one bounce later, drawing a
                    // sample dimension only for partial opacity
                    bool cut = false;
                    if (kExtra && m.opacity < 1.f) cut = m.opacity <= 0.f || ss.next() >= m.opacity;
                    if (cut) {
                        if (bounce + 1u <= R.max_depth) {
                            pushExt = true;
                            const uint32_t nm = (bounce + 1u) | (spec ? 0x100u : 0u) | (meta & 0x200u) | (ss.dim << 16);
                            eO = pack_u(spawn_origin(si.p, si.ng, d), pid);
                            eD = pack_u(d, nm);
                            eB = pack_u(beta, sc);
                            if constexpr (kAdj) {
                                eG0 = make_float4(0.f, 0.f, 0.f, __uint_as_float(kNoKey));
                                eG1 = make_float4(0.f, 0.f, 0.f, 0.f);
                            }
                        }
                    } else {
                        float3 wo = -d;
                        ShadeCtx c = make_ctx(si, d);
                        if (kExtra && p.aov && !(meta & 0x200u)) {
                            // first-hit AOVs (PathIntegrator.cpp:120-124): reflectance, si.n
                            float* A = p.q.aov + 6 * size_t(pid - p.chunk_first_path);
                            const float3 al = mat_reflectance(m, c);
                            A[0] = al.x;
                            A[1] = al.y;
                            A[2] = al.z;
                            A[3] = si.n.x;
                            A[4] = si.n.y;
                            A[5] = si.n.z;
                        }
                        float3 Le = mat_le(m);
                        if (!is_black(Le) && (bounce == 0 || spec)) Ladd = Ladd + beta * Le;
                        if constexpr (kAdj) {
                            if (adj && m.type == ANA_MAT_EMISSIVE && (bounce == 0 || spec)) {
                                const float3 ge = delta * beta;
                                keyEmit = 8u * uint32_t(mi) + 4u;
                                vEmit[0] = ge.x;
                                vEmit[1] = ge.y;
                                vEmit[2] = ge.z;
                            }
                        }
                        DevLight L;
                        bool misPending = false;
                        constexpr bool kShareSampler = (kFeat & kFeatStandard) != 0 || kFiber;
                        constexpr int kSampleUnroll = kShareSampler ? 1 : 2;
                        if (!m.is_delta && nL > 0) {
                            float ul = ss.next();
                            uint32_t lidx = min(uint32_t(ul * float(nL)), nL - 1u);
                            L = S.lights[R.light_base + lidx];
                            // light sampling
                            float lu0 = ss.next(), lu1 = ss.next();
                            LightSample ls = light_sample<kFeat>(S, L, si.p, lu0, lu1);
                            if (ls.pdf > 0.f && !is_black(ls.Li)) {
                                BsdfEval be = mat_eval<kFiber, kExtra, kFeat>(m, c, wo, ls.wi);
                                if (!is_black(be.f)) {
                                    float3 target = si.p + ls.wi * ls.dist;
                                    float3 dir = target - si.p;
                                    float dist = length(dir);
                                    dir = dir * (1.f / dist);
                                    float3 org = spawn_origin(si.p, si.n, dir);
                                    float w = ls.delta ? 1.f : power_heuristic(ls.pdf, be.pdf);
                                    float cosI;
                                    if (si.is_curve) {
                                        float dt = dot(ls.wi, c.t);
                                        cosI = sqrtf(fmaxf(0.f, 1.f - dt * dt));
                                    } else {
                                        cosI = absdot(ls.wi, si.n);
                                    }
                                    float3 contrib = beta * (be.f * ls.Li * cosI * w / ls.pdf) * float(nL);
                                    pushSh = true;
                                    shO = pack_u(org, pid);
                                    shD = pack(dir, dist * (1.f - 1e-4f));
                                    shC = pack_u(contrib, sc);
                                    if constexpr (kAdj) {
                                        // contrib = beta * f * Li * s, s = cosI w nL / pdf
                                        const float s = cosI * w / ls.pdf * float(nL);
                                        const BsdfGrad g = mat_grad<kFiber>(m, c, wo, ls.wi);
                                        const float3 db = delta * beta * s;
                                        const float3 ga = db * g.dfda * ls.Li;
                                        const bool area = adj && L.type == ANA_LIGHT_AREA;
                                        const float3 gl = area ? db * be.f : f3(0.f, 0.f, 0.f);
                                        const uint32_t lid = area ? R.light_base + lidx : 0xFFFFu;
                                        shG0 = make_float4(ga.x, ga.y, ga.z, sum3(db * g.dfdr * ls.Li));
                                        shG1 = pack_u(gl, (adj ? uint32_t(mi) : 0xFFFFu) | (lid << 16));
                                    }
                                }
                            }
                            // BSDF sampling toward the light: non-delta lights only,
                            // and only then are its sample dimensions drawn
                            // (estimateDirect, PathIntegrator.cpp:210); the sample is
                            // taken in the loop below
                            misPending = !((kFeat & kFeatDir) != 0 && L.type == ANA_LIGHT_DIRECTIONAL);
                        }
                        // BSDF samples: the one toward the light for MIS (k = 0, when
                        // drawn), then the continuation (k = 1), each drawing (uc, u0,
                        // u1) in that order. Kernels with standard_surface or hair code
                        // run both through one copy of the sampling code in a loop
                        // instead of two inlined ones: the throughput frame's shade
                        // stage 76.2 -> 68.9 ms (smaller code, fewer instruction-fetch
                        // stalls; outlining mat_sample as a call measured 89.6 ms).
                        // Lambert's sampling is small, and there the loop cost more
                        // than it saved (64 Cornell variants 72.2 -> 78.2 ms), so that
                        // kernel unrolls the loop into two copies.
#pragma unroll (kSampleUnroll)
                        for (int k = kShareSampler ? (misPending ? 0 : 1) : 0; k < 2; ++k) {
                            if (!kShareSampler && k == 0 && !misPending) continue;
                            const float uc = ss.next();
                            const float u0 = ss.next(), u1 = ss.next();
                            BsdfSample bs = mat_sample<kFiber, kExtra, kFeat>(m, c, wo, u0, u1, uc);
                            if (!bs.valid()) continue;
                            if (k == 0) {
                                float lp = light_pdf<kFeat>(S, L, si.p, bs.wi);
                                if (lp > 0.f) {
                                    float w = bs.delta() ? 1.f : power_heuristic(bs.pdf, lp);
                                    float3 org = spawn_origin(si.p, si.ng, bs.wi);
                                    float cosI = absdot(bs.wi, si.n);
                                    float3 contrib = beta * (bs.f * cosI * w / bs.pdf) * float(nL);
                                    pushMis = true;
                                    mO = pack_u(org, pid);
                                    mD = pack(bs.wi, 0.f);
                                    mC = pack_u(contrib, sc);
                                    if constexpr (kAdj) {
                                        // bs.f = f |cos wi|: K = beta * f * |cos wi| * cosI w nL / pdf
                                        const BsdfGrad g = mat_grad<kFiber>(m, c, wo, bs.wi);
                                        const float s = fabsf(c.to_local(bs.wi).z) * cosI * w / bs.pdf * float(nL);
                                        const float3 db = delta * beta * s;
                                        mG0 = pack_u(db * g.dfda, adj ? uint32_t(mi) : kNoKey);
                                        mG1 = pack(db * g.dfdr, 0.f);
                                    }
                                }
                                continue;
                            }
                            spec = bs.delta();
                            beta = beta * (bs.f / bs.pdf);
                            float3 org = spawn_origin(si.p, si.n, bs.wi);
                            bool alive = true;
                            if (bounce >= R.min_depth) {
                                float q = 1.f - fminf(max_comp(beta), 0.95f);
                                if (ss.next() < q) alive = false;
                                else beta = beta * (1.f / (1.f - q));
                            }
                            if (alive && bounce + 1u <= R.max_depth) {
                                pushExt = true;
                                uint32_t nm = (bounce + 1u) | (spec ? 0x100u : 0u) | 0x200u | (ss.dim << 16);
                                eO = pack_u(org, pid);
                                eD = pack_u(bs.wi, nm);
                                eB = pack_u(beta, sc);
                                if constexpr (kAdj) {
                                    // beta' = beta * f |cos| / pdf (pdf and roulette detached):
                                    // d log beta' / d theta = (d f / d theta) / f per channel
                                    const BsdfGrad g = mat_grad<kFiber>(m, c, wo, bs.wi);
                                    auto ratio = [](float num, float den) { return den > 0.f ? num / den : 0.f; };
                                    const float3 la = f3(ratio(g.dfda.x, g.f.x), ratio(g.dfda.y, g.f.y),
                                                         ratio(g.dfda.z, g.f.z));
                                    const float3 lr = f3(ratio(g.dfdr.x, g.f.x), ratio(g.dfdr.y, g.f.y),
                                                         ratio(g.dfdr.z, g.f.z));
                                    const bool any = adj && (!is_black(la) || !is_black(lr));
                                    eG0 = pack_u(la, any ? uint32_t(mi) : kNoKey);
                                    eG1 = pack(lr, 0.f);
                                }
                            }
                        }
                    }
                }
            }
            if (!is_black(Ladd)) add_L(p, pid, Ladd);
        }
        if constexpr (kAdj) {
            warp_accum(p.a.grad, keyPend, vPend);
            warp_accum(p.a.grad, keyEmit, vEmit);
        }
        uint32_t* cb = p.counters + b * kCountersPerBounce;
        uint32_t k, kMis, kExt;
        block_push3(pushSh, pushMis, pushExt, cb + 1, cb + 2, cb + kCountersPerBounce + 0, k, kMis, kExt);
        if (pushSh) {
            p.q.sh_o[k] = shO;
            p.q.sh_d[k] = shD;
            p.q.sh_c[k] = shC;
            if constexpr (kAdj) {
                p.a.sh_g0[k] = shG0;
                p.a.sh_g1[k] = shG1;
            }
        }
        k = kMis;
        if (pushMis) {
            p.q.mis_o[k] = mO;
            p.q.mis_d[k] = mD;
            p.q.mis_c[k] = mC;
            if constexpr (kAdj) {
                p.a.mis_g0[k] = mG0;
                p.a.mis_g1[k] = mG1;
            }
        }
        k = kExt;
        if (pushExt) {
            p.q.ext_o[nxt][k] = eO;
            p.q.ext_d[nxt][k] = eD;
            p.q.ext_b[nxt][k] = eB;
            if constexpr (kAdj) {
                p.a.ext_g0[nxt][k] = eG0;
                p.a.ext_g1[nxt][k] = eG1;
            }
        }
    }
}

// NEE shadow rays: shadowTransmittance (src/integrator/ShadowRay.h:26-61) for
// opaque scenes — any blocker in [1e-4, tmax] makes the transmittance black.
// Triangle-only batches test each leaf as they reach it (1920x1080x64
// throughput frame: shadow stage 53.1 ms parking leaves, 46.3 ms without; the
// motion frame 45.8 -> 42.1 ms); with curves the lanes park leaves (the hair
// frame's shadow stage 373.0 against 374.3 ms).
template <bool kCurves, bool kPersist, bool kAdj, bool kMotion = false>
__global__ void ANA_TRAVERSAL_BOUNDS k_shadow(const __grid_constant__ Params p) {
    uint32_t* cb = p.counters + p.bounce * kCountersPerBounce;
    run_traversal<true, false, kPersist, kCurves, kMotion, kCurves>(
        p.S, cb[1], cb + 4, p.err, nullptr,
        [&](uint32_t i, Ray& r, uint32_t& root, uint32_t& segRoot) {
            float4 o = p.q.sh_o[i], d = p.q.sh_d[i];
            r = Ray{f3(o), f3(d), 1e-4f, d.w};
            const DevSceneRec& R = p.S.scenes[scene_bits(p.q.sh_c[i].w)];
            if constexpr (kMotion) r.time = path_time(R, __float_as_uint(o.w));
            root = R.tri_root;
            segRoot = kCurves ? R.seg_root : kNoRoot;
        },
        [&](uint32_t i, const Traversal& T) {
            float4 o = p.q.sh_o[i], c = p.q.sh_c[i];
            const bool occluded = finish_any<kCurves>(T);
            if (!occluded) add_L(p, __float_as_uint(o.w), f3(c));
            if constexpr (kAdj) p.a.sh_vis[i] = occluded ? 0u : 1u;
        });
}

// BSDF-sampled MIS rays (PathIntegrator.cpp:214-259): the first surface hit
// within 1e10 contributes its material's Le, a miss the environment. In a
// batch without emissive surfaces every hit contributes zero, so the ray only
// needs to know whether anything is hit (kAny): identical result, cheaper
// query. MIS rays do not park leaves (kPark false): with grouped refills the
// speculative any-hit schedule cost them time (1920x1080x64 throughput frame:
// MIS stage 73.7 ms parking leaves, 61.1 ms without).
template <bool kAny, bool kCurves, bool kPersist, bool kAdj, bool kMotion = false>
__global__ void ANA_TRAVERSAL_BOUNDS k_mis(const __grid_constant__ Params p) {
    uint32_t* cb = p.counters + p.bounce * kCountersPerBounce;
    const DevScene& S = p.S;
    run_traversal<kAny, false, kPersist, kCurves, kMotion, false>(
        S, cb[2], cb + 5, p.err, nullptr,
        [&](uint32_t i, Ray& r, uint32_t& root, uint32_t& segRoot) {
            float4 o = p.q.mis_o[i], d = p.q.mis_d[i];
            r = Ray{f3(o), f3(d), 1e-4f, 1e10f};
            const DevSceneRec& R = S.scenes[scene_bits(p.q.mis_c[i].w)];
            if constexpr (kMotion) r.time = path_time(R, __float_as_uint(o.w));
            root = R.tri_root;
            segRoot = kCurves ? R.seg_root : kNoRoot;
        },
        [&](uint32_t i, const Traversal& T) {
            float4 o = p.q.mis_o[i], d = p.q.mis_d[i], c = p.q.mis_c[i];
            const float3 rd = f3(d);
            const DevSceneRec& R = S.scenes[scene_bits(c.w)];
            float3 Li;
            int mi = -1;
            if (kAny) {
                Li = finish_any<kCurves>(T) ? f3(0.f, 0.f, 0.f) : scene_env(S, R, rd);
            } else {
                SceneHit h = finish_closest<kCurves>(T, 1e10f);
                if (h.prim == kMiss) {
                    Li = scene_env(S, R, rd);
                } else {
                    mi = slot_material(S, R, hit_slot(S, h.prim));
                    Li = mi >= 0 ? mat_le(S.materials[mi]) : f3(0.f, 0.f, 0.f);
                }
            }
            if (!is_black(Li)) add_L(p, __float_as_uint(o.w), f3(c) * Li);
            if constexpr (kAdj) p.a.mis_res[i] = pack_u(Li, mi >= 0 ? uint32_t(mi) : kNoKey);
        });
}

// Rays that step through transmissive surfaces (batches whose materials
// include glass or alpha masks). Each lane keeps its entry's step state: the
// product of the tints passed, the current origin and tMax, and the surfaces
// passed. A transmissive closest hit multiplies the tint in and, unless less
// than 1e-4 of the distance remains or 8 surfaces have been traced, the ray
// is traced again from spawnRay(p, ng, d) with tMax = remaining - 1e-4.
struct StepState {
    float3 tr, org;
    float tmax, time;
    uint32_t steps;
    bool fresh;
    __device__ void begin(float3 o, float tm, float t) {
        if (!fresh) return;
        tr = f3(1.f, 1.f, 1.f);
        org = o;
        tmax = tm;
        time = t;
        steps = 0;
        fresh = false;
    }
    // After a transmissive hit with tr still non-black: true (and `next`) if
    // the ray continues past the surface.
    template <bool kCurves>
    __device__ bool advance(const DevScene& S, const SceneHit& h, float3 d, bool& tooClose, Ray& next) {
        const float remaining = tmax - h.t;
        tooClose = remaining <= 1e-4f;
        if (tooClose || steps >= 7u) return false;
        const float4 h1 = make_float4(h.tang.x, h.tang.y, h.tang.z, h.tseg);
        const SurfInt si = surf_int<kCurves>(S, org, d, h.t, h.prim, h.u, h.v, h1, time);
        next = Ray{spawn_origin(si.p, si.ng, d), d, 1e-4f, remaining - 1e-4f, time};
        org = next.o;
        tmax = next.tmax;
        ++steps;
        return true;
    }
};

// NEE shadow rays with transmissive surfaces: shadowTransmittance
// (src/integrator/ShadowRay.h:26-61) — an opaque surface (black
// transmittanceColor) blocks, glass and alpha-masked surfaces tint; after 8
// surfaces the tint so far is returned.
template <bool kCurves, bool kPersist, bool kMotion = false>
__global__ void ANA_TRAVERSAL_BOUNDS k_shadow_step(const __grid_constant__ Params p) {
    uint32_t* cb = p.counters + p.bounce * kCountersPerBounce;
    const DevScene& S = p.S;
    StepState st;
    st.fresh = true;
    run_traversal<false, false, kPersist, kCurves, kMotion>(
        S, cb[1], cb + 4, p.err, nullptr,
        [&](uint32_t i, Ray& r, uint32_t& root, uint32_t& segRoot) {
            float4 o = p.q.sh_o[i], d = p.q.sh_d[i];
            const DevSceneRec& R = S.scenes[scene_bits(p.q.sh_c[i].w)];
            r = Ray{f3(o), f3(d), 1e-4f, d.w, kMotion ? path_time(R, __float_as_uint(o.w)) : 0.f};
            st.begin(r.o, r.tmax, r.time);
            root = R.tri_root;
            segRoot = kCurves ? R.seg_root : kNoRoot;
        },
        [&](uint32_t i, const Traversal& T, Ray& next) -> bool {
            const float4 c = p.q.sh_c[i];
            const SceneHit h = finish_closest<kCurves>(T, st.tmax);
            bool lit = true;
            if (h.prim != kMiss) {
                const DevSceneRec& R = S.scenes[scene_bits(c.w)];
                const int mi = slot_material(S, R, hit_slot(S, h.prim));
                const float3 tint = mi >= 0 ? S.materials[mi].tint : f3(0.f, 0.f, 0.f);
                st.tr = st.tr * tint;
                lit = !is_black(tint) && !is_black(st.tr);
                bool tooClose;
                if (lit && st.advance<kCurves>(S, h, f3(p.q.sh_d[i]), tooClose, next)) return true;
            }
            if (lit) add_L(p, __float_as_uint(p.q.sh_o[i].w), f3(c) * st.tr);
            st.fresh = true;
            return false;
        });
}

// BSDF-sampled MIS rays with transmissive surfaces (PathIntegrator.cpp:
// 214-259): the first non-transmissive surface within 1e10 (or the 8th
// transmissive one) gives Le, a miss or a last step closer than 1e-4 the
// environment, times the tint of the surfaces passed.
template <bool kCurves, bool kPersist, bool kMotion = false>
__global__ void ANA_TRAVERSAL_BOUNDS k_mis_step(const __grid_constant__ Params p) {
    uint32_t* cb = p.counters + p.bounce * kCountersPerBounce;
    const DevScene& S = p.S;
    StepState st;
    st.fresh = true;
    run_traversal<false, false, kPersist, kCurves, kMotion>(
        S, cb[2], cb + 5, p.err, nullptr,
        [&](uint32_t i, Ray& r, uint32_t& root, uint32_t& segRoot) {
            float4 o = p.q.mis_o[i], d = p.q.mis_d[i];
            const DevSceneRec& R = S.scenes[scene_bits(p.q.mis_c[i].w)];
            r = Ray{f3(o), f3(d), 1e-4f, 1e10f, kMotion ? path_time(R, __float_as_uint(o.w)) : 0.f};
            st.begin(r.o, r.tmax, r.time);
            root = R.tri_root;
            segRoot = kCurves ? R.seg_root : kNoRoot;
        },
        [&](uint32_t i, const Traversal& T, Ray& next) -> bool {
            const float4 c = p.q.mis_c[i];
            const float3 rd = f3(p.q.mis_d[i]);
            const DevSceneRec& R = S.scenes[scene_bits(c.w)];
            const SceneHit h = finish_closest<kCurves>(T, st.tmax);
            float3 Li = f3(0.f, 0.f, 0.f);
            if (h.prim == kMiss) {
                Li = scene_env(S, R, rd);
            } else {
                const int mi = slot_material(S, R, hit_slot(S, h.prim));
                if (mi < 0) {
                    st.tr = f3(0.f, 0.f, 0.f);
                } else {
                    const DevMaterial& m = S.materials[mi];
                    const float3 tint = m.tint;
                    bool tooClose = false;
                    if (!is_black(tint)) {
                        st.tr = st.tr * tint;
                        if (!is_black(st.tr) && st.advance<kCurves>(S, h, rd, tooClose, next)) return true;
                    }
                    Li = tooClose ? scene_env(S, R, rd) : mat_le(m);
                }
            }
            if (!is_black(Li) && !is_black(st.tr)) add_L(p, __float_as_uint(p.q.mis_o[i].w), f3(c) * (Li * st.tr));
            st.fresh = true;
            return false;
        });
}

// Adjoint replay set-up, after generate: dLoss/dL of every path of the chunk
// (the film keeps finite samples only, each with weight 1/spp of its pixel),
// and no pending continuation gradient on the camera vertices.
__global__ void __launch_bounds__(256) k_adj_init(const __grid_constant__ Params p) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < p.chunk_paths; i += gridDim.x * blockDim.x) {
        const uint32_t gid = p.chunk_first_path + i;
        const DevSceneRec& R = p.S.scenes[scene_of(p.S, gid)];
        const uint32_t pixel = div_magic(gid - R.path_offset, R.spp_div);
        const float3 L = load3(p.a.Lp, i);
        float3 dl = f3(0.f, 0.f, 0.f);
        if (is_finite3(L)) dl = load3(p.a.d_image, film_index(R, pixel)) * (1.f / float(R.spp));
        p.a.dL[3 * size_t(i)] = dl.x;
        p.a.dL[3 * size_t(i) + 1] = dl.y;
        p.a.dL[3 * size_t(i) + 2] = dl.z;
        p.a.ext_g0[0][i] = make_float4(0.f, 0.f, 0.f, __uint_as_float(kNoKey));
    }
}

// Resolves the gradient payloads of one bounce once the shadow and MIS rays
// are traced. NEE (unoccluded only): material albedo / roughness terms and
// the area light's Le term. MIS: the material terms times the Li found, and
// delta * K for the emissive material hit.
__global__ void __launch_bounds__(256) k_adj_direct(const __grid_constant__ Params p) {
    const uint32_t* cb = p.counters + p.bounce * kCountersPerBounce;
    const uint32_t nsh = cb[1], nmis = cb[2], n = max(nsh, nmis);
    const uint32_t lightBase = 8u * p.a.num_materials;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t i = base + threadIdx.x;
        uint32_t kMat = kNoKey, kLe = kNoKey;
        float vMat[4] = {0.f, 0.f, 0.f, 0.f}, vLe[3] = {0.f, 0.f, 0.f};
        if (i < nsh && p.a.sh_vis[i]) {
            const float4 g0 = p.a.sh_g0[i], g1 = p.a.sh_g1[i];
            const uint32_t ids = __float_as_uint(g1.w), m = ids & 0xFFFFu, l = ids >> 16;
            if (m != 0xFFFFu) {
                kMat = 8u * m;
                vMat[0] = g0.x;
                vMat[1] = g0.y;
                vMat[2] = g0.z;
                vMat[3] = g0.w;
            }
            if (l != 0xFFFFu) {
                kLe = lightBase + 4u * l;
                vLe[0] = g1.x;
                vLe[1] = g1.y;
                vLe[2] = g1.z;
            }
        }
        warp_accum(p.a.grad, kMat, vMat);
        warp_accum(p.a.grad, kLe, vLe);
        kMat = kNoKey;
        kLe = kNoKey;
        if (i < nmis) {
            const float4 res = p.a.mis_res[i], g0 = p.a.mis_g0[i];
            const float3 Li = f3(res);
            const uint32_t m = __float_as_uint(g0.w), hit = __float_as_uint(res.w);
            if (m != kNoKey && !is_black(Li)) {
                const float4 g1 = p.a.mis_g1[i];
                kMat = 8u * m;
                vMat[0] = g0.x * Li.x;
                vMat[1] = g0.y * Li.y;
                vMat[2] = g0.z * Li.z;
                vMat[3] = sum3(f3(g1) * Li);
            }
            if (m != kNoKey && hit != kNoKey && p.S.materials[hit].type == ANA_MAT_EMISSIVE) {
                const uint32_t pid = __float_as_uint(p.q.mis_o[i].w);
                const float3 delta = load3(p.a.dL, size_t(pid - p.chunk_first_path));
                const float3 ge = delta * f3(p.q.mis_c[i]);
                kLe = 8u * hit + 4u;
                vLe[0] = ge.x;
                vLe[1] = ge.y;
                vLe[2] = ge.z;
            }
        }
        warp_accum(p.a.grad, kMat, vMat);
        warp_accum(p.a.grad, kLe, vLe);
    }
}

// Film accumulation (PathIntegrator.cpp:43-57 + Film::mergeTile, Film.cpp:34-56):
// finite samples summed in sample order, weight = sample count.
__global__ void __launch_bounds__(256) k_film(const __grid_constant__ Params p) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < p.chunk_pixels; q += gridDim.x * blockDim.x) {
        // the chunk's pixel run holding local pixel q
        uint32_t lo = 0, hi = p.num_segs;
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (p.segs[mid].local_pixel <= q) lo = mid;
            else hi = mid;
        }
        const ChunkSeg sg = p.segs[lo];
        const DevSceneRec& R = p.S.scenes[sg.scene];
        const uint32_t spp = R.spp;
        const uint32_t k = q - sg.local_pixel;
        float3 acc = f3(0.f, 0.f, 0.f);
        float lsq = 0.f;
        const float* Lp = p.q.L + (size_t(sg.local_path) + size_t(k) * spp) * 3;
        for (uint32_t s = 0; s < spp; ++s) {
            float3 L = f3(Lp[3 * s], Lp[3 * s + 1], Lp[3 * s + 2]);
            if (is_finite3(L)) {
                acc = acc + L;
                float lum = luminance(L);
                lsq += lum * lum;
            }
        }
        const float invSPP = 1.f / float(spp);
        const size_t fi = film_index(R, sg.first_pixel + k);
        ana_film_pixel& f = p.film[fi];
        float w = float(spp);
        f.r += (acc.x * invSPP) * w;
        f.g += (acc.y * invSPP) * w;
        f.b += (acc.z * invSPP) * w;
        f.w += w;
        f.sum_lum_sq += lsq;
        if (p.aov) {
            // renderTile's AOV averages over every sample of the pass
            // (PathIntegrator.cpp:44-66), merged with weight 1 as
            // Film::mergeTile does (Film.cpp:58-70)
            const float* A = p.q.aov + (size_t(sg.local_path) + size_t(k) * spp) * 6;
            float3 sa = f3(0.f, 0.f, 0.f), sn = f3(0.f, 0.f, 0.f);
            for (uint32_t s = 0; s < spp; ++s) {
                sa = xadd3(sa, f3(A[6 * s], A[6 * s + 1], A[6 * s + 2]));
                sn = xadd3(sn, f3(A[6 * s + 3], A[6 * s + 4], A[6 * s + 5]));
            }
            const float3 al = xmul3(sa, invSPP);
            float3 n = xmul3(sn, invSPP);
            const float len = __fsqrt_rn(xdot(n, n));
            if (len > 1e-6f) n = xmul3(n, xdiv(1.f, len));
            float* F = p.aov + 8 * fi;
            F[0] += al.x;
            F[1] += al.y;
            F[2] += al.z;
            F[3] += 1.f;
            F[4] += n.x;
            F[5] += n.y;
            F[6] += n.z;
            F[7] += 1.f;
        }
    }
}

// IAccelerationStructure::traceBatch / occludedBatch over CurveBrute semantics,
// against one scene of the batch.
template <bool kAny, bool kCurves, bool kPersist, bool kMotion = false>
__global__ void ANA_TRAVERSAL_BOUNDS k_trace_batch(const __grid_constant__ DevScene S, uint32_t scene,
                                                   const float* rays, const float* times, uint32_t n, ana_hit* out,
                                                   uint32_t* fetch, uint32_t* err) {
    const uint32_t triRoot = S.scenes[scene].tri_root, segRoot = S.scenes[scene].seg_root;
    auto load = [&](uint32_t i, Ray& r, uint32_t& root, uint32_t& sroot) {
        const float4* rp = reinterpret_cast<const float4*>(rays + 8 * size_t(i));
        float4 a = rp[0], b = rp[1];
        r = Ray{f3(a), f3(b), a.w, b.w, times ? times[i] : 0.f};
        root = triRoot;
        sroot = kCurves ? segRoot : kNoRoot;
    };
    // without `times` every ray has Ray::time's default 0 (Types.h:259)
    run_traversal<kAny, false, kPersist, kCurves, kMotion>(S, n, fetch, err, nullptr, load, [&](uint32_t i, const Traversal& T) {
        ana_hit h{0, -1, -1, -1, 0.f, 0.f, 0.f, 0.f};
        if (kAny) {
            h.hit = finish_any<kCurves>(T) ? 1 : 0;
        } else {
            const float tmax = reinterpret_cast<const float4*>(rays + 8 * size_t(i))[1].w;
            SceneHit sh = finish_closest<kCurves>(T, tmax);
            if (sh.prim != kMiss) {
                h.hit = 1;
                h.t = sh.t;
                h.u = sh.u;
                h.v = sh.v;
                if (sh.prim & 0x80000000u) {
                    float4 rec = ldg4(S.segs + 5 * size_t(sh.prim & 0x7FFFFFFFu) + 4);
                    h.mesh_id = int32_t(__float_as_uint(rec.z));
                    h.prim_id = int32_t(__float_as_uint(rec.y));
                    h.strand_id = int32_t(__float_as_uint(rec.x) - __float_as_uint(rec.w));
                } else {
                    uint32_t orig = __float_as_uint(ldg4(S.tri_isect + 3 * size_t(sh.prim)).w) & 0x01FFFFFFu;
                    const float4* sp = S.tri_shade + 4 * size_t(orig);
                    h.mesh_id = int32_t(__float_as_uint(ldg4(sp).w));
                    h.prim_id = int32_t(__float_as_uint(ldg4(sp + 1).w));
                }
            }
        }
        out[i] = h;
    });
}

// ---------------------------------------------------------------------------
static inline int blocks_for(uint32_t n, int block, int cap) {
    long long b = ((long long)n + block - 1) / block;
    if (b < 1) b = 1;
    return int(b < cap ? b : cap);
}

// Resident blocks per kernel on each device (one wave of the persistent
// schedule), filled by prime_kernels() before any launch so that no
// occupancy query or lazy module load happens while a stream is captured.
static std::mutex g_grid_mu;
static std::map<std::pair<int, const void*>, int> g_grid;

template <class K>
static int resident_grid(K kernel) {
    int dev = 0;
    cudaGetDevice(&dev);
    const void* key = reinterpret_cast<const void*>(kernel);
    {
        std::lock_guard<std::mutex> lk(g_grid_mu);
        auto it = g_grid.find({dev, key});
        if (it != g_grid.end()) return it->second;
    }
    int sms = 148, per = 1;
    cudaFuncAttributes attr;
    cudaFuncGetAttributes(&attr, kernel);  // loads the function
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kPersistBlock, 0);
    int g = sms * (per > 0 ? per : 1);
    std::lock_guard<std::mutex> lk(g_grid_mu);
    g_grid[{dev, key}] = g;
    return g;
}

// Grid for a traversal kernel: one resident wave when persistent, otherwise
// enough blocks to cover the chunk capacity (grid-stride beyond it).
template <bool kPersist, class K>
static int traversal_grid(K kernel, const LaunchCfg& c) {
    if (kPersist) return resident_grid(kernel);
    return c.grid_cap;
}

template <class K>
static void prime(K kernel) {
    resident_grid(kernel);
}

void prime_kernels() {
    prime(k_generate);
    prime(k_shade<false, false, false>);
    prime(k_shade<false, false, true>);
    prime(k_shade<false, true, false>);
    prime(k_shade<false, true, true>);
    prime(k_shade<false, false, false, kFeatStandard | kFeatDome>);
    prime(k_shade<false, false, false, kFeatLambert | kFeatArea>);
    prime(k_shade<false, true, false, kFeatLambert | kFeatArea>);
    prime(k_shade<true, false, false>);
    prime(k_shade<true, true, false>);
    prime(k_film);
    prime(k_adj_init);
    prime(k_adj_direct);
    prime(k_extend<false, false, false>);
    prime(k_extend<false, false, true>);
    prime(k_extend<false, true, false>);
    prime(k_extend<false, true, true>);
    prime(k_extend<true, false, false>);
    prime(k_extend<true, false, true>);
    prime(k_extend<true, true, false>);
    prime(k_extend<true, true, true>);
    prime(k_shadow<false, false, false>);
    prime(k_shadow<false, true, false>);
    prime(k_shadow<true, false, false>);
    prime(k_shadow<true, true, false>);
    prime(k_shadow<false, false, true>);
    prime(k_shadow<false, true, true>);
    prime(k_shadow<true, false, true>);
    prime(k_shadow<true, true, true>);
    prime(k_mis<false, false, false, false>);
    prime(k_mis<false, false, true, false>);
    prime(k_mis<false, true, false, false>);
    prime(k_mis<false, true, true, false>);
    prime(k_mis<true, false, false, false>);
    prime(k_mis<true, false, true, false>);
    prime(k_mis<true, true, false, false>);
    prime(k_mis<true, true, true, false>);
    prime(k_mis<false, false, false, true>);
    prime(k_mis<false, false, true, true>);
    prime(k_mis<false, true, false, true>);
    prime(k_mis<false, true, true, true>);
    prime(k_shadow_step<false, false>);
    prime(k_shadow_step<false, true>);
    prime(k_shadow_step<true, false>);
    prime(k_shadow_step<true, true>);
    prime(k_mis_step<false, false>);
    prime(k_mis_step<false, true>);
    prime(k_mis_step<true, false>);
    prime(k_mis_step<true, true>);
    prime(k_extend<false, false, true, true>);
    prime(k_extend<false, true, true, true>);
    prime(k_shadow<false, true, false, true>);
    prime(k_shadow<true, true, false, true>);
    prime(k_mis<false, false, true, false, true>);
    prime(k_mis<false, true, true, false, true>);
    prime(k_mis<true, false, true, false, true>);
    prime(k_mis<true, true, true, false, true>);
    prime(k_shadow_step<false, true, true>);
    prime(k_shadow_step<true, true, true>);
    prime(k_mis_step<false, true, true>);
    prime(k_mis_step<true, true, true>);
    prime(k_trace_batch<false, false, true, true>);
    prime(k_trace_batch<false, true, true, true>);
    prime(k_trace_batch<true, false, true, true>);
    prime(k_trace_batch<true, true, true, true>);
    prime(k_trace_batch<false, false, false>);
    prime(k_trace_batch<false, false, true>);
    prime(k_trace_batch<false, true, false>);
    prime(k_trace_batch<false, true, true>);
    prime(k_trace_batch<true, false, false>);
    prime(k_trace_batch<true, false, true>);
    prime(k_trace_batch<true, true, false>);
    prime(k_trace_batch<true, true, true>);
}

void launch_generate(const Params& p, const LaunchCfg& c, cudaStream_t s) {
    k_generate<<<blocks_for(p.chunk_paths, 256, c.grid_cap), 256, 0, s>>>(p);
}

// Batches with motion-blurred meshes take the persistent schedule (their
// kernels are instantiated for it only) without work counting.
template <bool kCount, bool kCurves, bool kPersist, bool kMotion = false>
static void ext_launch(const Params& p, const LaunchCfg& c, cudaStream_t s) {
    auto k = k_extend<kCount, kCurves, kPersist, kMotion>;
    k<<<traversal_grid<kPersist>(k, c), kPersistBlock, 0, s>>>(p);
}
void launch_extend(const Params& p, const LaunchCfg& c, cudaStream_t s, bool count_work) {
    const bool cv = p.S.has_curves != 0, ps = c.persistent != 0;
    if (p.S.has_motion) {
        cv ? ext_launch<false, true, true, true>(p, c, s) : ext_launch<false, false, true, true>(p, c, s);
    } else if (count_work) {
        if (cv) ps ? ext_launch<true, true, true>(p, c, s) : ext_launch<true, true, false>(p, c, s);
        else ps ? ext_launch<true, false, true>(p, c, s) : ext_launch<true, false, false>(p, c, s);
    } else {
        if (cv) ps ? ext_launch<false, true, true>(p, c, s) : ext_launch<false, true, false>(p, c, s);
        else ps ? ext_launch<false, false, true>(p, c, s) : ext_launch<false, false, false>(p, c, s);
    }
}
void launch_shade(const Params& p, const LaunchCfg& c0, cudaStream_t s) {
    LaunchCfg c = c0;
    c.block = std::min(c.block, kShadeBlock);
    const int g = std::min(c.grid_cap, c.stage_grid);
    const bool extra = p.S.has_extra_shading || p.aov;
    // kernels without the material / light classes a batch lacks: GGX
    // surfaces under a dome (the throughput scene), Lambert surfaces under
    // area lights (the Cornell boxes and the hair scene)
    constexpr uint32_t kStdDome = kFeatStandard | kFeatDome, kLambArea = kFeatLambert | kFeatArea;
    const uint32_t f = p.S.features;
    if (p.S.has_fibers) {
        if (extra) k_shade<false, true, true><<<g, c.block, 0, s>>>(p);
        else if ((f & ~kLambArea) == 0) k_shade<false, true, false, kLambArea><<<g, c.block, 0, s>>>(p);
        else k_shade<false, true, false><<<g, c.block, 0, s>>>(p);
    } else {
        if (extra) k_shade<false, false, true><<<g, c.block, 0, s>>>(p);
        else if ((f & ~kStdDome) == 0) k_shade<false, false, false, kStdDome><<<g, c.block, 0, s>>>(p);
        else if ((f & ~kLambArea) == 0) k_shade<false, false, false, kLambArea><<<g, c.block, 0, s>>>(p);
        else k_shade<false, false, false><<<g, c.block, 0, s>>>(p);
    }
}
template <bool kCurves, bool kPersist, bool kAdj, bool kMotion = false>
static void sh_launch(const Params& p, const LaunchCfg& c, cudaStream_t s) {
    auto k = k_shadow<kCurves, kPersist, kAdj, kMotion>;
    k<<<traversal_grid<kPersist>(k, c), kPersistBlock, 0, s>>>(p);
}
template <bool kAdj>
static void shadow_dispatch(const Params& p, const LaunchCfg& c, cudaStream_t s) {
    const bool cv = p.S.has_curves != 0, ps = c.persistent != 0;
    if (!kAdj && p.S.has_motion)
        cv ? sh_launch<true, true, false, true>(p, c, s) : sh_launch<false, true, false, true>(p, c, s);
    else if (cv) ps ? sh_launch<true, true, kAdj>(p, c, s) : sh_launch<true, false, kAdj>(p, c, s);
    else ps ? sh_launch<false, true, kAdj>(p, c, s) : sh_launch<false, false, kAdj>(p, c, s);
}
template <bool kCurves, bool kPersist, bool kMotion = false>
static void step_launch(const Params& p, const LaunchCfg& c, cudaStream_t s, bool mis) {
    auto k = mis ? k_mis_step<kCurves, kPersist, kMotion> : k_shadow_step<kCurves, kPersist, kMotion>;
    k<<<traversal_grid<kPersist>(k, c), kPersistBlock, 0, s>>>(p);
}
static void step_dispatch(const Params& p, const LaunchCfg& c, cudaStream_t s, bool mis) {
    const bool cv = p.S.has_curves != 0, ps = c.persistent != 0;
    if (p.S.has_motion)
        cv ? step_launch<true, true, true>(p, c, s, mis) : step_launch<false, true, true>(p, c, s, mis);
    else if (cv) ps ? step_launch<true, true>(p, c, s, mis) : step_launch<true, false>(p, c, s, mis);
    else ps ? step_launch<false, true>(p, c, s, mis) : step_launch<false, false>(p, c, s, mis);
}
void launch_shadow(const Params& p, const LaunchCfg& c, cudaStream_t s) {
    if (p.S.has_transmit) step_dispatch(p, c, s, false);
    else shadow_dispatch<false>(p, c, s);
}
template <bool kAny, bool kCurves, bool kPersist, bool kAdj, bool kMotion = false>
static void mis_launch(const Params& p, const LaunchCfg& c, cudaStream_t s) {
    auto k = k_mis<kAny, kCurves, kPersist, kAdj, kMotion>;
    k<<<traversal_grid<kPersist>(k, c), kPersistBlock, 0, s>>>(p);
}
void launch_mis(const Params& p, const LaunchCfg& c, cudaStream_t s) {
    const bool cv = p.S.has_curves != 0, ps = c.persistent != 0, any = !p.S.has_emitters;
    if (p.S.has_transmit) {
        step_dispatch(p, c, s, true);
    } else if (p.S.has_motion) {
        if (any) cv ? mis_launch<true, true, true, false, true>(p, c, s) : mis_launch<true, false, true, false, true>(p, c, s);
        else cv ? mis_launch<false, true, true, false, true>(p, c, s) : mis_launch<false, false, true, false, true>(p, c, s);
    } else if (any) {
        if (cv) ps ? mis_launch<true, true, true, false>(p, c, s) : mis_launch<true, true, false, false>(p, c, s);
        else ps ? mis_launch<true, false, true, false>(p, c, s) : mis_launch<true, false, false, false>(p, c, s);
    } else {
        if (cv) ps ? mis_launch<false, true, true, false>(p, c, s) : mis_launch<false, true, false, false>(p, c, s);
        else ps ? mis_launch<false, false, true, false>(p, c, s) : mis_launch<false, false, false, false>(p, c, s);
    }
}

// Adjoint replay. The MIS rays always look for the surface they hit (the
// emission gradient needs the emissive material), which gives the same Li as
// the any-hit form the forward pass may use.
void launch_adj_init(const Params& p, const LaunchCfg& c, cudaStream_t s) {
    k_adj_init<<<blocks_for(p.chunk_paths, 256, c.grid_cap), 256, 0, s>>>(p);
}
void launch_shade_adj(const Params& p, const LaunchCfg& c0, cudaStream_t s) {
    LaunchCfg c = c0;
    c.block = std::min(c.block, kShadeBlock);
    const int g = std::min(c.grid_cap, c.stage_grid);
    if (p.S.has_fibers) k_shade<true, true, false><<<g, c.block, 0, s>>>(p);
    else k_shade<true, false, false><<<g, c.block, 0, s>>>(p);
}
void launch_shadow_adj(const Params& p, const LaunchCfg& c, cudaStream_t s) { shadow_dispatch<true>(p, c, s); }
void launch_mis_adj(const Params& p, const LaunchCfg& c, cudaStream_t s) {
    const bool cv = p.S.has_curves != 0, ps = c.persistent != 0;
    if (cv) ps ? mis_launch<false, true, true, true>(p, c, s) : mis_launch<false, true, false, true>(p, c, s);
    else ps ? mis_launch<false, false, true, true>(p, c, s) : mis_launch<false, false, false, true>(p, c, s);
}
void launch_adj_direct(const Params& p, const LaunchCfg& c, cudaStream_t s) {
    k_adj_direct<<<std::min(c.grid_cap, c.stage_grid), 256, 0, s>>>(p);
}
void launch_film(const Params& p, const LaunchCfg& c, cudaStream_t s) {
    k_film<<<blocks_for(p.chunk_pixels, 256, c.grid_cap), 256, 0, s>>>(p);
}
template <bool kAny, bool kCurves, bool kPersist, bool kMotion = false>
static void tb_launch(const DevScene& S, uint32_t scene, const float* rays, const float* times, uint32_t n,
                      ana_hit* out, uint32_t* fetch, uint32_t* err, int grid, cudaStream_t s) {
    auto k = k_trace_batch<kAny, kCurves, kPersist, kMotion>;
    int g = kPersist ? resident_grid(k) : grid;
    k<<<g, kPersistBlock, 0, s>>>(S, scene, rays, times, n, out, fetch, err);
}
void launch_trace_batch(const DevScene& S, uint32_t scene, const float* rays, const float* times, size_t n,
                        ana_hit* out, int occlusion,
                        uint32_t* fetch, uint32_t* err, int persistent, cudaStream_t s) {
    const bool cv = S.has_curves != 0;
    int grid = blocks_for(uint32_t(n), kPersistBlock, 1 << 20);
    uint32_t nn = uint32_t(n);
    if (S.has_motion) {
        if (occlusion) cv ? tb_launch<true, true, true, true>(S, scene, rays, times, nn, out, fetch, err, grid, s)
                          : tb_launch<true, false, true, true>(S, scene, rays, times, nn, out, fetch, err, grid, s);
        else cv ? tb_launch<false, true, true, true>(S, scene, rays, times, nn, out, fetch, err, grid, s)
                : tb_launch<false, false, true, true>(S, scene, rays, times, nn, out, fetch, err, grid, s);
    } else if (occlusion) {
        if (cv) persistent ? tb_launch<true, true, true>(S, scene, rays, times, nn, out, fetch, err, grid, s)
                           : tb_launch<true, true, false>(S, scene, rays, times, nn, out, fetch, err, grid, s);
        else persistent ? tb_launch<true, false, true>(S, scene, rays, times, nn, out, fetch, err, grid, s)
                        : tb_launch<true, false, false>(S, scene, rays, times, nn, out, fetch, err, grid, s);
    } else {
        if (cv) persistent ? tb_launch<false, true, true>(S, scene, rays, times, nn, out, fetch, err, grid, s)
                           : tb_launch<false, true, false>(S, scene, rays, times, nn, out, fetch, err, grid, s);
        else persistent ? tb_launch<false, false, true>(S, scene, rays, times, nn, out, fetch, err, grid, s)
                        : tb_launch<false, false, false>(S, scene, rays, times, nn, out, fetch, err, grid, s);
    }
}

// ---------------------------------------------------------------------------
// BSDF queries (ana_bsdf_batch): IMaterial::evaluate and IMaterial::sample of
// one material over a batch of shading frames, through the same device
// functions the shade kernel calls (make_ctx, mat_eval, mat_sample).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_bsdf_query(DevMaterial m, const ana_bsdf_query* q, uint32_t n,
                                                    ana_bsdf_result* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const ana_bsdf_query Q = q[i];
    SurfInt si;
    si.p = f3(0.f, 0.f, 0.f);
    si.n = f3(Q.n[0], Q.n[1], Q.n[2]);
    si.ng = si.n;
    si.dpdu = f3(Q.t[0], Q.t[1], Q.t[2]);
    si.color = f3(Q.color[0], Q.color[1], Q.color[2]);
    si.slot = 0;
    si.is_curve = Q.is_curve != 0;
    const float3 wo = f3(Q.wo[0], Q.wo[1], Q.wo[2]);
    const ShadeCtx c = make_ctx(si, -wo);
    const BsdfEval e = mat_eval(m, c, wo, f3(Q.wi[0], Q.wi[1], Q.wi[2]));
    const BsdfSample b = mat_sample(m, c, wo, Q.u[0], Q.u[1], Q.u_comp);
    ana_bsdf_result r;
    r.f[0] = e.f.x;
    r.f[1] = e.f.y;
    r.f[2] = e.f.z;
    r.pdf = e.pdf;
    const bool ok = b.valid();
    r.sample_f[0] = ok ? b.f.x : 0.f;
    r.sample_f[1] = ok ? b.f.y : 0.f;
    r.sample_f[2] = ok ? b.f.z : 0.f;
    r.sample_pdf = ok ? b.pdf : 0.f;
    r.sample_wi[0] = ok ? b.wi.x : 0.f;
    r.sample_wi[1] = ok ? b.wi.y : 0.f;
    r.sample_wi[2] = ok ? b.wi.z : 0.f;
    r.sample_flags = ok ? b.flags : 0u;
    out[i] = r;
}

void launch_bsdf_query(const DevMaterial& m, const ana_bsdf_query* q, uint32_t n, ana_bsdf_result* out,
                       cudaStream_t s) {
    k_bsdf_query<<<blocks_for(n, 128, 1 << 20), 128, 0, s>>>(m, q, n, out);
}

// ---------------------------------------------------------------------------
// Scratch of the allocation-free trace entry point: module global memory,
// created with the module on each device (about 4 MiB), so the entry point
// never asks the allocator for memory. One copy per device, shared by every
// context on that device.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_trace[kNoAllocBytes];

// The address is cached per device together with the context it was looked
// up in: a device reset (cudaDeviceReset) destroys the primary context and
// the module with it, and the next context loads the module again, possibly
// elsewhere. The current context comes from the driver's cuCtxGetCurrent,
// reached through cudaGetDriverEntryPoint (no link against the driver
// library).
static cudaError_t current_context(void** ctx) {
    using GetCurrent = int (*)(void**);
    static GetCurrent fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        const cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q);
        if (e != cudaSuccess) return e;
        if (q != cudaDriverEntryPointSuccess || !f) return cudaErrorSymbolNotFound;
        fn = reinterpret_cast<GetCurrent>(f);
    }
    return fn(ctx) == 0 ? cudaSuccess : cudaErrorDeviceUninitialized;
}

cudaError_t noalloc_trace_scratch(int device, unsigned char** base) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static void* addr[kMaxDevices] = {};
    static void* owner[kMaxDevices] = {};  // the context each address belongs to
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    void* ctx = nullptr;
    cudaError_t e = current_context(&ctx);
    if (e != cudaSuccess) return e;
    if (!addr[device] || owner[device] != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_trace);
        if (e != cudaSuccess) return e;
        addr[device] = p;
        owner[device] = ctx;
    }
    *base = static_cast<unsigned char*>(addr[device]);
    return cudaSuccess;
}

}  // namespace ana
