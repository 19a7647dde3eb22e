// Closest-hit and any-hit traversal of the triangle BVH2 and the curve BVH2.
//
// Hit-identity parity: the triangle test restates BVHBackend::intersectTriangle
// (src/accel/BVHBackend.cpp:264-283) with every operation rounded on its own
// (no FMA), so (t, u, v) equal the reference's float results compiled without
// contraction; the box tests restate intersectAABB (BVHBackend.cpp:249-262):
// ray tMin/tMax, the dirNeg slab selection and the `tMax <= tMin` rejection,
// plus the caller's `tNear > closestT` cull; the curve path restates
// CurveBrute::trace's aabbHit and the ray-ribbon subdivide
// (src/accel/CurveBrute.cpp:85-234, 478-498).
#pragma once
#include <type_traits>
#include "dmath.cuh"
#include "layout.h"
#include "motion.cuh"

namespace ana {

struct Ray {
    float3 o, d;
    float tmin, tmax;
    float time;  // normalized shutter time (motion-blurred meshes)
};

// BVHBackend::makeRay4 (BVHBackend.cpp:233-247): invDir = 1/safe(d) where
// safe(v) = |v| > 1e-9 ? v : 1e-9 (the sign of tiny components is dropped),
// and the triangle test rebuilds dir = 1/invDir.
struct TriRay {
    float3 o, inv, dir;
    float tmin, tmax;
    bool nx, ny, nz;
};

__device__ __forceinline__ float safe_comp(float v) { return fabsf(v) > 1e-9f ? v : 1e-9f; }

__device__ __forceinline__ TriRay make_tri_ray(const Ray& r) {
    TriRay q;
    q.o = r.o;
    q.inv = f3(xdiv(1.f, safe_comp(r.d.x)), xdiv(1.f, safe_comp(r.d.y)), xdiv(1.f, safe_comp(r.d.z)));
    q.dir = f3(xdiv(1.f, q.inv.x), xdiv(1.f, q.inv.y), xdiv(1.f, q.inv.z));
    q.tmin = r.tmin;
    q.tmax = r.tmax;
    q.nx = r.d.x < 0.f;
    q.ny = r.d.y < 0.f;
    q.nz = r.d.z < 0.f;
    return q;
}

// Slab test of one child box. Returns true and tNear when the box is entered
// before `cull` (the current closest hit) and its interval is not empty.
__device__ __forceinline__ bool box_hit(const TriRay& r, float lox, float hix, float loy, float hiy,
                                        float loz, float hiz, float cull, float& tnear) {
    float nx = r.nx ? hix : lox, fx = r.nx ? lox : hix;
    float ny = r.ny ? hiy : loy, fy = r.ny ? loy : hiy;
    float nz = r.nz ? hiz : loz, fz = r.nz ? loz : hiz;
    float t0x = xmul(xsub(nx, r.o.x), r.inv.x), t1x = xmul(xsub(fx, r.o.x), r.inv.x);
    float t0y = xmul(xsub(ny, r.o.y), r.inv.y), t1y = xmul(xsub(fy, r.o.y), r.inv.y);
    float t0z = xmul(xsub(nz, r.o.z), r.inv.z), t1z = xmul(xsub(fz, r.o.z), r.inv.z);
    float tmn = fmaxf(fmaxf(fmaxf(r.tmin, t0x), t0y), t0z);
    float tmx = fminf(fminf(fminf(r.tmax, t1x), t1y), t1z);
    tnear = tmn;
    return tmx > tmn && tmn <= cull;
}

// Moller-Trumbore, BVHBackend::intersectTriangle.
__device__ __forceinline__ bool tri_hit(const TriRay& r, float3 v0, float3 e1, float3 e2, float tmax,
                                        float& t, float& u, float& v) {
    float3 h = xcross(r.dir, e2);
    float a = xdot(e1, h);
    if (fabsf(a) < 1e-9f) return false;
    float f = xdiv(1.f, a);
    float3 s = xsub3(r.o, v0);
    u = xmul(f, xdot(s, h));
    if (u < 0.f || u > 1.f) return false;
    float3 q = xcross(s, e1);
    v = xmul(f, xdot(r.dir, q));
    if (v < 0.f || xadd(u, v) > 1.f) return false;
    t = xmul(f, xdot(e2, q));
    return t >= r.tmin && t <= tmax;
}

// Stack entry: interior node index, or a leaf (bit 31) with count-1 in bits
// 25..30 and the first primitive in bits 0..24.
__device__ __forceinline__ uint32_t leaf_entry(uint32_t off, uint32_t cnt) {
    return 0x80000000u | ((cnt - 1u) << 25) | off;
}

struct TriHit {
    float t, u, v;
    int32_t tri;  // leaf-order index, -1 on miss
};

struct Counters {
    uint32_t nodes, prims, segs, cnodes;  // triangle nodes, triangles, segments, curve nodes
};

// ---------------------------------------------------------------------------
// Persistent-warp triangle traversal. Each lane owns one ray at a time; a
// warp loops over
//   1. refill: once enough lanes are without a ray (kRefill*), they take the
//      next queue entries together (one warp-aggregated atomicAdd on the
//      stage's fetch counter);
//   2. interior phase: lanes descend interior nodes until they reach a
//      leaf; the phase ends when every lane has a leaf to test (or nothing
//      left), when no lane can take another interior step, or when at most
//      kLeafPhaseLanes (any hit: kLeafPhaseLanesAny) lanes still descend
//      while others wait with a leaf, so lanes stay converged on the
//      node-test code. Any-hit queries can be speculative (kPark; Aila and
//      Laine, "Understanding the efficiency of ray traversal on GPUs", 2009):
//      a lane that reaches a leaf parks it and keeps descending from its next
//      stack entry. Closest-hit queries do not speculate: a leaf tested early
//      shortens the ray and culls later nodes (measured on the throughput
//      frame: speculation cost closest hit 3 %, saved any hit 8-12 % with
//      one-lane refills; with grouped refills it costs the triangle shadow
//      and MIS kernels too, and only the curve shadow kernels and the
//      occlusion queries of ana_trace_batch park);
//   3. leaf phase: the parked leaf's (else the current leaf's) triangles.
// A lane whose stack is exhausted (or, for occlusion, that found a blocker)
// reports its ray and picks up a new one at the next refill, so finished rays
// do not idle the warp until its slowest ray completes. Box and triangle
// tests are the same functions as above, so results are identical.
// ---------------------------------------------------------------------------
// Interior phases end once this few lanes still descend (and a lane has a
// leaf). On the 1920x1080x64 throughput frame the extend stage took 142.0 ms
// when the phase ran until no lane descended, 118.4 ms at 4 lanes, 117.2 ms at
// 8 and 124.6 ms at 16; the any-hit shadow + MIS stages, parking leaves and
// refilling one lane at a time, 146.5 ms, 137.0 at 4, 132.8 at 8, 128.1 at 16,
// 129.8 at 24 and 191.2 at 32. Any-hit kernels that test leaves as reached use
// the closest-hit count (shadow + MIS 107.0 ms at 8, 111.4 at 4, 108.1 at 12,
// 111.9 at 16); the parked count serves the kernels that still park (curve
// shadow rays, occlusion queries of ana_trace_batch). Kernels with
// motion-blurred meshes, whose leaf tests invert interpolated matrices, keep
// the phase until no lane descends (1280x720x16 motion frame: 25.9 ms against
// 28.6 ms at 8 / 16 lanes). Hits and occlusion answers are unchanged.
constexpr uint32_t kLeafPhaseLanes = 8;      // closest hit, any hit without parking
constexpr uint32_t kLeafPhaseLanesAny = 16;  // any hit (parked leaves)

// Refill thresholds: idle lanes take new rays only once at least this many
// lanes of the warp are idle (or the queue is drained and every lane is).
// Queue entries in path order are the samples of one pixel, so lanes that
// start together trace neighbouring rays and stay converged, where one lane
// refilled at a time starts at the root beside lanes deep in the tree. On the
// 1920x1080x64 throughput frame (closest hit / any hit thresholds): extend
// 115.7 ms at 1, 114.6 at 4, 111.0 at 8, 108.8 at 12, 108.3 at 14, 107.7 at
// 16, 108.2 at 18, 108.4 at 20, 112.4 at 24, 122.5 at 28, 140.5 at 32; shadow +
// MIS 128.3 ms at 1, 127.3 at 8, 126.8 at 12, 127.2 at 16, 134.6 at 20. The
// curve kernels' ribbon walks diverge anyway and want smaller groups: the
// 1280x720x32 hair frame's extend stage 647.5 ms at 1, 634.2 at 4, 636.7 at 6,
// 642.9 at 8, 649.3 at 10, 657.7 at 12; its shadow stage 376.6 ms at 1, 370.4
// at 2, 369.6 at 3, 371.0 at 4, 376.4 at 6, 384.0 at 8.
constexpr int kRefillLanes = 16;
constexpr int kRefillLanesAny = 12;
constexpr int kRefillLanesCurves = 4;
constexpr int kRefillLanesCurvesAny = 4;

struct Traversal {
    TriRay r;
    float closest, u, v;
    int32_t tri;
    uint32_t cur;
    int sp;
    bool exhausted;
    // curve stage (scenes with curves): the triangle BVH is traversed first,
    // then the curve BVH from the triangle hit distance (CurveBrute::trace)
    uint32_t stage;  // 0 triangles, 1 curves
    int32_t seg;     // leaf-order segment of the closest ribbon hit, -1 if none
    float tseg;
    float3 tang;
    float3 cd, fx, fy, cinv;  // exact direction, ray-space frame x/y, 1/d
    float time;               // ray time: object rays of motion-blurred triangles
};

// Starts a traversal at a scene's root (kNoRoot: the scene has no triangles).
// Closest hit keeps the nearest accepted triangle; ties (t == closest) go to
// the later-tested triangle, as `t <= r.tMax` does in the reference; any hit
// (kAny) stops at the first accepted triangle (BVHBackend::occluded,
// BVHBackend.cpp:409-444).
__device__ __forceinline__ void trav_init(Traversal& T, const Ray& ray, uint32_t root) {
    T.r = make_tri_ray(ray);
    T.cd = ray.d;  // read by the motion test (and reset by curve_begin)
    T.time = ray.time;
    T.closest = ray.tmax;
    T.u = T.v = 0.f;
    T.tri = -1;
    T.cur = root;
    T.sp = 0;
    T.exhausted = root == kNoRoot;
    T.stage = 0;
    T.seg = -1;
}

// Traversal stack entry (thread-local memory): x = node or leaf entry, y = the
// entry distance's bits (closest hit; any hit writes x only). One 64-bit
// access per push and pop instead of two 32-bit ones: the throughput frame's
// extend stage 116.4 -> 115.7 ms, the 1920x1080x64 hair frame 4549 -> 4505 ms.
template <bool kAny = false>
__device__ __forceinline__ bool trav_pop(Traversal& T, const uint2* stack) {
    if (kAny) {  // an any-hit query ends at its first hit: nothing on the stack is culled
        if (T.sp == 0) return false;
        T.cur = stack[--T.sp].x;
        return true;
    }
    while (T.sp > 0) {
        --T.sp;
        const uint2 e = stack[T.sp];
        if (__uint_as_float(e.y) > T.closest) continue;
        T.cur = e.x;
        return true;
    }
    return false;
}

// Interior step: one 128-byte node fetch and four child-box tests. The
// children entered are ordered by entry distance with a 4-key sorting
// network; the nearest becomes the current node, the others are pushed
// farthest first (popped nearest first, and skipped once a closer hit is
// known). Any-hit queries skip the sort and the entry distances: the children
// entered are taken in stored order, and nothing is culled at a pop because
// the query ends at its first hit. On the 1920x1080x64 throughput frame that
// cut the shadow and MIS stages from 72.9 and 125.7 ms to 60.2 and 85.1 ms;
// near first without keys (the shortcuts below) measured 66.6 and 113.3 ms,
// so the stored order (the SAH build's lower side of each split first) finds
// blockers sooner there. The curve BVH keeps near-first any-hit steps, which
// measured faster on the hair frame.
__device__ __forceinline__ void cswap(float& ka, uint32_t& va, float& kb, uint32_t& vb) {
    if (kb < ka) {
        const float k = ka;
        ka = kb;
        kb = k;
        const uint32_t v = va;
        va = vb;
        vb = v;
    }
}

// Enters the children a closest-hit step found (key: entry distance, +inf
// for a child not entered): the nearest becomes the current node, the others
// are pushed farthest first (popped nearest first, and skipped once a closer
// hit is known). Children entered are ordered with a 4-key sorting network,
// which keeps equal keys in stored order; one or two children entered (most
// steps of incoherent rays) skip the network with the same result (extend
// stage of the throughput frame: 146.6 -> 141.9 ms). Shared by the triangle
// and the curve BVH steps.
__device__ __forceinline__ void enter_near_first(Traversal& T, float (&key)[4], uint32_t (&ref)[4], uint2* stack, uint32_t* err) {
    const int n = int(key[0] < INFINITY) + int(key[1] < INFINITY) + int(key[2] < INFINITY) + int(key[3] < INFINITY);
    if (n == 0) {
        if (!trav_pop(T, stack)) T.exhausted = true;
        return;
    }
    if (n == 1) {  // one child entered: it becomes the current node
        T.cur = key[0] < INFINITY ? ref[0] : key[1] < INFINITY ? ref[1] : key[2] < INFINITY ? ref[2] : ref[3];
        return;
    }
    if (n == 2) {  // two entered: the first and the last in stored order, nearer first
        const bool h0 = key[0] < INFINITY, h1 = key[1] < INFINITY;
        const bool g3 = key[3] < INFINITY, g2 = key[2] < INFINITY;
        float ka = h0 ? key[0] : h1 ? key[1] : key[2];
        uint32_t ra = h0 ? ref[0] : h1 ? ref[1] : ref[2];
        float kb = g3 ? key[3] : g2 ? key[2] : key[1];
        uint32_t rb = g3 ? ref[3] : g2 ? ref[2] : ref[1];
        if (T.sp + 1 > int(kMaxStack4)) {
            atomicOr(err, 1u);
            T.exhausted = true;
            return;
        }
        cswap(ka, ra, kb, rb);
        stack[T.sp] = make_uint2(rb, __float_as_uint(kb));
        ++T.sp;
        T.cur = ra;
        return;
    }
    // misses carry key +inf, so the n children entered come first
    cswap(key[0], ref[0], key[1], ref[1]);
    cswap(key[2], ref[2], key[3], ref[3]);
    cswap(key[0], ref[0], key[2], ref[2]);
    cswap(key[1], ref[1], key[3], ref[3]);
    cswap(key[1], ref[1], key[2], ref[2]);
    if (T.sp + n - 1 > int(kMaxStack4)) {
        atomicOr(err, 1u);
        T.exhausted = true;
        return;
    }
#pragma unroll
    for (int k = 3; k >= 1; --k) {
        if (k < n) {
            stack[T.sp] = make_uint2(ref[k], __float_as_uint(key[k]));
            ++T.sp;
        }
    }
    T.cur = ref[0];
}

template <bool kAny, bool kCount>
__device__ __forceinline__ void trav_interior(Traversal& T, const DevScene& S, uint2* stack,
                                              uint32_t* err, Counters* cnt) {
    const float4* np = reinterpret_cast<const float4*>(S.tri_nodes + T.cur);
    const float4 lx = ldg4(np), hx = ldg4(np + 1), ly = ldg4(np + 2), hy = ldg4(np + 3), lz = ldg4(np + 4),
                 hz = ldg4(np + 5), rf = ldg4(np + 6);
    if (kCount) cnt->nodes++;
    const float cull = kAny ? T.r.tmax : T.closest;
    float key[4];
    uint32_t ref[4] = {fbits_u(rf.x), fbits_u(rf.y), fbits_u(rf.z), fbits_u(rf.w)};
    {
        const float l0[4] = {lx.x, lx.y, lx.z, lx.w}, h0[4] = {hx.x, hx.y, hx.z, hx.w};
        const float l1[4] = {ly.x, ly.y, ly.z, ly.w}, h1[4] = {hy.x, hy.y, hy.z, hy.w};
        const float l2[4] = {lz.x, lz.y, lz.z, lz.w}, h2[4] = {hz.x, hz.y, hz.z, hz.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float tn;
            const bool h = ref[k] != kEmptyChild && box_hit(T.r, l0[k], h0[k], l1[k], h1[k], l2[k], h2[k], cull, tn);
            key[k] = h ? tn : INFINITY;
        }
    }
    if constexpr (kAny) {  // any hit: children entered in stored order, no distance sort
        const int n = int(key[0] < INFINITY) + int(key[1] < INFINITY) + int(key[2] < INFINITY) + int(key[3] < INFINITY);
        if (n == 0) {
            if (!trav_pop<kAny>(T, stack)) T.exhausted = true;
            return;
        }
        if (T.sp + n - 1 > int(kMaxStack4)) {
            atomicOr(err, 1u);
            T.exhausted = true;
            return;
        }
        uint32_t first = kEmptyChild;
#pragma unroll
        for (int k = 3; k >= 0; --k) {
            if (key[k] < INFINITY) {
                if (first != kEmptyChild) stack[T.sp++].x = first;
                first = ref[k];
            }
        }
        T.cur = first;
        return;
    }
    enter_near_first(T, key, ref, stack, err);
}

// BVHBackend::makeObjectSpaceRay4: the world ray (origin, exact direction)
// taken to the object space of motion mesh `mm` at the ray's time.
__device__ __forceinline__ TriRay object_ray(const DevScene& S, uint32_t mm, const Traversal& T, float tmax) {
    M4 o2w, w2o;
    o2w_at(S, mm, T.time, o2w);
    m4_inverse(o2w, w2o);
    Ray r;
    r.o = m4_point(w2o, T.r.o);
    r.d = m4_vector(w2o, T.cd);
    r.tmin = T.r.tmin;
    r.tmax = tmax;
    r.time = T.time;
    return make_tri_ray(r);
}

// Tests the triangles of leaf entry `leaf`; true when an any-hit query found
// its blocker. kMotion: triangles flagged object-space (bit 31 of the index
// word) meet the ray in their mesh's object space at the ray's time.
template <bool kAny, bool kCount, bool kMotion = false>
__device__ __forceinline__ bool leaf_test(Traversal& T, const DevScene& S, uint32_t leaf, Counters* cnt) {
    const uint32_t off = leaf & 0x01FFFFFFu, c = ((leaf >> 25) & 63u) + 1u;
    // the object ray of the leaf's last motion mesh, reused while the mesh
    // repeats (the same value the reference recomputes per triangle)
    uint32_t cachedMM = 0xFFFFFFFFu;
    TriRay ro;
    for (uint32_t i = off; i < off + c; ++i) {
        const float4* tp = S.tri_isect + 3 * size_t(i);
        float4 a = ldg4(tp), b = ldg4(tp + 1), e = ldg4(tp + 2);
        if (kCount) cnt->prims++;
        float t, u, v;
        const float tmax = kAny ? T.r.tmax : T.closest;
        bool h;
        if (kMotion && (__float_as_uint(a.w) & 0x80000000u)) {
            const uint32_t mm = __float_as_uint(b.w);
            if (mm != cachedMM) {
                ro = object_ray(S, mm, T, tmax);
                cachedMM = mm;
            }
            h = tri_hit(ro, f3(a), f3(b), f3(e), tmax, t, u, v);
        } else {
            h = tri_hit(T.r, f3(a), f3(b), f3(e), tmax, t, u, v);
        }
        if (h) {
            T.closest = t;
            T.u = u;
            T.v = v;
            T.tri = int32_t(i);
            if (kAny) return true;
        }
    }
    return false;
}

// Leaf step of the one-thread-per-ray schedule: test the current leaf, then pop.
template <bool kAny, bool kCount>
__device__ __forceinline__ void trav_leaf(Traversal& T, const DevScene& S, const uint2* stack, Counters* cnt) {
    if (leaf_test<kAny, kCount>(T, S, T.cur, cnt)) {
        T.exhausted = true;
        return;
    }
    if (!trav_pop<kAny>(T, stack)) T.exhausted = true;
}

// ===========================================================================
// Curves
// ===========================================================================

// CurveBrute::aabbHit (CurveBrute.cpp:478-498).
__device__ __forceinline__ bool curve_box_hit(const Ray& r, float3 inv, float lox, float hix, float loy,
                                              float hiy, float loz, float hiz, float maxT, float& tnear) {
    float tmn = r.tmin, tmx = maxT;
    float lo[3] = {lox, loy, loz}, hi[3] = {hix, hiy, hiz};
    float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z}, iv[3] = {inv.x, inv.y, inv.z};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (fabsf(d[i]) < 1e-9f) {
            if (o[i] < lo[i] || o[i] > hi[i]) return false;
            continue;
        }
        float t0 = xmul(xsub(lo[i], o[i]), iv[i]);
        float t1 = xmul(xsub(hi[i], o[i]), iv[i]);
        if (iv[i] < 0.f) {
            float tt = t0;
            t0 = t1;
            t1 = tt;
        }
        tmn = fmaxf(tmn, t0);
        tmx = fminf(tmx, t1);
        if (tmx < tmn) return false;
    }
    tnear = tmn;
    return true;
}

// Ray-space frame of makeRayFrame (CurveBrute.cpp:29-47): z = direction, x/y
// from buildOrthonormalBasis (Types.h:108-114).
struct RayFrame {
    float3 o, x, y, z;
};

__device__ __forceinline__ void onb_exact(float3 n, float3& t, float3& b) {
    float sign = copysignf(1.f, n.z);
    float a = xdiv(-1.f, xadd(sign, n.z));
    float bb = xmul(xmul(n.x, n.y), a);
    t = f3(xadd(1.f, xmul(xmul(xmul(sign, n.x), n.x), a)), xmul(sign, bb), -xmul(sign, n.x));
    b = f3(bb, xadd(sign, xmul(xmul(n.y, n.y), a)), -n.y);
}

__device__ __forceinline__ RayFrame make_frame(const Ray& r) {
    RayFrame f;
    f.o = r.o;
    f.z = r.d;
    onb_exact(r.d, f.x, f.y);
    return f;
}

__device__ __forceinline__ float3 project(const RayFrame& f, float3 p) {
    float3 q = xsub3(p, f.o);
    return f3(xdot(q, f.x), xdot(q, f.y), xdot(q, f.z));
}

__device__ __forceinline__ float3 xmid(float3 a, float3 b) { return xmul3(xadd3(a, b), 0.5f); }

// bezierTangent (CurveBrute.cpp:59-64)
__device__ __forceinline__ float3 bezier_tangent(float3 P0, float3 P1, float3 P2, float3 P3, float t) {
    float mt = xsub(1.f, t);
    float3 a = xmul3(xsub3(P1, P0), xmul(xmul(3.f, mt), mt));
    float3 b = xmul3(xsub3(P2, P1), xmul(xmul(6.f, mt), t));
    float3 c = xmul3(xsub3(P3, P2), xmul(xmul(3.f, t), t));
    return xadd3(xadd3(a, b), c);
}

__device__ __forceinline__ float min4(float a, float b, float c, float d) {
    return fminf(fminf(a, b), fminf(c, d));
}
__device__ __forceinline__ float max4(float a, float b, float c, float d) {
    return fmaxf(fmaxf(a, b), fmaxf(c, d));
}

// The bounds tests of subdivide (CurveBrute.cpp:97-117) on projected control
// points: depth range against [tmin, bestT], and the projected box's distance
// from the ray axis against the larger half-width. zlo receives zMin - maxHalfW.
__device__ __forceinline__ bool ribbon_bounds(float3 c0, float3 c1, float3 c2, float3 c3, float hw0, float hw3,
                                              float tmin, float bestT, float& zlo) {
    const float maxHalfW = fmaxf(hw0, hw3);
    const float zMin = min4(c0.z, c1.z, c2.z, c3.z), zMax = max4(c0.z, c1.z, c2.z, c3.z);
    zlo = xsub(zMin, maxHalfW);
    if (zlo > bestT) return false;
    if (xadd(zMax, maxHalfW) < tmin) return false;
    const float xMin = min4(c0.x, c1.x, c2.x, c3.x), xMax = max4(c0.x, c1.x, c2.x, c3.x);
    const float yMin = min4(c0.y, c1.y, c2.y, c3.y), yMax = max4(c0.y, c1.y, c2.y, c3.y);
    const float cx = (0.f < xMin) ? xMin : (0.f > xMax ? xMax : 0.f);
    const float cy = (0.f < yMin) ? yMin : (0.f > yMax ? yMax : 0.f);
    return !(xadd(xmul(cx, cx), xmul(cy, cy)) > xmul(maxHalfW, maxHalfW));
}

struct SubSeg {
    float3 P0, P1, P2, P3;  // world-space control points
    float zlo;              // zMin - maxHalfW: the test that depends on bestT
    uint32_t dp;            // depth (bits 0-2, 6 = root) | path from the root (bits 3-8, 1 = right)
};

// The half-widths and strand-parameter interval of the node (depth, path)
// below a segment's (hw0r, hw3r, toffr, tscr): the splits' own updates
// (CurveBrute.cpp:152-176) replayed from the root.
__device__ __forceinline__ void ribbon_params(uint32_t dp, float hw0r, float hw3r, float toffr, float tscr,
                                              float& hw0, float& hw3, float& toff, float& tscale) {
    const int levels = 6 - int(dp & 7u);
    const uint32_t path = dp >> 3;
    hw0 = hw0r;
    hw3 = hw3r;
    toff = toffr;
    tscale = tscr;
    for (int k = levels - 1; k >= 0; --k) {
        const float hm = xmul(xadd(hw0, hw3), 0.5f), tsh = xmul(tscale, 0.5f);
        if ((path >> k) & 1u) {
            hw0 = hm;
            toff = xadd(toff, tsh);
        } else {
            hw3 = hm;
        }
        tscale = tsh;
    }
}

// subdivide (CurveBrute.cpp:85-176): depth-6 de Casteljau subdivision in ray
// space, the left half first, updating bestT on a closer hit. The reference
// projects a node's four control points when it visits the node; a child
// shares two of them with its parent and one with its sibling, so here a split
// projects the five new points once (the same world points give the same
// projections), both children are bounds-tested at once and only survivors are
// pushed. The one test that depends on bestT (which only decreases) is
// repeated when a child is popped, so every node is accepted or culled, and
// every leaf evaluated, exactly as in the recursion and in the same order.
// A stack entry keeps the node's four world points, that test's bound and its
// (depth, path); the end points' projections are recomputed at a pop and the
// half-widths and parameter interval replayed along the path with the same
// operations (56 instead of 100 bytes per entry: hair frame's shadow stage
// 398.6 -> 379.3 ms). (A walk that kept no points at all, rebuilding each
// right half from the segment's four points along its path, measured slower:
// extend 1024 against 842 ms at leaves of four.)
__device__ __forceinline__ bool ribbon_hit(const RayFrame& fr, float tmin, float3 P0, float3 P1, float3 P2,
                                           float3 P3, float hw0r, float hw3r, float toffr, float tscaler,
                                           float& bestT, float& tSeg, float3& tang) {
    SubSeg st[8];
    int sp = 0;
    {
        const float3 c0 = project(fr, P0), c1 = project(fr, P1), c2 = project(fr, P2), c3 = project(fr, P3);
        float zlo;
        if (!ribbon_bounds(c0, c1, c2, c3, hw0r, hw3r, tmin, bestT, zlo)) return false;
        st[sp++] = SubSeg{P0, P1, P2, P3, zlo, 6u};
    }
    bool hit = false;
    while (sp > 0) {
        const SubSeg s = st[--sp];
        if (s.zlo > bestT) continue;
        float hw0, hw3, toff, tscale;
        ribbon_params(s.dp, hw0r, hw3r, toffr, tscaler, hw0, hw3, toff, tscale);
        const float3 c0 = project(fr, s.P0), c3 = project(fr, s.P3);
        if ((s.dp & 7u) == 0u) {
            const float ax = c0.x, ay = c0.y, bx = c3.x, by = c3.y;
            const float dx = xsub(bx, ax), dy = xsub(by, ay);
            const float lenSq = xadd(xmul(dx, dx), xmul(dy, dy));
            float tLine;
            if (lenSq < 1e-12f) tLine = 0.f;
            else
                tLine = fmaxf(0.f, fminf(1.f, xdiv(xsub(xmul(-ax, dx), xmul(ay, dy)), lenSq)));
            const float px = xadd(ax, xmul(dx, tLine)), py = xadd(ay, xmul(dy, tLine));
            const float dist2 = xadd(xmul(px, px), xmul(py, py));
            const float halfW = xadd(xmul(hw0, xsub(1.f, tLine)), xmul(hw3, tLine));
            if (dist2 > xmul(halfW, halfW)) continue;
            const float tRay = xadd(c0.z, xmul(xsub(c3.z, c0.z), tLine));
            if (tRay < tmin || tRay >= bestT) continue;
            float3 tg = bezier_tangent(s.P0, s.P1, s.P2, s.P3, tLine);
            if (xdot(tg, tg) < 1e-12f) tg = xsub3(s.P3, s.P0);
            const float len = __fsqrt_rn(xdot(tg, tg));
            tg = len > 1e-8f ? xmul3(tg, xdiv(1.f, len)) : f3(0.f, 0.f, 1.f);
            bestT = tRay;
            tSeg = xadd(toff, xmul(tLine, tscale));
            tang = tg;
            hit = true;
            continue;
        }
        const float3 Q01 = xmid(s.P0, s.P1), Q12 = xmid(s.P1, s.P2), Q23 = xmid(s.P2, s.P3);
        const float3 R01 = xmid(Q01, Q12), R12 = xmid(Q12, Q23), M = xmid(R01, R12);
        const float3 cq01 = project(fr, Q01), cr01 = project(fr, R01), cm = project(fr, M),
                     cr12 = project(fr, R12), cq23 = project(fr, Q23);
        const float hwMid = xmul(xadd(hw0, hw3), 0.5f);
        float zl, zr;
        const bool okL = ribbon_bounds(c0, cq01, cr01, cm, hw0, hwMid, tmin, bestT, zl);
        const bool okR = ribbon_bounds(cm, cr12, cq23, c3, hwMid, hw3, tmin, bestT, zr);
        const uint32_t cd = (s.dp & 7u) - 1u, cp = (s.dp >> 3) << 1;
        if (okR) st[sp++] = SubSeg{M, R12, Q23, s.P3, zr, cd | ((cp | 1u) << 3)};
        if (okL) st[sp++] = SubSeg{s.P0, Q01, R01, M, zl, cd | (cp << 3)};
    }
    return hit;
}

// ---------------------------------------------------------------------------
// Curve stage of a traversal (CurveBrute::trace's curve pass,
// CurveBrute.cpp:398-440): after the triangle BVH, the curve BVH is traversed
// from the triangle hit distance, keeping only strictly closer ribbon hits.
// Node and leaf steps mirror the triangle ones, so both stages share the
// converged interior / leaf phases and the stack.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void curve_begin(Traversal& T, float3 d, uint32_t segRoot) {
    T.stage = 1;
    T.cd = d;
    onb_exact(d, T.fx, T.fy);
    T.cinv = f3(xdiv(1.f, d.x), xdiv(1.f, d.y), xdiv(1.f, d.z));
    T.cur = segRoot;
    T.sp = 0;
    T.exhausted = segRoot == kNoRoot;
}

// One curve-BVH node: four child boxes (CurveBrute::aabbHit), entered nearest
// first for closest and any hit alike (on the hair frame near-first any-hit
// steps measured faster than the stored order).
template <bool kCount>
__device__ __forceinline__ void curve_interior(Traversal& T, const DevScene& S, uint2* stack,
                                               uint32_t* err, Counters* cnt) {
    const Ray ray{T.r.o, T.cd, T.r.tmin, T.r.tmax};
    const float4* np = reinterpret_cast<const float4*>(S.seg_nodes + T.cur);
    const float4 lx = ldg4(np), hx = ldg4(np + 1), ly = ldg4(np + 2), hy = ldg4(np + 3), lz = ldg4(np + 4),
                 hz = ldg4(np + 5), rf = ldg4(np + 6);
    if (kCount) cnt->cnodes++;
    float key[4];
    uint32_t ref[4] = {fbits_u(rf.x), fbits_u(rf.y), fbits_u(rf.z), fbits_u(rf.w)};
    const float l0[4] = {lx.x, lx.y, lx.z, lx.w}, h0[4] = {hx.x, hx.y, hx.z, hx.w};
    const float l1[4] = {ly.x, ly.y, ly.z, ly.w}, h1[4] = {hy.x, hy.y, hy.z, hy.w};
    const float l2[4] = {lz.x, lz.y, lz.z, lz.w}, h2[4] = {hz.x, hz.y, hz.z, hz.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float tn = 0.f;
        const bool h = ref[k] != kEmptyChild &&
                       curve_box_hit(ray, T.cinv, l0[k], h0[k], l1[k], h1[k], l2[k], h2[k], T.closest, tn);
        key[k] = h ? tn : INFINITY;
    }
    enter_near_first(T, key, ref, stack, err);
}

// Ribbon tests of one curve leaf; true when an any-hit query found its blocker.
template <bool kAny, bool kCount>
__device__ __forceinline__ bool curve_leaf_test(Traversal& T, const DevScene& S, uint32_t leaf, Counters* cnt) {
    const RayFrame fr{T.r.o, T.fx, T.fy, T.cd};
    const uint32_t off = leaf & 0x01FFFFFFu, c = ((leaf >> 25) & 63u) + 1u;
    for (uint32_t i = off; i < off + c; ++i) {
        const float4* sp4 = S.segs + 5 * size_t(i);
        const float4 a = ldg4(sp4), b = ldg4(sp4 + 1), e = ldg4(sp4 + 2), g = ldg4(sp4 + 3);
        if (kCount) cnt->segs++;
        float ts, bt = T.closest;
        float3 tg;
        if (ribbon_hit(fr, T.r.tmin, f3(a), f3(b), f3(e), f3(g), a.w, b.w, e.w, g.w, bt, ts, tg)) {
            T.seg = int32_t(i);
            T.closest = bt;
            T.tseg = ts;
            T.tang = tg;
            if (kAny) return true;
        }
    }
    return false;
}

// Stage dispatch of the node and leaf steps.
template <bool kAny, bool kCount, bool kCurves>
__device__ __forceinline__ void node_step(Traversal& T, const DevScene& S, uint2* stack,
                                          uint32_t* err, Counters* cnt) {
    if (kCurves && T.stage) curve_interior<kCount>(T, S, stack, err, cnt);
    else trav_interior<kAny, kCount>(T, S, stack, err, cnt);
}
template <bool kAny, bool kCount, bool kCurves, bool kMotion = false>
__device__ __forceinline__ bool leaf_step(Traversal& T, const DevScene& S, uint32_t leaf, Counters* cnt) {
    if (kCurves && T.stage) return curve_leaf_test<kAny, kCount>(T, S, leaf, cnt);
    return leaf_test<kAny, kCount, kMotion>(T, S, leaf, cnt);
}

// A lane whose triangle traversal ended moves on to the curve BVH (unless an
// any-hit query already found a blocker). Returns true when the ray is done.
template <bool kAny, bool kCurves>
__device__ __forceinline__ bool stage_done(Traversal& T, float3 d, uint32_t segRoot) {
    if (kCurves && T.stage == 0 && !(kAny && T.tri >= 0)) curve_begin(T, d, segRoot);
    return T.exhausted;
}

// Done(i, T) consumes a finished traversal; Done(i, T, next) -> bool may
// instead ask for entry i to be traced again along `next` (same direction:
// a ray stepping through a transmissive surface) by returning true.
template <class Done>
__device__ __forceinline__ bool trace_again(Done& done, uint32_t i, const Traversal& T, Ray& next) {
    if constexpr (std::is_invocable_r_v<bool, Done&, uint32_t, const Traversal&, Ray&>) {
        return done(i, T, next);
    } else {
        done(i, T);
        return false;
    }
}

// Runs the persistent loop. Load(i, ray, root, segRoot) reads queue entry i
// and its scene's triangle and curve BVH roots; Done consumes the finished
// traversal of entry i (a lane-local call, see trace_again: a lane asked to
// trace again keeps its entry). With kCurves a lane that finishes the
// triangle BVH continues with the curve BVH in the same phases.
// kPark: any-hit lanes park the first leaf they reach and keep descending
// (speculative); false: any-hit lanes test each leaf as they reach it.
template <bool kAny, bool kCount, bool kCurves, bool kMotion, bool kPark, class Load, class Done>
__device__ __forceinline__ void persistent_traverse(const DevScene& S, uint32_t n, uint32_t* fetch, uint32_t* err,
                                                    Counters* cnt, Load load, Done done) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t ltmask = (1u << lane) - 1u;
    uint2 stack[kMaxStack4];
    Traversal T;
    bool active = false, drained = false;
    uint32_t idx = 0, parked = kEmptyChild;
    while (true) {
        // 1. refill idle lanes
        if (!drained) {
            uint32_t need = __ballot_sync(0xFFFFFFFFu, !active);
            constexpr int kRefill = kCurves ? (kAny ? kRefillLanesCurvesAny : kRefillLanesCurves)
                                            : (kAny ? kRefillLanesAny : kRefillLanes);
            if (__popc(need) >= kRefill) {
                uint32_t leader = __ffs(need) - 1u, base = 0;
                if (lane == leader) base = atomicAdd(fetch, __popc(need));
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                if (base >= n) drained = true;
                if (!active) {
                    idx = base + __popc(need & ltmask);
                    if (idx < n) {
                        Ray ray;
                        uint32_t root, segRoot;
                        load(idx, ray, root, segRoot);
                        trav_init(T, ray, root);
                        active = true;
                    }
                }
            }
        }
        if (!__any_sync(0xFFFFFFFFu, active)) break;
        // 2. interior phase (speculative)
        while (true) {
            if (kPark && active && !T.exhausted && (T.cur & 0x80000000u) && parked == kEmptyChild) {
                parked = T.cur;
                if (!trav_pop<kAny>(T, stack)) T.exhausted = true;
            }
            const bool want = active && !T.exhausted && !(T.cur & 0x80000000u);
            const bool ready = !active || T.exhausted || (kPark ? parked != kEmptyChild : bool(T.cur & 0x80000000u));
            const uint32_t wantMask = __ballot_sync(0xFFFFFFFFu, want);
            if (!wantMask || __all_sync(0xFFFFFFFFu, ready)) break;
            // Once at most kPhaseLanes lanes still descend and another lane
            // holds a leaf (any hit: a parked one), the phase ends and the
            // leaves are tested (the descending lanes resume in the next
            // interior phase), so few lanes do not hold the warp in the node
            // loop. A lane with a leaf must exist, so every pass makes progress.
            constexpr uint32_t kPhaseLanes = kMotion ? 0u : (kPark ? kLeafPhaseLanesAny : kLeafPhaseLanes);
            if (kPhaseLanes > 0 && __popc(wantMask) <= kPhaseLanes &&
                __any_sync(0xFFFFFFFFu, active && !T.exhausted &&
                                            (kPark ? parked != kEmptyChild : bool(T.cur & 0x80000000u))))
                break;
            if (want) node_step<kAny, kCount, kCurves>(T, S, stack, err, cnt);
        }
        // 3. leaf phase: one leaf per lane
        if (active) {
            if (parked != kEmptyChild) {
                if (leaf_step<kAny, kCount, kCurves, kMotion>(T, S, parked, cnt)) T.exhausted = true;
                parked = kEmptyChild;
            } else if (!T.exhausted && (T.cur & 0x80000000u)) {
                if (leaf_step<kAny, kCount, kCurves, kMotion>(T, S, T.cur, cnt)) T.exhausted = true;
                else if (!trav_pop<kAny>(T, stack)) T.exhausted = true;
            }
        }
        if (active && T.exhausted && parked == kEmptyChild) {
            bool finished = true;
            if (kCurves && T.stage == 0) {  // the curve BVH follows (the entry is read again for d)
                Ray ray;
                uint32_t root, segRoot;
                load(idx, ray, root, segRoot);
                finished = stage_done<kAny, kCurves>(T, ray.d, segRoot);
            }
            if (finished) {
                Ray next;
                if (trace_again(done, idx, T, next)) {
                    Ray ray;
                    uint32_t root, segRoot;
                    load(idx, ray, root, segRoot);
                    trav_init(T, next, root);
                } else {
                    active = false;
                }
            }
        }
    }
}

}  // namespace ana
