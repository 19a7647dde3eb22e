// Device build of the triangle sections of a scene: BVHBackend::commit's
// triangle setup (src/accel/BVHBackend.cpp:17-111), the binned SAH build of
// buildRecursive / sahSplit (BVHBackend.cpp:120-228) and the 4-wide collapse of
// prepare.cpp's flatten_bvh4, producing the bytes prepare_scene's host path
// produces. Compiled with -fmad=false: every float operation rounds on its own,
// as in the host code (-ffp-contract=off) and the reference.
//
// Schedule. Nodes of more than kSmall triangles are split level by level over
// the whole primitive array: a privatised reduction gives each open node its
// bounds and centroid bounds, a privatised pass fills its 3 x 12 SAH buckets,
// one thread per node sweeps the buckets exactly as sahSplit does, and the
// partition is applied as std::partition (libstdc++, bidirectional form) would
// leave it: the k-th element failing the predicate from the left of the left
// part trades places with the k-th element passing it from the right of the
// right part; both ranks come from one exclusive scan of the predicate. Nodes
// of at most kSmall triangles are finished by one thread each with the
// sequential algorithm. Binary node ids are allocated in any order: the
// collapse lays the 4-wide nodes out depth-first from the tree's shape, and
// leaves are emitted left to right, so a leaf's first triangle is its start.
//
// Min/max reductions run on order-preserving integer keys, which order -0
// below +0; a box bound that is zero with both signs among its inputs can
// differ in the sign of zero from the sequential std::min, which slab tests
// do not distinguish.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "build.h"

namespace ana {

DeviceTris::~DeviceTris() {
    if (nodes) cudaFree(nodes);
    if (isect) cudaFree(isect);
    if (shade) cudaFree(shade);
}

namespace {

constexpr int kBk = 12;              // BVHBackend kSAHBuckets
constexpr uint32_t kSmall = 128;     // subtrees at most this large: one thread each
constexpr int kChunkThreads = 256;   // privatised passes: positions per block
constexpr int kPerThread = 16;
constexpr int kChunk = kChunkThreads * kPerThread;
constexpr int kMaxRuns = kChunk / int(kSmall + 1) + 2;  // open nodes one chunk can touch
constexpr int kBinWords = 3 * kBk * 7;                  // per node: axis x bucket x (count, lo3, hi3)

// ---- order-preserving float keys (exact atomic min / max) ------------------
__device__ __forceinline__ uint32_t fkey(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float funkey(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}
constexpr uint32_t kKeyPosInf = 0xFF800000u;  // fkey(+inf): identity of min
constexpr uint32_t kKeyNegInf = 0x007FFFFFu;  // fkey(-inf): identity of max

// std::min / std::max as the host code calls them (the first argument wins ties)
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }

struct Prims {  // build-order primitive records, structure of arrays
    float* lo[3];
    float* hi[3];
    float* c[3];
    uint32_t* idx;
};

struct BinNode {  // binary build node (prepare.cpp BuildNode)
    float lo[3], hi[3];
    int32_t left, right;
    uint32_t start, count;
};

struct Open {  // a node of the current level
    uint32_t bin, start, count;
};

struct SlotInfo {  // per open node, derived during the level
    float cmin[3], range[3];
    uint32_t cand;      // bins wanted (count > maxLeaf, parent area >= 1e-12)
    int32_t axis, split;
    uint32_t mid, swap; // swap: the partition moves elements (not the median fallback)
    int32_t lslot, rslot;  // next-level slots of the children (-1: small or leaf)
    uint32_t leaf;
};

// 2 (dx dy + dy dz + dz dx), BVHBackend.cpp:190-193
__device__ __forceinline__ float box_area(const float* lo, const float* hi) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return 2.f * (dx * dy + dy * dz + dz * dx);
}

__device__ __forceinline__ int bucket_of(float c, float cmin, float range) {
    int b = static_cast<int>(float(kBk) * ((c - cmin) / range));
    return b < 0 ? 0 : (b > kBk - 1 ? kBk - 1 : b);
}

__device__ __forceinline__ float3 ld3(const float* p) { return make_float3(p[0], p[1], p[2]); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// safeNormalize (Types.h:80-89)
__device__ __forceinline__ float3 safe_norm(float3 v) {
    const float len = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    if (!(len > 1e-8f)) return make_float3(0.f, 0.f, 1.f);
    const float inv = 1.f / len;
    return make_float3(v.x * inv, v.y * inv, v.z * inv);
}
__device__ __forceinline__ bool finite3(float3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

// ---- triangle setup (BVHBackend.cpp:17-111) ---------------------------------
struct SetupArgs {
    const float* pos;
    const float* nrm;
    const uint32_t* ind;
    const uint32_t* vo;
    const uint32_t* to;
    const uint8_t* hasN;
    uint32_t num_meshes, num_tris;
    float4* isect_mesh;  // 3 per triangle, mesh order
    float4* shade;       // 4 per triangle, mesh order
    Prims P;
    uint32_t* err;
};

__global__ void __launch_bounds__(256) k_setup(const SetupArgs a) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.num_tris) return;
    uint32_t lo = 0, hi = a.num_meshes;  // last mesh whose first triangle is <= t
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.to[mid] <= t) lo = mid;
        else hi = mid;
    }
    const uint32_t m = lo;
    const uint32_t v0i = a.vo[m], nv = a.vo[m + 1] - v0i, t0 = a.to[m];
    const uint32_t ia = a.ind[3 * size_t(t)], ib = a.ind[3 * size_t(t) + 1], ic = a.ind[3 * size_t(t) + 2];
    if (ia >= nv || ib >= nv || ic >= nv) {
        atomicOr(a.err, 1u);
        return;
    }
    const float3 pa = ld3(a.pos + 3 * size_t(v0i + ia)), pb = ld3(a.pos + 3 * size_t(v0i + ib)),
                 pc = ld3(a.pos + 3 * size_t(v0i + ic));
    if (!finite3(pa) || !finite3(pb) || !finite3(pc)) {
        atomicOr(a.err, 2u);
        return;
    }
    const float3 v0 = pa, e1 = sub3(pb, v0), e2 = sub3(pc, v0);
    const float3 n = safe_norm(cross3(e1, e2));
    const bool hasN = a.hasN && a.hasN[m] && a.nrm;
    const float3 s0 = hasN ? safe_norm(ld3(a.nrm + 3 * size_t(v0i + ia))) : n;
    const float3 s1 = hasN ? safe_norm(ld3(a.nrm + 3 * size_t(v0i + ib))) : n;
    const float3 s2 = hasN ? safe_norm(ld3(a.nrm + 3 * size_t(v0i + ic))) : n;
    a.isect_mesh[3 * size_t(t)] = make_float4(v0.x, v0.y, v0.z, __uint_as_float(t));
    a.isect_mesh[3 * size_t(t) + 1] = make_float4(e1.x, e1.y, e1.z, 0.f);
    a.isect_mesh[3 * size_t(t) + 2] = make_float4(e2.x, e2.y, e2.z, 0.f);
    a.shade[4 * size_t(t)] = make_float4(n.x, n.y, n.z, __uint_as_float(m));
    a.shade[4 * size_t(t) + 1] = make_float4(s0.x, s0.y, s0.z, __uint_as_float(t - t0));
    a.shade[4 * size_t(t) + 2] = make_float4(s1.x, s1.y, s1.z, 0.f);
    a.shade[4 * size_t(t) + 3] = make_float4(s2.x, s2.y, s2.z, 0.f);
    // bounds of v0, v0 + e1, v0 + e2 with flat axes padded by 1e-7
    const float3 w1 = add3(v0, e1), w2 = add3(v0, e2);
    const float p0[3] = {v0.x, v0.y, v0.z}, p1[3] = {w1.x, w1.y, w1.z}, p2[3] = {w2.x, w2.y, w2.z};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        float l = smin(smin(smin(INFINITY, p0[ax]), p1[ax]), p2[ax]);
        float h = smax(smax(smax(-INFINITY, p0[ax]), p1[ax]), p2[ax]);
        if (h - l < 1e-7f) {
            l -= 1e-7f;
            h += 1e-7f;
        }
        a.P.lo[ax][t] = l;
        a.P.hi[ax][t] = h;
        a.P.c[ax][t] = (l + h) * 0.5f;
    }
    a.P.idx[t] = t;
}

// ---- level-synchronous SAH build over nodes of more than kSmall ------------
struct LevelArgs {
    Prims P;
    uint32_t T;
    int32_t* slot;         // per position: open slot of this level, or -1
    const Open* open;      // this level's nodes
    Open* next;            // next level's nodes
    uint32_t* nextCount;
    Open* small;           // subtrees left to one thread each
    uint32_t* smallCount;
    uint32_t nOpen;
    SlotInfo* info;
    uint32_t* bkeys;       // 12 per slot: lo3 hi3 clo3 chi3 keys
    uint32_t* bins;        // kBinWords per slot
    BinNode* pool;
    uint32_t* poolCount;
    uint32_t maxLeaf;
    uint32_t* flag;        // per position
    uint32_t* excl;        // exclusive scan of flag, T + 1
    uint32_t* A;           // per node: positions that fail the predicate, left part
    uint32_t* B;           // per node: positions that pass it, right part, from the right
    uint32_t openCap, smallCap, poolCap;
    uint32_t* err;         // bit 3: an internal bound was exceeded (nothing written past it)
};

__global__ void k_level_init(const LevelArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.nOpen * 12u) {
        const uint32_t k = i % 12u;
        a.bkeys[i] = (k < 3u || (k >= 6u && k < 9u)) ? kKeyPosInf : kKeyNegInf;
    }
    if (i < a.nOpen * uint32_t(kBinWords)) {
        const uint32_t w = i % 7u;
        a.bins[i] = w == 0 ? 0u : (w < 4u ? kKeyPosInf : kKeyNegInf);
    }
}

// Runs of one block's positions: run index of each position (or -1) and the
// slot of every run. Positions are [base, base + kChunk) in steps of the block.
struct Runs {
    uint32_t words[kChunk / 32];
    uint32_t prefix[kChunk / 32];
    int32_t runSlot[kMaxRuns];
    uint32_t nRuns;
};

__device__ void find_runs(const LevelArgs& a, uint32_t base, Runs& R, int32_t (&slotOf)[kPerThread],
                          int32_t (&runOf)[kPerThread]) {
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
#pragma unroll
    for (int j = 0; j < kPerThread; ++j) {
        const uint32_t pos = base + uint32_t(j) * kChunkThreads + tid;
        const int32_t s = pos < a.T ? a.slot[pos] : -1;
        const int32_t prev = (pos < a.T && pos > base) ? a.slot[pos - 1] : -2;
        slotOf[j] = s;
        const bool head = s >= 0 && s != prev;
        const uint32_t bits = __ballot_sync(0xFFFFFFFFu, head);
        if (lane == 0) R.words[j * (kChunkThreads / 32) + warp] = bits;
    }
    __syncthreads();
    if (warp == 0) {  // exclusive prefix of the words' popcounts
        constexpr int kW = kChunk / 32, kPer = kW / 32;
        uint32_t c[kPer], sum = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            c[k] = __popc(R.words[lane * kPer + k]);
            sum += c[k];
        }
        uint32_t inc = sum;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, inc, off);
            if (lane >= uint32_t(off)) inc += v;
        }
        uint32_t run = inc - sum;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            R.prefix[lane * kPer + k] = run;
            run += c[k];
        }
        if (lane == 31) R.nRuns = inc < uint32_t(kMaxRuns) ? inc : uint32_t(kMaxRuns);
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kPerThread; ++j) {
        runOf[j] = -1;
        if (slotOf[j] < 0) continue;
        const uint32_t w = uint32_t(j) * (kChunkThreads / 32) + warp;
        const uint32_t below = lane == 31 ? 0xFFFFFFFFu : ((2u << lane) - 1u);
        const int32_t r = int32_t(R.prefix[w] + __popc(R.words[w] & below)) - 1;
        if (r >= kMaxRuns) {
            atomicOr(a.err, 8u);
            continue;
        }
        runOf[j] = r;
        if ((R.words[w] >> lane) & 1u) R.runSlot[r] = slotOf[j];
    }
    __syncthreads();
}

// bounds and centroid bounds of every open node
__global__ void __launch_bounds__(kChunkThreads) k_bounds(const LevelArgs a) {
    __shared__ Runs R;
    __shared__ uint32_t acc[kMaxRuns * 12];
    const uint32_t base = blockIdx.x * uint32_t(kChunk);
    int32_t slotOf[kPerThread], runOf[kPerThread];
    find_runs(a, base, R, slotOf, runOf);
    for (uint32_t i = threadIdx.x; i < R.nRuns * 12u; i += blockDim.x) {
        const uint32_t k = i % 12u;
        acc[i] = (k < 3u || (k >= 6u && k < 9u)) ? kKeyPosInf : kKeyNegInf;
    }
    __syncthreads();
    int32_t cur = -1;
    uint32_t v[12];
    auto flush = [&]() {
        if (cur < 0) return;
        for (int k = 0; k < 12; ++k) {
            if (k < 3 || (k >= 6 && k < 9)) atomicMin(&acc[cur * 12 + k], v[k]);
            else atomicMax(&acc[cur * 12 + k], v[k]);
        }
    };
    for (int j = 0; j < kPerThread; ++j) {
        if (runOf[j] < 0) continue;
        const uint32_t pos = base + uint32_t(j) * kChunkThreads + threadIdx.x;
        if (runOf[j] != cur) {
            flush();
            cur = runOf[j];
            for (int k = 0; k < 12; ++k) v[k] = (k < 3 || (k >= 6 && k < 9)) ? kKeyPosInf : kKeyNegInf;
        }
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            v[ax] = min(v[ax], fkey(a.P.lo[ax][pos]));
            v[3 + ax] = max(v[3 + ax], fkey(a.P.hi[ax][pos]));
            const uint32_t ck = fkey(a.P.c[ax][pos]);
            v[6 + ax] = min(v[6 + ax], ck);
            v[9 + ax] = max(v[9 + ax], ck);
        }
    }
    flush();
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < R.nRuns * 12u; i += blockDim.x) {
        const uint32_t r = i / 12u, k = i % 12u;
        uint32_t* g = a.bkeys + size_t(R.runSlot[r]) * 12u + k;
        if (k < 3u || (k >= 6u && k < 9u)) atomicMin(g, acc[i]);
        else atomicMax(g, acc[i]);
    }
}

// per open node: box into the pool, the bucketing frame and whether to bin
__global__ void k_prep(const LevelArgs a) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nOpen) return;
    const uint32_t* K = a.bkeys + size_t(s) * 12u;
    BinNode& n = a.pool[a.open[s].bin];
    float lo[3], hi[3];
    SlotInfo& I = a.info[s];
    for (int ax = 0; ax < 3; ++ax) {
        lo[ax] = funkey(K[ax]);
        hi[ax] = funkey(K[3 + ax]);
        n.lo[ax] = lo[ax];
        n.hi[ax] = hi[ax];
        const float cl = funkey(K[6 + ax]), ch = funkey(K[9 + ax]);
        I.cmin[ax] = cl;
        I.range[ax] = ch - cl;
    }
    const float parentArea = box_area(lo, hi);
    I.cand = (a.open[s].count > a.maxLeaf && !(parentArea < 1e-12f)) ? 1u : 0u;
}

// SAH buckets of the candidate nodes (axes whose centroid range is >= 1e-7)
__global__ void __launch_bounds__(kChunkThreads) k_bin(const LevelArgs a) {
    __shared__ Runs R;
    __shared__ uint32_t bins[kMaxRuns * kBinWords];
    const uint32_t base = blockIdx.x * uint32_t(kChunk);
    int32_t slotOf[kPerThread], runOf[kPerThread];
    find_runs(a, base, R, slotOf, runOf);
    for (uint32_t i = threadIdx.x; i < R.nRuns * uint32_t(kBinWords); i += blockDim.x) {
        const uint32_t w = i % 7u;
        bins[i] = w == 0 ? 0u : (w < 4u ? kKeyPosInf : kKeyNegInf);
    }
    __syncthreads();
    for (int j = 0; j < kPerThread; ++j) {
        if (runOf[j] < 0) continue;
        const SlotInfo& I = a.info[slotOf[j]];
        if (!I.cand) continue;
        const uint32_t pos = base + uint32_t(j) * kChunkThreads + threadIdx.x;
        const uint32_t lk[3] = {fkey(a.P.lo[0][pos]), fkey(a.P.lo[1][pos]), fkey(a.P.lo[2][pos])};
        const uint32_t hk[3] = {fkey(a.P.hi[0][pos]), fkey(a.P.hi[1][pos]), fkey(a.P.hi[2][pos])};
        for (int ax = 0; ax < 3; ++ax) {
            if (I.range[ax] < 1e-7f) continue;
            const int b = bucket_of(a.P.c[ax][pos], I.cmin[ax], I.range[ax]);
            uint32_t* w = bins + runOf[j] * kBinWords + (ax * kBk + b) * 7;
            atomicAdd(w, 1u);
            for (int k = 0; k < 3; ++k) {
                atomicMin(w + 1 + k, lk[k]);
                atomicMax(w + 4 + k, hk[k]);
            }
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < R.nRuns * uint32_t(kBinWords); i += blockDim.x) {
        const uint32_t r = i / uint32_t(kBinWords), k = i % uint32_t(kBinWords), w = k % 7u;
        const uint32_t v = bins[i];
        uint32_t* g = a.bins + size_t(R.runSlot[r]) * kBinWords + k;
        if (w == 0) {
            if (v) atomicAdd(g, v);
        } else if (w < 4u) {
            if (v != kKeyPosInf) atomicMin(g, v);
        } else if (v != kKeyNegInf) {
            atomicMax(g, v);
        }
    }
}

struct HBox {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    __device__ void expand(const HBox& b) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = smin(lo[k], b.lo[k]);
            hi[k] = smax(hi[k], b.hi[k]);
        }
    }
    __device__ float area() const { return box_area(lo, hi); }
};

// sahSplit's sweep over 12 buckets of one axis (BVHBackend.cpp:158-228)
__device__ void sweep_axis(const HBox* bb, const uint32_t* bc, int axis, float parentArea, float& bestCost,
                           int& bestSplit, int& outAxis) {
    HBox lb[kBk - 1];
    uint32_t lcnt[kBk - 1];
    HBox acc;
    uint32_t ac = 0;
    for (int i = 0; i < kBk - 1; ++i) {
        acc.expand(bb[i]);
        ac += bc[i];
        lb[i] = acc;
        lcnt[i] = ac;
    }
    HBox rb;
    uint32_t rc = 0;
    for (int i = kBk - 2; i >= 0; --i) {
        rb.expand(bb[i + 1]);
        rc += bc[i + 1];
        const float cost = 1.f + 1.f * (lb[i].area() * float(lcnt[i]) + rb.area() * float(rc)) / parentArea;
        if (cost < bestCost) {
            bestCost = cost;
            bestSplit = i;
            outAxis = axis;
        }
    }
}

__device__ __forceinline__ void push_child(const LevelArgs& a, uint32_t bin, uint32_t start, uint32_t count,
                                           int32_t& slot) {
    slot = -1;
    if (count > kSmall) {
        const uint32_t s = atomicAdd(a.nextCount, 1u);
        if (s >= a.openCap) {
            atomicOr(a.err, 8u);
            return;
        }
        a.next[s] = Open{bin, start, count};
        slot = int32_t(s);
    } else {
        const uint32_t s = atomicAdd(a.smallCount, 1u);
        if (s >= a.smallCap) {
            atomicOr(a.err, 8u);
            return;
        }
        a.small[s] = Open{bin, start, count};
    }
}

// per open node: the split (or a leaf), the children and their slots
__global__ void k_choose(const LevelArgs a) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nOpen) return;
    const Open o = a.open[s];
    SlotInfo& I = a.info[s];
    BinNode& n = a.pool[o.bin];
    int axis = -1, split = -1;
    if (I.cand) {
        const float parentArea = box_area(n.lo, n.hi);
        float bestCost = INFINITY;
        for (int ax = 0; ax < 3; ++ax) {
            if (I.range[ax] < 1e-7f) continue;
            HBox bb[kBk];
            uint32_t bc[kBk];
            const uint32_t* W = a.bins + size_t(s) * kBinWords + ax * kBk * 7;
            for (int b = 0; b < kBk; ++b) {
                bc[b] = W[b * 7];
                for (int k = 0; k < 3; ++k) {
                    bb[b].lo[k] = funkey(W[b * 7 + 1 + k]);
                    bb[b].hi[k] = funkey(W[b * 7 + 4 + k]);
                }
            }
            sweep_axis(bb, bc, ax, parentArea, bestCost, split, axis);
        }
        if (bestCost >= 1.f * float(o.count)) axis = -1;
    }
    I.axis = axis;
    I.split = split;
    if (axis < 0 || split < 0) {
        n.left = n.right = -1;
        n.start = o.start;
        n.count = o.count;
        I.leaf = 1;
        I.swap = 0;
        I.lslot = I.rslot = -1;
        return;
    }
    I.leaf = 0;
    uint32_t L = 0;
    const uint32_t* W = a.bins + size_t(s) * kBinWords + axis * kBk * 7;
    for (int b = 0; b <= split; ++b) L += W[b * 7];
    const bool fallback = L == 0 || L == o.count;
    const uint32_t mid = fallback ? o.start + o.count / 2 : o.start + L;
    I.mid = mid;
    I.swap = fallback ? 0u : 1u;
    const uint32_t kids = atomicAdd(a.poolCount, 2u);
    if (kids + 2u > a.poolCap) {
        atomicOr(a.err, 8u);
        n.left = n.right = -1;
        n.start = o.start;
        n.count = o.count;
        I.leaf = 1;
        I.swap = 0;
        I.lslot = I.rslot = -1;
        return;
    }
    n.left = int32_t(kids);
    n.right = int32_t(kids + 1);
    n.start = 0;
    n.count = 0;
    push_child(a, kids, o.start, mid - o.start, I.lslot);
    push_child(a, kids + 1, mid, o.start + o.count - mid, I.rslot);
}

__device__ __forceinline__ bool split_pos(const LevelArgs& a, uint32_t pos, int32_t& s, const SlotInfo*& I) {
    s = pos < a.T ? a.slot[pos] : -1;
    if (s < 0) return false;
    I = &a.info[s];
    return !I->leaf;
}

__device__ __forceinline__ bool pred_at(const LevelArgs& a, const SlotInfo& I, uint32_t pos) {
    return bucket_of(a.P.c[I.axis][pos], I.cmin[I.axis], I.range[I.axis]) <= I.split;
}

__global__ void k_flags(const LevelArgs a) {
    for (uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x; pos < a.T; pos += gridDim.x * blockDim.x) {
        int32_t s;
        const SlotInfo* I;
        uint32_t f = 0;
        if (split_pos(a, pos, s, I) && I->swap) f = pred_at(a, *I, pos) ? 1u : 0u;
        a.flag[pos] = f;
    }
}

// std::partition's exchange pairs: ranks from the exclusive scan of the predicate
__global__ void k_lists(const LevelArgs a) {
    for (uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x; pos < a.T; pos += gridDim.x * blockDim.x) {
        int32_t s;
        const SlotInfo* I;
        if (!split_pos(a, pos, s, I) || !I->swap) continue;
        const Open o = a.open[s];
        const uint32_t e = o.start + o.count;
        const bool p = a.flag[pos] != 0;
        if (pos < I->mid && !p) {
            const uint32_t k = (pos - o.start) - (a.excl[pos] - a.excl[o.start]);
            a.A[o.start + k] = pos;
        } else if (pos >= I->mid && p) {
            const uint32_t k = a.excl[e] - a.excl[pos + 1];
            a.B[o.start + k] = pos;
        }
    }
}

__global__ void k_swap(const LevelArgs a) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < a.T; j += gridDim.x * blockDim.x) {
        int32_t s;
        const SlotInfo* I;
        if (!split_pos(a, j, s, I) || !I->swap) continue;
        const Open o = a.open[s];
        const uint32_t m = (I->mid - o.start) - (a.excl[I->mid] - a.excl[o.start]);
        if (j - o.start >= m) continue;
        const uint32_t x = a.A[j], y = a.B[j];
        if (x >= a.T || y >= a.T) {
            atomicOr(a.err, 8u);
            continue;
        }
        for (int ax = 0; ax < 3; ++ax) {
            float t = a.P.lo[ax][x];
            a.P.lo[ax][x] = a.P.lo[ax][y];
            a.P.lo[ax][y] = t;
            t = a.P.hi[ax][x];
            a.P.hi[ax][x] = a.P.hi[ax][y];
            a.P.hi[ax][y] = t;
            t = a.P.c[ax][x];
            a.P.c[ax][x] = a.P.c[ax][y];
            a.P.c[ax][y] = t;
        }
        const uint32_t t = a.P.idx[x];
        a.P.idx[x] = a.P.idx[y];
        a.P.idx[y] = t;
    }
}

__global__ void k_update(const LevelArgs a) {
    for (uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x; pos < a.T; pos += gridDim.x * blockDim.x) {
        const int32_t s = a.slot[pos];
        if (s < 0) continue;
        const SlotInfo& I = a.info[s];
        a.slot[pos] = I.leaf ? -1 : (pos < I.mid ? I.lslot : I.rslot);
    }
}

// ---- exclusive scan (3 passes) ---------------------------------------------
constexpr int kScanThreads = 1024, kScanPer = 4, kScanTile = kScanThreads * kScanPer;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t inc = v;
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, off);
        if (lane >= uint32_t(off)) inc += t;
    }
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < (blockDim.x >> 5) ? sh[lane] : 0u;
        uint32_t wi = w;
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, wi, off);
            if (lane >= uint32_t(off)) wi += t;
        }
        sh[lane] = wi - w;
        if (lane == 31) sh[32] = wi;
    }
    __syncthreads();
    total = sh[32];
    const uint32_t r = sh[warp] + inc - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const uint32_t* in, uint32_t n, uint32_t* tileSum) {
    __shared__ uint32_t sh[33];
    const size_t b = size_t(blockIdx.x) * kScanTile + threadIdx.x * kScanPer;
    uint32_t s = 0;
    for (int k = 0; k < kScanPer; ++k) s += (b + k < n) ? in[b + k] : 0u;
    uint32_t total;
    block_excl_scan(s, sh, total);
    if (threadIdx.x == 0) tileSum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(uint32_t* tileSum, uint32_t nTiles) {
    __shared__ uint32_t sh[33];
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nTiles; base += kScanThreads) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nTiles ? tileSum[i] : 0u;
        uint32_t total;
        const uint32_t e = block_excl_scan(v, sh, total);
        if (i < nTiles) tileSum[i] = carry + e;
        carry += total;
    }
    if (threadIdx.x == 0) tileSum[nTiles] = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const uint32_t* in, uint32_t n, const uint32_t* tileSum,
                                                            uint32_t* out) {
    __shared__ uint32_t sh[33];
    const size_t b = size_t(blockIdx.x) * kScanTile + threadIdx.x * kScanPer;
    uint32_t v[kScanPer], s = 0;
    for (int k = 0; k < kScanPer; ++k) {
        v[k] = (b + k < n) ? in[b + k] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t run = block_excl_scan(s, sh, total) + tileSum[blockIdx.x];
    for (int k = 0; k < kScanPer; ++k) {
        if (b + k < n) out[b + k] = run;
        run += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = tileSum[gridDim.x];
}

// ---- subtrees of at most kSmall triangles: one thread, sequential ----------
struct SmallArgs {
    Prims P;
    const Open* small;
    uint32_t nSmall;
    BinNode* pool;
    uint32_t* poolCount;
    uint32_t maxLeaf;
    uint32_t poolCap;
    uint32_t* err;
};

__device__ __forceinline__ void load_box(const Prims& P, uint32_t i, HBox& b) {
    for (int k = 0; k < 3; ++k) {
        b.lo[k] = P.lo[k][i];
        b.hi[k] = P.hi[k][i];
    }
}

__global__ void __launch_bounds__(128) k_small(const SmallArgs a) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= a.nSmall) return;
    struct Item {
        uint32_t start, count, bin;
    };
    Item stack[kSmall];
    int top = 0;
    stack[top++] = Item{a.small[w].start, a.small[w].count, a.small[w].bin};
    const Prims& P = a.P;
    while (top > 0) {
        const Item it = stack[--top];
        const uint32_t start = it.start, end = it.start + it.count, count = it.count;
        HBox bounds, cb;
        for (uint32_t i = start; i < end; ++i) {
            HBox b;
            load_box(P, i, b);
            bounds.expand(b);
            for (int k = 0; k < 3; ++k) {
                const float c = P.c[k][i];
                cb.lo[k] = smin(cb.lo[k], c);
                cb.hi[k] = smax(cb.hi[k], c);
            }
        }
        BinNode& n = a.pool[it.bin];
        for (int k = 0; k < 3; ++k) {
            n.lo[k] = bounds.lo[k];
            n.hi[k] = bounds.hi[k];
        }
        int axis = -1, split = -1;
        if (count > a.maxLeaf) {
            const float parentArea = bounds.area();  // sahSplit recomputes the same union
            if (!(parentArea < 1e-12f)) {
                float bestCost = INFINITY;
                for (int ax = 0; ax < 3; ++ax) {
                    const float range = cb.hi[ax] - cb.lo[ax];
                    if (range < 1e-7f) continue;
                    HBox bb[kBk];
                    uint32_t bc[kBk] = {};
                    for (uint32_t i = start; i < end; ++i) {
                        const int b = bucket_of(P.c[ax][i], cb.lo[ax], range);
                        bc[b]++;
                        HBox pb;
                        load_box(P, i, pb);
                        bb[b].expand(pb);
                    }
                    sweep_axis(bb, bc, ax, parentArea, bestCost, split, axis);
                }
                if (bestCost >= 1.f * float(count)) axis = -1;
            }
        }
        if (axis < 0 || split < 0) {
            n.left = n.right = -1;
            n.start = start;
            n.count = count;
            continue;
        }
        const float cmin = cb.lo[axis], range = cb.hi[axis] - cb.lo[axis];
        uint32_t mid = start;
        if (range > 0.f) {  // std::partition, bidirectional form (libstdc++)
            uint32_t f = start, l = end;
            auto pred = [&](uint32_t i) { return bucket_of(P.c[axis][i], cmin, range) <= split; };
            while (true) {
                while (f != l && pred(f)) ++f;
                if (f == l) break;
                --l;
                while (f != l && !pred(l)) --l;
                if (f == l) break;
                for (int k = 0; k < 3; ++k) {
                    float t = P.lo[k][f];
                    P.lo[k][f] = P.lo[k][l];
                    P.lo[k][l] = t;
                    t = P.hi[k][f];
                    P.hi[k][f] = P.hi[k][l];
                    P.hi[k][l] = t;
                    t = P.c[k][f];
                    P.c[k][f] = P.c[k][l];
                    P.c[k][l] = t;
                }
                const uint32_t t = P.idx[f];
                P.idx[f] = P.idx[l];
                P.idx[l] = t;
                ++f;
            }
            mid = f;
        }
        if (mid == start || mid == end) mid = start + count / 2;
        const uint32_t kids = atomicAdd(a.poolCount, 2u);
        if (kids + 2u > a.poolCap || top + 2 > int(kSmall)) {
            atomicOr(a.err, 8u);
            n.left = n.right = -1;
            n.start = start;
            n.count = count;
            continue;
        }
        n.left = int32_t(kids);
        n.right = int32_t(kids + 1);
        n.start = 0;
        n.count = 0;
        stack[top++] = Item{mid, end - mid, kids + 1};
        stack[top++] = Item{start, mid - start, kids};
    }
}

// ---- 4-wide collapse (prepare.cpp flatten_bvh4) ------------------------------
struct Rec4 {
    uint32_t bin;
    uint32_t kids[4];
    int32_t child[4];  // record of an interior kid, -1 for a leaf kid
    uint32_t nk, depth, size, idx;
};

struct CollapseArgs {
    const BinNode* pool;
    uint32_t poolCount;  // binary nodes built
    Rec4* rec;
    uint32_t* recCount;
    uint32_t recCap;
    uint32_t r0, r1;  // this level's records
    uint32_t* bound;  // worst root-to-leaf pushes
    uint32_t* err;
};

__device__ __forceinline__ bool interior(const BinNode& n) { return n.count == 0 && n.left >= 0; }
__device__ __forceinline__ float half_area(const BinNode& n) {
    const float dx = n.hi[0] - n.lo[0], dy = n.hi[1] - n.lo[1], dz = n.hi[2] - n.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

__global__ void k_collapse(const CollapseArgs a) {
    const uint32_t r = a.r0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.r1) return;
    Rec4& R = a.rec[r];
    const BinNode& b = a.pool[R.bin];
    auto bad = [&](int32_t i) { return i < 0 || uint32_t(i) >= a.poolCount; };
    if (bad(b.left) || bad(b.right)) {
        atomicOr(a.err, 4u);
        R.nk = 0;
        return;
    }
    uint32_t kids[4] = {uint32_t(b.left), uint32_t(b.right), 0, 0};
    int nk = 2;
    while (nk < 4) {
        int pick = -1;
        float best = -1.f;
        for (int k = 0; k < nk; ++k) {
            const BinNode& c = a.pool[kids[k]];
            if (interior(c) && (bad(c.left) || bad(c.right))) {
                atomicOr(a.err, 4u);
                R.nk = 0;
                return;
            }
            if (interior(c) && half_area(c) > best) {
                best = half_area(c);
                pick = k;
            }
        }
        if (pick < 0) break;
        const BinNode& c = a.pool[kids[pick]];
        for (int k = nk; k > pick + 1; --k) kids[k] = kids[k - 1];
        kids[pick] = uint32_t(c.left);
        kids[pick + 1] = uint32_t(c.right);
        ++nk;
    }
    const uint32_t d = R.depth + uint32_t(nk - 1);
    R.nk = uint32_t(nk);
    bool anyLeaf = false;
    for (int k = 0; k < 4; ++k) {
        R.kids[k] = kids[k];
        R.child[k] = -1;
        if (k >= nk) continue;
        if (interior(a.pool[kids[k]])) {
            const uint32_t c = atomicAdd(a.recCount, 1u);
            if (c >= a.recCap) {
                atomicOr(a.err, 4u);
                continue;
            }
            Rec4& C = a.rec[c];
            C.bin = kids[k];
            C.depth = d;
            R.child[k] = int32_t(c);
        } else {
            anyLeaf = true;
        }
    }
    if (anyLeaf) atomicMax(a.bound, d);
}

__global__ void k_sizes(Rec4* rec, uint32_t r0, uint32_t r1) {
    const uint32_t r = r0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= r1) return;
    uint32_t s = 1;
    for (int k = 0; k < 4; ++k)
        if (rec[r].child[k] >= 0) s += rec[rec[r].child[k]].size;
    rec[r].size = s;
}

__global__ void k_indices(Rec4* rec, uint32_t r0, uint32_t r1) {
    const uint32_t r = r0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= r1) return;
    uint32_t run = rec[r].idx + 1;
    for (int k = 0; k < 4; ++k) {
        const int32_t c = rec[r].child[k];
        if (c < 0) continue;
        rec[c].idx = run;
        run += rec[c].size;
    }
}

__device__ __forceinline__ void put_child(float (&v)[6][4], uint32_t (&ref)[4], int k, const float* lo,
                                          const float* hi, uint32_t r) {
    v[0][k] = lo[0];
    v[1][k] = hi[0];
    v[2][k] = lo[1];
    v[3][k] = hi[1];
    v[4][k] = lo[2];
    v[5][k] = hi[2];
    ref[k] = r;
}

__device__ __forceinline__ uint32_t leaf_ref(const BinNode& n) {
    return 0x80000000u | ((n.count - 1u) << 25) | n.start;
}

__device__ __forceinline__ void store_node(Bvh4Node* out, uint32_t idx, const float (&v)[6][4], const uint32_t (&ref)[4]) {
    Bvh4Node n;
    n.lox = make_float4(v[0][0], v[0][1], v[0][2], v[0][3]);
    n.hix = make_float4(v[1][0], v[1][1], v[1][2], v[1][3]);
    n.loy = make_float4(v[2][0], v[2][1], v[2][2], v[2][3]);
    n.hiy = make_float4(v[3][0], v[3][1], v[3][2], v[3][3]);
    n.loz = make_float4(v[4][0], v[4][1], v[4][2], v[4][3]);
    n.hiz = make_float4(v[5][0], v[5][1], v[5][2], v[5][3]);
    n.ref = make_uint4(ref[0], ref[1], ref[2], ref[3]);
    n.pad = make_uint4(0u, 0u, 0u, 0u);
    out[idx] = n;
}

__global__ void k_write_nodes(const BinNode* pool, const Rec4* rec, uint32_t nRec, Bvh4Node* out, uint32_t* err) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nRec) return;
    const Rec4& R = rec[r];
    if (R.idx >= nRec || R.nk > 4u) {
        atomicOr(err, 8u);
        return;
    }
    const float empty_lo[3] = {INFINITY, INFINITY, INFINITY}, empty_hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    float v[6][4];
    uint32_t ref[4];
    for (int k = 0; k < 4; ++k) {
        if (uint32_t(k) >= R.nk) {
            put_child(v, ref, k, empty_lo, empty_hi, kEmptyChild);
            continue;
        }
        const BinNode& c = pool[R.kids[k]];
        put_child(v, ref, k, c.lo, c.hi, R.child[k] >= 0 ? rec[R.child[k]].idx : leaf_ref(c));
    }
    store_node(out, R.idx, v, ref);
}

// a root that is a leaf: one node holding it as child 0
__global__ void k_root_leaf(const BinNode* pool, Bvh4Node* out) {
    const float empty_lo[3] = {INFINITY, INFINITY, INFINITY}, empty_hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    float v[6][4];
    uint32_t ref[4];
    for (int k = 1; k < 4; ++k) put_child(v, ref, k, empty_lo, empty_hi, kEmptyChild);
    put_child(v, ref, 0, pool[0].lo, pool[0].hi, leaf_ref(pool[0]));
    store_node(out, 0, v, ref);
}

__global__ void k_gather_isect(const float4* mesh, const uint32_t* idx, uint32_t T, float4* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T * 3u; i += gridDim.x * blockDim.x) {
        const uint32_t t = i / 3u, k = i % 3u;
        out[i] = mesh[3 * size_t(idx[t]) + k];
    }
}

__global__ void k_root_open(Open* open, uint32_t T, int32_t* slot) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) slot[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) open[0] = Open{0u, 0u, T};
}

// ---- host orchestration -------------------------------------------------------
struct DevBuf {
    std::vector<void*> ptrs;
    ~DevBuf() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t alloc(T*& p, size_t n) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(q);
        p = static_cast<T*>(q);
        return e;
    }
};

inline int grid_for(size_t n, int block, int cap = 148 * 16) {
    return int(std::max<size_t>(1, std::min<size_t>((n + block - 1) / block, size_t(cap))));
}

}  // namespace

#define BK(x)                                                                          \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            err = std::string("device BVH build: ") + cudaGetErrorString(e_);          \
            return ANA_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

int build_tris_on_device(const ana_scene_desc& d, uint32_t maxLeaf, cudaStream_t st, DeviceTris& out,
                         std::string& err) {
    const uint32_t M = d.num_meshes;
    const uint32_t T = M ? d.mesh_tri_offset[M] : 0;
    const uint32_t V = M ? d.mesh_vert_offset[M] : 0;
    if (T == 0) {
        err = "device BVH build: no triangles";
        return ANA_ERR_INVALID_ARG;
    }
    using Clock = std::chrono::steady_clock;
    auto t0 = Clock::now();
    auto lap = [&](int k) {
        const auto t = Clock::now();
        out.ms[k] = std::chrono::duration<float, std::milli>(t - t0).count();
        t0 = t;
    };
    DevBuf tmp;
    float *pos = nullptr, *nrm = nullptr;
    uint32_t *ind = nullptr, *vo = nullptr, *to = nullptr, *derr = nullptr;
    uint8_t* hasN = nullptr;
    BK(tmp.alloc(pos, size_t(V) * 3));
    BK(tmp.alloc(ind, size_t(T) * 3));
    BK(tmp.alloc(vo, M + 1));
    BK(tmp.alloc(to, M + 1));
    BK(tmp.alloc(derr, 4));
    BK(cudaMemcpyAsync(pos, d.positions, size_t(V) * 12, cudaMemcpyHostToDevice, st));
    BK(cudaMemcpyAsync(ind, d.indices, size_t(T) * 12, cudaMemcpyHostToDevice, st));
    BK(cudaMemcpyAsync(vo, d.mesh_vert_offset, (M + 1) * 4, cudaMemcpyHostToDevice, st));
    BK(cudaMemcpyAsync(to, d.mesh_tri_offset, (M + 1) * 4, cudaMemcpyHostToDevice, st));
    BK(cudaMemsetAsync(derr, 0, 16, st));
    if (d.normals && d.mesh_has_normals) {
        BK(tmp.alloc(nrm, size_t(V) * 3));
        BK(tmp.alloc(hasN, M));
        BK(cudaMemcpyAsync(nrm, d.normals, size_t(V) * 12, cudaMemcpyHostToDevice, st));
        BK(cudaMemcpyAsync(hasN, d.mesh_has_normals, M, cudaMemcpyHostToDevice, st));
    }
    // outputs
    BK(cudaMalloc(&out.shade, size_t(T) * 64));
    BK(cudaMalloc(&out.isect, size_t(T) * 48));
    out.num_tris = T;
    // primitive records and build state
    Prims P;
    float4* isectMesh = nullptr;
    BK(tmp.alloc(isectMesh, size_t(T) * 3));
    for (int ax = 0; ax < 3; ++ax) {
        BK(tmp.alloc(P.lo[ax], T));
        BK(tmp.alloc(P.hi[ax], T));
        BK(tmp.alloc(P.c[ax], T));
    }
    BK(tmp.alloc(P.idx, T));
    SetupArgs sa{pos, nrm, ind, vo, to, hasN, M, T, isectMesh, out.shade, P, derr};
    k_setup<<<grid_for(T, 256, 1 << 30), 256, 0, st>>>(sa);
    BK(cudaGetLastError());
    uint32_t herr = 0;
    BK(cudaMemcpyAsync(&herr, derr, 4, cudaMemcpyDeviceToHost, st));
    BK(cudaStreamSynchronize(st));
    if (herr) {
        err = (herr & 1u) ? "triangle index out of range" : "non-finite vertex";
        return ANA_ERR_INVALID_ARG;
    }
    lap(0);

    // binary build
    const uint32_t maxOpen = T / (kSmall + 1) + 1;
    const uint32_t maxSmall = T;  // one per small subtree at most
    BinNode* pool = nullptr;
    uint32_t *counters = nullptr, *flag = nullptr, *excl = nullptr, *A = nullptr, *B = nullptr, *bkeys = nullptr,
             *bins = nullptr, *tileSum = nullptr;
    int32_t* slot = nullptr;
    Open *openA = nullptr, *openB = nullptr, *small = nullptr;
    SlotInfo* info = nullptr;
    BK(tmp.alloc(pool, 2 * size_t(T)));
    BK(tmp.alloc(counters, 8));  // 0 pool, 1 next open, 2 small, 3 records, 4 bound
    BK(tmp.alloc(slot, T));
    BK(tmp.alloc(flag, T));
    BK(tmp.alloc(excl, size_t(T) + 1));
    BK(tmp.alloc(A, T));
    BK(tmp.alloc(B, T));
    BK(tmp.alloc(openA, maxOpen));
    BK(tmp.alloc(openB, maxOpen));
    BK(tmp.alloc(small, maxSmall));
    BK(tmp.alloc(info, maxOpen));
    BK(tmp.alloc(bkeys, size_t(maxOpen) * 12));
    BK(tmp.alloc(bins, size_t(maxOpen) * kBinWords));
    const uint32_t nTiles = (T + kScanTile - 1) / kScanTile;
    BK(tmp.alloc(tileSum, size_t(nTiles) + 1));
    BK(cudaMemsetAsync(counters, 0, 32, st));
    const uint32_t one = 1;
    BK(cudaMemcpyAsync(counters, &one, 4, cudaMemcpyHostToDevice, st));  // the root is node 0

    uint32_t hc[8] = {};
    if (T > kSmall) {
        k_root_open<<<grid_for(T, 256), 256, 0, st>>>(openA, T, slot);
        uint32_t nOpen = 1;
        Open *cur = openA, *nxt = openB;
        const int chunkBlocks = int((T + kChunk - 1) / kChunk);
        for (int level = 0; nOpen > 0; ++level) {
            if (level > 4096) {
                err = "device BVH build: no progress";
                return ANA_ERR_CUDA;
            }
            LevelArgs la{P, T, slot, cur, nxt, counters + 1, small, counters + 2, nOpen, info, bkeys, bins,
                         pool, counters, maxLeaf, flag, excl, A, B, maxOpen, maxSmall, 2 * T, derr};
            BK(cudaMemsetAsync(counters + 1, 0, 4, st));
            k_level_init<<<grid_for(size_t(nOpen) * kBinWords, 256, 1 << 30), 256, 0, st>>>(la);
            k_bounds<<<chunkBlocks, kChunkThreads, 0, st>>>(la);
            k_prep<<<grid_for(nOpen, 128, 1 << 30), 128, 0, st>>>(la);
            k_bin<<<chunkBlocks, kChunkThreads, 0, st>>>(la);
            k_choose<<<grid_for(nOpen, 128, 1 << 30), 128, 0, st>>>(la);
            k_flags<<<grid_for(T, 256), 256, 0, st>>>(la);
            k_scan_tiles<<<nTiles, kScanThreads, 0, st>>>(flag, T, tileSum);
            k_scan_sums<<<1, kScanThreads, 0, st>>>(tileSum, nTiles);
            k_scan_apply<<<nTiles, kScanThreads, 0, st>>>(flag, T, tileSum, excl);
            k_lists<<<grid_for(T, 256), 256, 0, st>>>(la);
            k_swap<<<grid_for(T, 256), 256, 0, st>>>(la);
            k_update<<<grid_for(T, 256), 256, 0, st>>>(la);
            BK(cudaGetLastError());
            BK(cudaMemcpyAsync(hc, counters, 32, cudaMemcpyDeviceToHost, st));
            BK(cudaMemcpyAsync(&herr, derr, 4, cudaMemcpyDeviceToHost, st));
            BK(cudaStreamSynchronize(st));
            nOpen = hc[1];
            if (herr) {
                err = "device BVH build: an internal bound was exceeded";
                return ANA_ERR_CUDA;
            }
            if (nOpen > maxOpen) {
                err = "device BVH build: open-node table overflow";
                return ANA_ERR_CUDA;
            }
            std::swap(cur, nxt);
            out.levels = uint32_t(level + 1);
        }
    } else {
        const Open root{0u, 0u, T};
        BK(cudaMemcpyAsync(small, &root, sizeof(root), cudaMemcpyHostToDevice, st));
        const uint32_t ns = 1;
        BK(cudaMemcpyAsync(counters + 2, &ns, 4, cudaMemcpyHostToDevice, st));
    }
    BK(cudaMemcpyAsync(hc, counters, 32, cudaMemcpyDeviceToHost, st));
    BK(cudaStreamSynchronize(st));
    lap(1);
    const uint32_t nSmall = hc[2];
    if (nSmall) {
        SmallArgs sm{P, small, nSmall, pool, counters, maxLeaf, 2 * T, derr};
        k_small<<<grid_for(nSmall, 128, 1 << 30), 128, 0, st>>>(sm);
        BK(cudaGetLastError());
    }
    // leaf order of the intersection records
    k_gather_isect<<<grid_for(size_t(T) * 3, 256), 256, 0, st>>>(isectMesh, P.idx, T, out.isect);

    // 4-wide collapse
    BinNode root;
    BK(cudaMemcpyAsync(&root, pool, sizeof(root), cudaMemcpyDeviceToHost, st));
    BK(cudaMemcpyAsync(hc, counters, 32, cudaMemcpyDeviceToHost, st));
    BK(cudaMemcpyAsync(&herr, derr, 4, cudaMemcpyDeviceToHost, st));
    BK(cudaStreamSynchronize(st));
    if (herr) {
        err = "device BVH build: an internal bound was exceeded";
        return ANA_ERR_CUDA;
    }
    lap(2);
    if (hc[0] > 2 * T) {
        err = "device BVH build: node pool overflow";
        return ANA_ERR_CUDA;
    }
    if (!(root.count == 0 && root.left >= 0)) {
        BK(cudaMalloc(&out.nodes, sizeof(Bvh4Node)));
        out.num_nodes = 1;
        k_root_leaf<<<1, 1, 0, st>>>(pool, out.nodes);
        BK(cudaGetLastError());
        BK(cudaStreamSynchronize(st));
        return ANA_OK;
    }
    Rec4* rec = nullptr;
    BK(tmp.alloc(rec, size_t(T)));  // one per interior binary node at most
    Rec4 r0{};
    r0.bin = 0;
    r0.depth = 0;
    r0.idx = 0;
    BK(cudaMemcpyAsync(rec, &r0, sizeof(r0), cudaMemcpyHostToDevice, st));
    const uint32_t nr = 1, zero = 0;
    BK(cudaMemcpyAsync(counters + 3, &nr, 4, cudaMemcpyHostToDevice, st));
    BK(cudaMemcpyAsync(counters + 4, &zero, 4, cudaMemcpyHostToDevice, st));
    std::vector<uint32_t> levels{0u, 1u};  // record ranges per 4-wide level
    while (levels.back() > levels[levels.size() - 2]) {
        const uint32_t a0 = levels[levels.size() - 2], a1 = levels.back();
        CollapseArgs ca{pool, hc[0], rec, counters + 3, T, a0, a1, counters + 4, derr};
        k_collapse<<<grid_for(a1 - a0, 128, 1 << 30), 128, 0, st>>>(ca);
        BK(cudaGetLastError());
        uint32_t n = 0;
        BK(cudaMemcpyAsync(&n, counters + 3, 4, cudaMemcpyDeviceToHost, st));
        BK(cudaStreamSynchronize(st));
        if (n > T) {
            err = "device BVH build: 4-wide record overflow";
            return ANA_ERR_CUDA;
        }
        levels.push_back(n);
    }
    BK(cudaMemcpyAsync(&herr, derr, 4, cudaMemcpyDeviceToHost, st));
    BK(cudaStreamSynchronize(st));
    if (herr) {
        err = "device BVH build: inconsistent binary tree";
        return ANA_ERR_CUDA;
    }
    const uint32_t nRec = levels.back();
    for (size_t l = levels.size() - 1; l-- > 0;) {
        const uint32_t a0 = levels[l], a1 = levels[l + 1];
        if (a1 > a0) k_sizes<<<grid_for(a1 - a0, 128, 1 << 30), 128, 0, st>>>(rec, a0, a1);
    }
    for (size_t l = 0; l + 1 < levels.size(); ++l) {
        const uint32_t a0 = levels[l], a1 = levels[l + 1];
        if (a1 > a0) k_indices<<<grid_for(a1 - a0, 128, 1 << 30), 128, 0, st>>>(rec, a0, a1);
    }
    BK(cudaMalloc(&out.nodes, size_t(nRec) * sizeof(Bvh4Node)));
    out.num_nodes = nRec;
    k_write_nodes<<<grid_for(nRec, 128, 1 << 30), 128, 0, st>>>(pool, rec, nRec, out.nodes, derr);
    BK(cudaGetLastError());
    uint32_t bound = 0;
    BK(cudaMemcpyAsync(&bound, counters + 4, 4, cudaMemcpyDeviceToHost, st));
    BK(cudaMemcpyAsync(&herr, derr, 4, cudaMemcpyDeviceToHost, st));
    BK(cudaStreamSynchronize(st));
    if (herr) {
        err = "device BVH build: an internal bound was exceeded";
        return ANA_ERR_CUDA;
    }
    if (bound > kMaxStack4) {
        err = "triangle BVH deeper than the traversal stack";
        return ANA_ERR_UNSUPPORTED;
    }
    lap(3);
    return ANA_OK;
}

}  // namespace ana
