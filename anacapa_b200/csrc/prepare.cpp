// Host scene preparation. Compiled with -ffp-contract=off: every float
// operation here rounds on its own, so the triangle data, BVH boxes, strand
// widths and dome distribution are bit-identical to what the reference
// computes in the same order of operations.
#include "prepare.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>
#include <numeric>
#include <thread>

namespace ana {

namespace {

struct V3 {
    float x, y, z;
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length(V3 v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
// Types.h:80-89
inline V3 normalize(V3 v) { return mul(v, 1.f / length(v)); }
inline V3 safeNormalize(V3 v, V3 fb = {0.f, 0.f, 1.f}) {
    float len = length(v);
    return len > 1e-8f ? mul(v, 1.f / len) : fb;
}
inline V3 load3(const float* p) { return {p[0], p[1], p[2]}; }
// Mat4f::transformPoint (Types.h:144-150), row-major m
inline V3 xform_point(const float* m, V3 p) {
    float x = m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3];
    float y = m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7];
    float z = m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11];
    float w = m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15];
    return {x / w, y / w, z / w};
}
inline float4 f4(V3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
inline float bits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

struct Box {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void expand(const float* p) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    void expand(const Box& b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    float diag(int a) const { return hi[a] - lo[a]; }
    // 2 (dx dy + dy dz + dz dx), BVHBackend.cpp:324, 350-353
    float area() const {
        float dx = diag(0), dy = diag(1), dz = diag(2);
        return 2.f * (dx * dy + dy * dz + dz * dx);
    }
};

// ---------------------------------------------------------------------------
// Binary BVH build tree (both builders produce this; flatten_bvh4 lays the
// triangle and the curve trees out as 128-byte 4-wide nodes).
// ---------------------------------------------------------------------------
struct BuildNode {
    Box box;
    int32_t left = -1, right = -1;  // children (interior)
    uint32_t start = 0, count = 0;  // primitive range in the build order (leaf)
};

struct NodePool {
    std::vector<BuildNode> nodes;
    std::atomic<uint32_t> next{0};
    explicit NodePool(size_t cap) : nodes(cap) {}
    uint32_t alloc() { return next.fetch_add(1, std::memory_order_relaxed); }
};

// ---------------------------------------------------------------------------
// Triangle SAH build: the algorithm of BVHBackend::commit / buildRecursive /
// sahSplit (src/accel/BVHBackend.cpp:17-228): primitive boxes padded by 1e-7
// where flat, 12 centroid buckets per axis, split cost 1 + sum(area * count) /
// parentArea against a leaf cost of count, leaves of at most max_leaf
// triangles, std::partition on the chosen bucket and a median fallback.
// ---------------------------------------------------------------------------
struct PrimInfo {
    Box box;
    float c[3];
    uint32_t idx;
};

constexpr int kBuckets = 12;

int sah_split(const std::vector<PrimInfo>& pi, uint32_t start, uint32_t end, const Box& cb,
              int& outAxis) {
    float bestCost = INFINITY;
    int bestSplit = -1;
    outAxis = -1;
    Box parent;
    for (uint32_t i = start; i < end; ++i) parent.expand(pi[i].box);
    float parentArea = parent.area();
    if (parentArea < 1e-12f) return -1;
    for (int axis = 0; axis < 3; ++axis) {
        float range = cb.diag(axis);
        if (range < 1e-7f) continue;
        Box bb[kBuckets];
        uint32_t bc[kBuckets] = {};
        for (uint32_t i = start; i < end; ++i) {
            int b = static_cast<int>(kBuckets * ((pi[i].c[axis] - cb.lo[axis]) / range));
            b = std::clamp(b, 0, kBuckets - 1);
            bc[b]++;
            bb[b].expand(pi[i].box);
        }
        Box lb[kBuckets - 1];
        uint32_t lcnt[kBuckets - 1];
        Box acc;
        uint32_t ac = 0;
        for (int i = 0; i < kBuckets - 1; ++i) {
            acc.expand(bb[i]);
            ac += bc[i];
            lb[i] = acc;
            lcnt[i] = ac;
        }
        Box rb;
        uint32_t rc = 0;
        for (int i = kBuckets - 2; i >= 0; --i) {
            rb.expand(bb[i + 1]);
            rc += bc[i + 1];
            float cost = 1.f + 1.f * (lb[i].area() * float(lcnt[i]) + rb.area() * float(rc)) /
                                   parentArea;
            if (cost < bestCost) {
                bestCost = cost;
                bestSplit = i;
                outAxis = axis;
            }
        }
    }
    float leafCost = 1.f * static_cast<float>(end - start);
    if (bestCost >= leafCost) {
        outAxis = -1;
        return -1;
    }
    return bestSplit;
}

uint32_t sah_build(std::vector<PrimInfo>& pi, uint32_t start, uint32_t end, uint32_t maxLeaf,
                   NodePool& pool, int depth) {
    uint32_t ni = pool.alloc();
    Box bounds, cb;
    for (uint32_t i = start; i < end; ++i) {
        bounds.expand(pi[i].box);
        cb.expand(pi[i].c);
    }
    uint32_t count = end - start;
    int axis = -1, split = -1;
    if (count > maxLeaf) split = sah_split(pi, start, end, cb, axis);
    BuildNode& n = pool.nodes[ni];
    n.box = bounds;
    if (axis < 0 || split < 0) {
        n.start = start;
        n.count = count;
        return ni;
    }
    float range = cb.diag(axis);
    uint32_t mid = start;
    if (range > 0.f) {
        PrimInfo* p = std::partition(pi.data() + start, pi.data() + end, [&](const PrimInfo& q) {
            int b = static_cast<int>(kBuckets * ((q.c[axis] - cb.lo[axis]) / range));
            return std::clamp(b, 0, kBuckets - 1) <= split;
        });
        mid = static_cast<uint32_t>(p - pi.data());
    }
    if (mid == start || mid == end) mid = start + count / 2;
    uint32_t l, r;
    // Large subtrees on separate threads: the result does not depend on it
    // (subtrees touch disjoint primitive ranges; node ids are renumbered when
    // the tree is flattened depth-first).
    if (depth < 6 && count > 65536) {
        auto fut = std::async(std::launch::async, [&] {
            return sah_build(pi, start, mid, maxLeaf, pool, depth + 1);
        });
        r = sah_build(pi, mid, end, maxLeaf, pool, depth + 1);
        l = fut.get();
    } else {
        l = sah_build(pi, start, mid, maxLeaf, pool, depth + 1);
        r = sah_build(pi, mid, end, maxLeaf, pool, depth + 1);
    }
    pool.nodes[ni].left = int32_t(l);
    pool.nodes[ni].right = int32_t(r);
    return ni;
}

// ---------------------------------------------------------------------------
// Curve segment BVH: the algorithm of buildCurveBVH (src/accel/CurveBrute.cpp:
// 247-320): node box = union of segment boxes, leaves of at most max_leaf
// segments, otherwise split at the median (std::nth_element) along the axis of
// largest centroid extent.
// ---------------------------------------------------------------------------
struct SegWork {
    uint32_t strand, seg;
    float lo[3], hi[3], c[3];
};

uint32_t curve_build(std::vector<SegWork>& w, uint32_t start, uint32_t end, uint32_t maxLeaf,
                     NodePool& pool, int depth) {
    uint32_t ni = pool.alloc();
    Box b;
    for (uint32_t i = start; i < end; ++i)
        for (int k = 0; k < 3; ++k) {
            if (w[i].lo[k] < b.lo[k]) b.lo[k] = w[i].lo[k];
            if (w[i].hi[k] > b.hi[k]) b.hi[k] = w[i].hi[k];
        }
    // The reference initialises with +-FLT_MAX rather than +-inf; a node always
    // holds at least one segment, so both give the same box.
    uint32_t count = end - start;
    pool.nodes[ni].box = b;
    if (count <= maxLeaf) {
        pool.nodes[ni].start = start;
        pool.nodes[ni].count = count;
        return ni;
    }
    float cmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = start; i < end; ++i)
        for (int k = 0; k < 3; ++k) {
            if (w[i].c[k] < cmin[k]) cmin[k] = w[i].c[k];
            if (w[i].c[k] > cmax[k]) cmax[k] = w[i].c[k];
        }
    int axis = 0;
    float ext[3] = {cmax[0] - cmin[0], cmax[1] - cmin[1], cmax[2] - cmin[2]};
    if (ext[1] > ext[0]) axis = 1;
    if (ext[2] > ext[axis]) axis = 2;
    uint32_t mid = (start + end) / 2;
    std::nth_element(w.begin() + start, w.begin() + mid, w.begin() + end,
                     [axis](const SegWork& a, const SegWork& c) { return a.c[axis] < c.c[axis]; });
    uint32_t l, r;
    if (depth < 6 && count > 65536) {
        auto fut = std::async(std::launch::async,
                              [&] { return curve_build(w, start, mid, maxLeaf, pool, depth + 1); });
        r = curve_build(w, mid, end, maxLeaf, pool, depth + 1);
        l = fut.get();
    } else {
        l = curve_build(w, start, mid, maxLeaf, pool, depth + 1);
        r = curve_build(w, mid, end, maxLeaf, pool, depth + 1);
    }
    pool.nodes[ni].left = int32_t(l);
    pool.nodes[ni].right = int32_t(r);
    return ni;
}

// ---------------------------------------------------------------------------
// Collapse a binary build tree into 4-wide nodes. A node's children start as
// its binary node's two children; the interior child of largest surface area
// is replaced by its own two children until there are four or only leaves
// remain. Every child box is therefore a box of the binary tree, bit for bit,
// and a box contains its descendants' boxes, so a ray that passes a child's
// slab test passes every skipped ancestor's: the triangles tested are those
// the binary traversal would test (the same holds for the curve tree and
// CurveBrute's box test, whose slab and inside tests are monotone in the
// box). Nodes are laid out depth-first; returns the
// worst root-to-leaf sum of (children - 1), the traversal stack bound.
// ---------------------------------------------------------------------------
template <class EmitLeaf>
uint32_t flatten_bvh4(const NodePool& pool, uint32_t root, std::vector<Bvh4Node>& out, bool& rootEmpty,
                      EmitLeaf emit_leaf) {
    out.clear();
    auto set_child = [](Bvh4Node& n, int k, const Box& b, uint32_t ref) {
        (&n.lox.x)[k] = b.lo[0];
        (&n.hix.x)[k] = b.hi[0];
        (&n.loy.x)[k] = b.lo[1];
        (&n.hiy.x)[k] = b.hi[1];
        (&n.loz.x)[k] = b.lo[2];
        (&n.hiz.x)[k] = b.hi[2];
        (&n.ref.x)[k] = ref;
    };
    auto empty_node = [&]() {
        Bvh4Node n;
        std::memset(&n, 0, sizeof(n));
        Box e;
        for (int k = 0; k < 4; ++k) set_child(n, k, e, kEmptyChild);
        return n;
    };
    auto area = [](const Box& b) {
        float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
        return dx * dy + dy * dz + dz * dx;
    };
    const BuildNode& R = pool.nodes[root];
    if (R.count > 0 || R.left < 0) {
        rootEmpty = R.count == 0;
        Bvh4Node n = empty_node();
        if (R.count) set_child(n, 0, R.box, 0x80000000u | ((R.count - 1u) << 25) | emit_leaf(R.start, R.count));
        out.push_back(n);
        return 0;
    }
    rootEmpty = false;
    struct Item {
        uint32_t bn;
        int32_t parent;
        int slot;
        uint32_t depth;  // pushes on the way from the root to this node
    };
    std::vector<Item> stack;
    stack.push_back({root, -1, 0, 0});
    uint32_t bound = 0;
    while (!stack.empty()) {
        const Item it = stack.back();
        stack.pop_back();
        const BuildNode& b = pool.nodes[it.bn];
        if (b.count > 0) {
            const uint32_t off = emit_leaf(b.start, b.count);
            set_child(out[size_t(it.parent)], it.slot, b.box, 0x80000000u | ((b.count - 1u) << 25) | off);
            bound = std::max(bound, it.depth);
            continue;
        }
        const uint32_t idx = uint32_t(out.size());
        out.push_back(empty_node());
        if (it.parent >= 0) set_child(out[size_t(it.parent)], it.slot, b.box, idx);
        uint32_t kids[4] = {uint32_t(b.left), uint32_t(b.right), 0, 0};
        int nk = 2;
        while (nk < 4) {
            int pick = -1;
            float best = -1.f;
            for (int k = 0; k < nk; ++k) {
                const BuildNode& c = pool.nodes[kids[k]];
                if (c.count == 0 && c.left >= 0 && area(c.box) > best) {
                    best = area(c.box);
                    pick = k;
                }
            }
            if (pick < 0) break;
            const BuildNode& c = pool.nodes[kids[pick]];
            for (int k = nk; k > pick + 1; --k) kids[k] = kids[k - 1];  // keep left-to-right order
            kids[pick] = uint32_t(c.left);
            kids[pick + 1] = uint32_t(c.right);
            ++nk;
        }
        const uint32_t d = it.depth + uint32_t(nk - 1);
        // push in reverse so the leftmost child is placed (and its leaves emitted) first
        for (int k = nk - 1; k >= 0; --k) stack.push_back({kids[k], int32_t(idx), k, d});
    }
    return bound;
}

// StrandDesc::widthAt (include/anacapa/accel/CurvePool.h:45-54)
float width_at(const float* w, uint32_t n, float v) {
    if (n == 0) return 0.001f;
    if (n == 1) return w[0];
    if (n == 2) return w[0] * (1.f - v) + w[1] * v;
    float idx = v * float(int(n) - 1);
    int lo = std::max(0, int(idx));
    int hi = std::min(int(n) - 1, lo + 1);
    float frac = idx - float(lo);
    return w[lo] * (1.f - frac) + w[hi] * frac;
}

// Distribution1D::build (src/shading/lights/DomeLight.h:152-164)
float dist_build(const float* vals, uint32_t n, float* func, float* cdf) {
    for (uint32_t i = 0; i < n; ++i) func[i] = vals[i];
    cdf[0] = 0.f;
    for (uint32_t i = 0; i < n; ++i) cdf[i + 1] = cdf[i] + func[i];
    float integral = cdf[n];
    if (integral > 0.f) {
        float inv = 1.f / integral;
        for (uint32_t i = 0; i <= n; ++i) cdf[i] *= inv;
    }
    return integral;
}

bool finite3(const float* p) { return std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]); }

}  // namespace

uint64_t Prepared::bytes() const {
    return tri_nodes.size() * sizeof(Bvh4Node) + tri_isect.size() * 16 + tri_shade.size() * 16 +
           seg_nodes.size() * sizeof(Bvh4Node) + segs.size() * 16 + strand_color.size() * 4 +
           materials.size() * sizeof(DevMaterial) + slot_material.size() * 4 +
           lights.size() * sizeof(DevLight) +
           (env.rgb.size() + env.cond_func.size() + env.cond_cdf.size() + env.cond_int.size() +
            env.marg_func.size() + env.marg_cdf.size()) * 4;
}

DevCamera make_camera(const ana_camera& c, uint32_t width, uint32_t height) {
    if (c.explicit_basis) {
        DevCamera d{};
        auto f3 = [](const float* p) { return make_float3(p[0], p[1], p[2]); };
        d.origin = f3(c.origin);
        d.lower_left = f3(c.lower_left);
        d.horizontal = f3(c.horizontal);
        d.vertical = f3(c.vertical);
        d.basis_u = f3(c.basis_u);
        d.basis_v = f3(c.basis_v);
        d.aperture = c.aperture_radius;
        d.focal_distance = c.focal_distance;
        d.shutter_open = c.shutter_open;
        d.shutter_close = c.shutter_close;
        d.width = width;
        d.height = height;
        return d;
    }
    float theta = c.vfov_deg * 3.14159265f / 180.f;
    float h = std::tan(theta * 0.5f);
    float aspect = static_cast<float>(width) / static_cast<float>(height);
    V3 from = load3(c.from), at = load3(c.at), up = load3(c.up);
    V3 w = normalize(sub(from, at));
    V3 u = normalize(cross(up, w));
    V3 v = cross(w, u);
    float vpH = 2.f * h;
    float vpW = aspect * vpH;
    DevCamera d{};
    d.origin = make_float3(from.x, from.y, from.z);
    V3 hz = mul(u, vpW), vt = mul(v, vpH);
    V3 ll = sub(sub(sub(from, mul(u, vpW * 0.5f)), mul(v, vpH * 0.5f)), w);
    d.horizontal = make_float3(hz.x, hz.y, hz.z);
    d.vertical = make_float3(vt.x, vt.y, vt.z);
    d.lower_left = make_float3(ll.x, ll.y, ll.z);
    d.basis_u = make_float3(u.x, u.y, u.z);
    d.basis_v = make_float3(v.x, v.y, v.z);
    d.aperture = c.aperture_radius;
    d.focal_distance = c.focal_distance;
    d.shutter_open = c.shutter_open;
    d.shutter_close = c.shutter_close;
    d.width = width;
    d.height = height;
    return d;
}

void derive_standard(DevMaterial& o) {
    const float r = o.rough;
    const float a = std::max(1e-4f, r * r);  // sample/evaluate: max(1e-4, rough^2)
    o.alpha2 = a * a;
    float at = r * r;  // evaluate(), transmission lobe: rough^2 squared, no clamp
    at *= at;
    o.alpha2_t = at;
    uint32_t f = 16u;
    if (o.transmission > 0.001f) f |= 8u;
    if (r < 0.001f) f |= 4u;
    else if (r < 0.3f) f |= 2u;
    else f |= 1u;
    o.flags = f;
    const bool smoothGlass = r < 0.001f && o.transmission > 0.001f && o.metal < 0.001f;
    o.is_delta = (smoothGlass || (r < 0.001f && (o.metal > 0.999f || o.spec > 0.f))) ? 1 : 0;
}

// One material in the device layout, with the derived constants each
// reference class precomputes in its constructor (Lambertian.h:29-99,
// StandardSurface.h:152-218, MarschnerHair.h:200-216). Returns nullptr, or
// the reason the material is rejected.
const char* make_material(const ana_material& m, DevMaterial& o) {
    std::memset(&o, 0, sizeof(o));
    o.type = m.type;
    o.opacity = 1.f;  // IMaterial::evalOpacity's default
    switch (m.type) {
        case ANA_MAT_LAMBERT:
        case ANA_MAT_EMISSIVE:  // Lambertian.h:29-99
            o.flags = 1u | 16u;
            o.albedo = make_float3(m.albedo[0], m.albedo[1], m.albedo[2]);
            if (m.type == ANA_MAT_EMISSIVE)
                o.emission = make_float3(m.emission[0], m.emission[1], m.emission[2]);
            break;
        case ANA_MAT_STANDARD: {  // StandardSurface.h:152-218
            o.albedo = make_float3(m.base_color[0], m.base_color[1], m.base_color[2]);
            o.base = m.base;
            o.metal = m.metalness;
            o.rough = m.roughness;
            o.spec = m.specular;
            o.spec_color = make_float3(m.specular_color[0], m.specular_color[1], m.specular_color[2]);
            o.coat = m.coat;
            o.transmission = m.transmission;
            o.ior = m.specular_ior;
            derive_standard(o);
            float ca = std::max(1e-4f, m.coat_roughness * m.coat_roughness);
            o.coat_alpha2 = ca * ca;
            float r = (1.f - m.specular_ior) / (1.f + m.specular_ior);
            o.f0_dielectric = r * r;
            float rc = (1.f - 1.5f) / (1.f + 1.5f);
            o.coat_f0 = rc * rc;
            if (m.emission_weight > 0.f)
                o.emission = make_float3(m.emission_color[0] * m.emission_weight,
                                         m.emission_color[1] * m.emission_weight,
                                         m.emission_color[2] * m.emission_weight);
            // evalOpacity and transmittanceColor (StandardSurface.h:197-218)
            o.opacity = m.alpha_mask ? m.opacity : 1.f;
            if (m.alpha_mask) {
                const float t = 1.f - m.opacity;
                if (t > 0.f) o.tint = make_float3(t, t, t);
            } else if (m.transmission >= 0.001f && !(m.metalness > 0.001f)) {
                // Fresnel reflectance at normal incidence, fresnelDielectric(1, IOR)
                const float eta = m.specular_ior;
                const float Rs = (1.f - eta * 1.f) / (1.f + eta * 1.f);
                const float Rp = (eta * 1.f - 1.f) / (eta * 1.f + 1.f);
                const float Fr = 0.5f * (Rs * Rs + Rp * Rp);
                const float k = m.transmission * (1.f - Fr);
                o.tint = make_float3(m.base_color[0] * k, m.base_color[1] * k, m.base_color[2] * k);
            }
            break;
        }
        case ANA_MAT_HAIR: {  // MarschnerHair.h:200-216
            o.hair_mode = m.hair_mode;
            if (m.hair_mode > ANA_HAIR_MARSCHNER) return "unknown hair mode";
            o.eta = m.eta;
            o.sigma_a = make_float3(m.sigma_a[0], m.sigma_a[1], m.sigma_a[2]);
            o.beta_m = m.beta_m;
            float bm = std::clamp(m.beta_m, 1e-3f, 1.f);
            float v0 = 0.726f * bm + 0.812f * bm * bm + 3.7f * std::pow(bm, 20.f);
            o.v[0] = v0 * v0;
            o.v[1] = o.v[0] * 0.25f;
            o.v[2] = o.v[0] * 4.0f;
            float bn = std::clamp(m.beta_n, 1e-3f, 1.f);
            o.s = 0.626657069f * (0.265f * bn + 1.194f * bn * bn + 5.372f * std::pow(bn, 22.f));
            const float kPi = 3.14159265358979323846f;
            o.alpha_shift[0] = -m.alpha_deg * kPi / 180.f;
            o.alpha_shift[1] = m.alpha_deg * kPi / 180.f * 0.5f;
            o.alpha_shift[2] = -m.alpha_deg * kPi / 180.f * 1.5f;
            o.flags = 2u | 16u | 8u;
            break;
        }
        default:
            return "unknown material type";
    }
    return nullptr;
}

int prepare_scene(const ana_scene_desc& d, Prepared& P, std::string& err, bool tris_on_device) {
    auto bad = [&](const char* m) {
        err = m;
        return int(ANA_ERR_INVALID_ARG);
    };
    auto unsupported = [&](const char* m) {
        err = m;
        return int(ANA_ERR_UNSUPPORTED);
    };
    if (d.num_meshes && (!d.mesh_vert_offset || !d.mesh_tri_offset || !d.positions || !d.indices))
        return bad("mesh arrays missing");
    if (d.num_strands && (!d.strand_cp_offset || !d.control_points || !d.strand_width_offset ||
                          !d.strand_slot))
        return bad("strand arrays missing");
    if (d.num_materials && !d.materials) return bad("materials missing");
    if (d.num_slots && !d.slot_material) return bad("slot table missing");
    if (d.num_lights && !d.lights) return bad("lights missing");
    if (d.env_rgb && (d.env_width == 0 || d.env_height == 0)) return bad("empty env map");

    // ---- triangles: BVHBackend::commit (BVHBackend.cpp:17-111) ------------
    const uint32_t T = d.num_meshes ? d.mesh_tri_offset[d.num_meshes] : 0;
    // Leaf references carry the first primitive in 25 bits (traverse.cuh).
    if (T >= (1u << 25)) return bad("more than 2^25 triangles");
    P.num_tris = T;
    P.mesh_motion.clear();
    P.motion_keys.clear();
    const auto motion_keys_of = [&](uint32_t m) -> uint32_t {
        return d.mesh_motion_offset ? d.mesh_motion_offset[m + 1] - d.mesh_motion_offset[m] : 0u;
    };
    bool anyMotion = false;
    for (uint32_t m = 0; m < d.num_meshes; ++m) {
        if (d.mesh_motion_offset && d.mesh_motion_offset[m + 1] < d.mesh_motion_offset[m])
            return bad("motion key offsets not monotone");
        if (motion_keys_of(m)) anyMotion = true;
    }
    if (anyMotion && !d.motion_keys) return bad("motion keys missing");
    P.tris_on_device = tris_on_device && T > 0 && !anyMotion;  // motion meshes: host build
    P.dev_tri_nodes = 0;
    if (P.tris_on_device) {
        for (uint32_t m = 0; m < d.num_meshes; ++m)
            if (d.mesh_vert_offset[m + 1] < d.mesh_vert_offset[m] || d.mesh_tri_offset[m + 1] < d.mesh_tri_offset[m])
                return bad("mesh offsets not monotone");
    }
    std::vector<float4> isect(P.tris_on_device ? 0 : size_t(T) * 3);  // build order = mesh order first
    P.tri_shade.assign(P.tris_on_device ? 0 : size_t(T) * 4, make_float4(0, 0, 0, 0));
    std::vector<PrimInfo> pi(P.tris_on_device ? 0 : T);
    for (uint32_t m = 0; m < (P.tris_on_device ? 0u : d.num_meshes); ++m) {
        uint32_t v0i = d.mesh_vert_offset[m], v1i = d.mesh_vert_offset[m + 1];
        uint32_t t0 = d.mesh_tri_offset[m], t1 = d.mesh_tri_offset[m + 1];
        if (v1i < v0i || t1 < t0) return bad("mesh offsets not monotone");
        uint32_t nv = v1i - v0i;
        bool hasN = d.mesh_has_normals && d.mesh_has_normals[m] && d.normals;
        // motion mesh: object-space triangle data, time-expanded world bounds
        const uint32_t nk = motion_keys_of(m);
        const ana_motion_key* keys = nk ? d.motion_keys + d.mesh_motion_offset[m] : nullptr;
        const uint32_t mm = uint32_t(P.mesh_motion.size());
        if (nk) {
            P.mesh_motion.push_back(make_uint2(uint32_t(P.motion_keys.size() / 5), nk));
            for (uint32_t k = 0; k < nk; ++k) {
                const float* M = keys[k].object_to_world;
                for (int j = 0; j < 16; ++j)
                    if (!std::isfinite(M[j])) return bad("non-finite motion key");
                if (!std::isfinite(keys[k].time)) return bad("non-finite motion key");
                P.motion_keys.push_back(make_float4(keys[k].time, 0.f, 0.f, 0.f));
                for (int r = 0; r < 4; ++r) P.motion_keys.push_back(make_float4(M[4 * r], M[4 * r + 1], M[4 * r + 2], M[4 * r + 3]));
            }
        }
        for (uint32_t t = t0; t < t1; ++t) {
            uint32_t ia = d.indices[3 * size_t(t)], ib = d.indices[3 * size_t(t) + 1],
                     ic = d.indices[3 * size_t(t) + 2];
            if (ia >= nv || ib >= nv || ic >= nv) return bad("triangle index out of range");
            const float* pa = d.positions + 3 * size_t(v0i + ia);
            const float* pb = d.positions + 3 * size_t(v0i + ib);
            const float* pc = d.positions + 3 * size_t(v0i + ic);
            if (!finite3(pa) || !finite3(pb) || !finite3(pc)) return bad("non-finite vertex");
            V3 v0 = load3(pa), e1 = sub(load3(pb), v0), e2 = sub(load3(pc), v0);
            V3 n = safeNormalize(cross(e1, e2));
            auto sn = [&](uint32_t i) {
                return hasN ? safeNormalize(load3(d.normals + 3 * size_t(v0i + i))) : n;
            };
            V3 s0 = sn(ia), s1 = sn(ib), s2 = sn(ic);
            isect[3 * size_t(t) + 0] = f4(v0, bits(nk ? (t | 0x80000000u) : t));
            isect[3 * size_t(t) + 1] = f4(e1, nk ? bits(mm) : 0.f);
            isect[3 * size_t(t) + 2] = f4(e2, 0.f);
            P.tri_shade[4 * size_t(t) + 0] = f4(n, bits(m));
            P.tri_shade[4 * size_t(t) + 1] = f4(s0, bits(t - t0));
            P.tri_shade[4 * size_t(t) + 2] = f4(s1, 0.f);
            P.tri_shade[4 * size_t(t) + 3] = f4(s2, 0.f);
            // bounds from v0, v0 + e1, v0 + e2 (BVHBackend.cpp:78-80), for a
            // motion mesh their world positions at every key (BVHBackend.cpp:86-95)
            Box b;
            V3 w1 = add(v0, e1), w2 = add(v0, e2);
            if (nk) {
                for (uint32_t k = 0; k < nk; ++k) {
                    const float* M = keys[k].object_to_world;
                    const V3 q0 = xform_point(M, v0), q1 = xform_point(M, w1), q2 = xform_point(M, w2);
                    float a0[3] = {q0.x, q0.y, q0.z}, a1[3] = {q1.x, q1.y, q1.z}, a2[3] = {q2.x, q2.y, q2.z};
                    b.expand(a0);
                    b.expand(a1);
                    b.expand(a2);
                }
            } else {
                float a0[3] = {v0.x, v0.y, v0.z}, a1[3] = {w1.x, w1.y, w1.z}, a2[3] = {w2.x, w2.y, w2.z};
                b.expand(a0);
                b.expand(a1);
                b.expand(a2);
            }
            for (int ax = 0; ax < 3; ++ax)
                if (b.diag(ax) < 1e-7f) {
                    b.lo[ax] -= 1e-7f;
                    b.hi[ax] += 1e-7f;
                }
            PrimInfo& q = pi[t];
            q.box = b;
            for (int ax = 0; ax < 3; ++ax) q.c[ax] = (b.lo[ax] + b.hi[ax]) * 0.5f;
            q.idx = t;
        }
    }
    uint32_t maxLeafT = d.max_leaf_tris ? d.max_leaf_tris : 4;
    // Curve leaves default to one segment (the reference builds leaves of 4,
    // CurveBrute.cpp:455): the 4-wide nodes then bounds-test every segment's
    // own box before its ribbon test, which culls most root projections
    // (1280x720x32 hair frame: 1085 ms against 1367 ms with leaves of 4). The
    // tree is still the reference's median split, so hits are the same.
    uint32_t maxLeafS = d.max_leaf_segments ? d.max_leaf_segments : 1;
    if (maxLeafT > 64 || maxLeafS > 64) return bad("leaf size > 64");
    P.tri_isect.clear();
    if (P.tris_on_device) {
        P.tri_nodes.clear();
        P.tri_root_is_empty = false;
    } else if (T > 0) {
        NodePool pool(2 * size_t(T) + 1);
        uint32_t root = sah_build(pi, 0, T, maxLeafT, pool, 0);
        P.tri_isect.reserve(size_t(T) * 3);
        const uint32_t stackBound = flatten_bvh4(pool, root, P.tri_nodes, P.tri_root_is_empty, [&](uint32_t s, uint32_t c) {
            uint32_t off = uint32_t(P.tri_isect.size() / 3);
            for (uint32_t i = s; i < s + c; ++i)
                for (int k = 0; k < 3; ++k) P.tri_isect.push_back(isect[3 * size_t(pi[i].idx) + k]);
            return off;
        });
        if (stackBound > kMaxStack4) return unsupported("triangle BVH deeper than the traversal stack");
    } else {
        P.tri_nodes.clear();
        P.tri_root_is_empty = true;
    }

    // ---- curves: CurveBrute::commit (CurveBrute.cpp:332-396) ---------------
    std::vector<SegWork> work;
    std::vector<float4> segRec;  // 5 per (strand, seg) in enumeration order
    P.strand_color.assign(size_t(d.num_strands) * 3, 1.f);
    for (uint32_t s = 0; s < d.num_strands; ++s) {
        uint32_t c0 = d.strand_cp_offset[s], c1 = d.strand_cp_offset[s + 1];
        uint32_t w0 = d.strand_width_offset[s], w1 = d.strand_width_offset[s + 1];
        if (c1 < c0 || w1 < w0) return bad("strand offsets not monotone");
        if (d.strand_color)
            for (int k = 0; k < 3; ++k) P.strand_color[3 * size_t(s) + k] = d.strand_color[3 * size_t(s) + k];
        uint32_t ncp = c1 - c0;
        uint32_t N = ncp < 4 ? 0 : (ncp - 1) / 3;
        const float* W = d.widths ? d.widths + w0 : nullptr;
        uint32_t nw = W ? (w1 - w0) : 0;
        for (uint32_t k = 0; k < N; ++k) {
            const float* P0 = d.control_points + 3 * size_t(c0 + 3 * k);
            V3 p[4] = {load3(P0), load3(P0 + 3), load3(P0 + 6), load3(P0 + 9)};
            for (auto& q : p)
                if (!std::isfinite(q.x) || !std::isfinite(q.y) || !std::isfinite(q.z))
                    return bad("non-finite control point");
            float v0 = float(k) / float(N);
            float v3 = float(k + 1) / float(N);
            float wa = width_at(W, nw, v0), wb = width_at(W, nw, v3);
            float maxHalfW = std::max(wa, wb) * 0.5f;
            SegWork sw;
            sw.strand = s;
            sw.seg = k;
            for (int a = 0; a < 3; ++a) {
                sw.lo[a] = std::min({p[0][a], p[1][a], p[2][a], p[3][a]}) - maxHalfW;
                sw.hi[a] = std::max({p[0][a], p[1][a], p[2][a], p[3][a]}) + maxHalfW;
            }
            for (int a = 0; a < 3; ++a) sw.c[a] = (sw.lo[a] + sw.hi[a]) * 0.5f;
            work.push_back(sw);
            // intersectOneSegment's per-segment constants (CurveBrute.cpp:182-206)
            segRec.push_back(f4(p[0], wa * 0.5f));
            segRec.push_back(f4(p[1], wb * 0.5f));
            segRec.push_back(f4(p[2], v0));
            segRec.push_back(f4(p[3], v3 - v0));
            uint32_t slot = d.strand_slot[s];
            segRec.push_back(make_float4(bits(s), bits(k), bits(slot), 0.f));
        }
    }
    if (work.size() >= (size_t(1) << 25)) return bad("more than 2^25 curve segments");
    P.num_segs = uint32_t(work.size());
    P.segs.clear();
    P.seg_nodes.clear();
    if (!work.empty()) {
        // enumeration index of each SegWork, for the leaf-order copy
        std::vector<uint32_t> segBase(d.num_strands + 1, 0);
        for (const SegWork& sw : work) segBase[sw.strand + 1] = std::max(segBase[sw.strand + 1], sw.seg + 1);
        for (uint32_t s = 0; s < d.num_strands; ++s) segBase[s + 1] += segBase[s];
        NodePool pool(2 * work.size() + 1);
        uint32_t root = curve_build(work, 0, uint32_t(work.size()), maxLeafS, pool, 0);
        bool empty;
        P.segs.reserve(work.size() * 5);
        const uint32_t stackBound = flatten_bvh4(pool, root, P.seg_nodes, empty, [&](uint32_t s, uint32_t c) {
            uint32_t off = uint32_t(P.segs.size() / 5);
            for (uint32_t i = s; i < s + c; ++i) {
                size_t e = segBase[work[i].strand] + work[i].seg;
                for (int k = 0; k < 5; ++k) P.segs.push_back(segRec[5 * e + k]);
            }
            return off;
        });
        if (stackBound > kMaxStack4) return unsupported("curve BVH deeper than the traversal stack");
    }

    // ---- materials -----------------------------------------------------------
    P.materials.resize(d.num_materials);
    for (uint32_t i = 0; i < d.num_materials; ++i) {
        const char* why = make_material(d.materials[i], P.materials[i]);
        if (why) return bad(why);
    }
    P.slot_material.assign(d.slot_material, d.slot_material + d.num_slots);
    P.has_emitters = false;
    P.has_transmit = false;
    for (int32_t s : P.slot_material) {
        if (s >= int32_t(d.num_materials)) return bad("slot refers to a missing material");
        if (s >= 0) {
            const float3 e = P.materials[size_t(s)].emission;
            if (e.x != 0.f || e.y != 0.f || e.z != 0.f) P.has_emitters = true;
            const float3 t = P.materials[size_t(s)].tint;
            if (t.x != 0.f || t.y != 0.f || t.z != 0.f) P.has_transmit = true;
        }
    }

    // ---- lights --------------------------------------------------------------
    P.lights.clear();
    bool hasDome = false;
    for (uint32_t i = 0; i < d.num_lights; ++i) {
        const ana_light& l = d.lights[i];
        DevLight o;
        std::memset(&o, 0, sizeof(o));
        o.type = l.type;
        if (l.type == ANA_LIGHT_AREA) {  // AreaLight.h:22-30
            V3 u = load3(l.u), v = load3(l.v);
            V3 c = cross(u, v);
            V3 n = safeNormalize(c);
            o.center = make_float3(l.center[0], l.center[1], l.center[2]);
            o.u = make_float3(u.x, u.y, u.z);
            o.v = make_float3(v.x, v.y, v.z);
            o.normal = make_float3(n.x, n.y, n.z);
            o.Le = make_float3(l.Le[0], l.Le[1], l.Le[2]);
            o.area = length(c) * 4.f;
            float ul = length(u), vl = length(v);
            o.uLen2 = ul * ul;
            o.vLen2 = vl * vl;
        } else if (l.type == ANA_LIGHT_DOME) {
            if (hasDome) return bad("more than one dome light");
            hasDome = true;
        } else if (l.type == ANA_LIGHT_DIRECTIONAL) {  // DirectionalLight.h:33-45
            const V3 dir = safeNormalize(load3(l.u));
            o.normal = make_float3(dir.x, dir.y, dir.z);
            o.Le = make_float3(l.Le[0], l.Le[1], l.Le[2]);
            const float kPi = 3.14159265358979323846f;
            o.cos_cone = std::cos(l.half_angle_deg * kPi / 180.f);
        } else {
            return bad("unknown light type");
        }
        P.lights.push_back(o);
    }

    // ---- dome: DomeLight::buildDistribution (DomeLight.h:355-386) -------------
    HostEnv& E = P.env;
    E = HostEnv{};
    E.radiance[0] = d.env_radiance[0];
    E.radiance[1] = d.env_radiance[1];
    E.radiance[2] = d.env_radiance[2];
    if (hasDome && !d.env_rgb) return bad("dome light without an env map");
    if (d.env_rgb) {
        E.present = true;
        E.intensity = d.env_intensity;
        uint32_t W = d.env_width, H = d.env_height;
        E.width = W;
        E.height = H;
        E.rgb.assign(d.env_rgb, d.env_rgb + size_t(W) * H * 3);
        E.cond_func.resize(size_t(W) * H);
        E.cond_cdf.resize(size_t(W + 1) * H);
        E.cond_int.resize(H);
        std::vector<float> rowFunc(W), rowSums(H);
        const float kPi = 3.14159265358979323846f;
        for (uint32_t r = 0; r < H; ++r) {
            float theta = kPi * (r + 0.5f) / static_cast<float>(H);
            float sinTheta = std::sin(theta);
            for (uint32_t c = 0; c < W; ++c) {
                const float* px = E.rgb.data() + (size_t(r) * W + c) * 3;
                float lum = 0.2126f * px[0] + 0.7152f * px[1] + 0.0722f * px[2];
                rowFunc[c] = lum * sinTheta;
            }
            E.cond_int[r] = dist_build(rowFunc.data(), W, E.cond_func.data() + size_t(r) * W,
                                       E.cond_cdf.data() + size_t(r) * (W + 1));
            rowSums[r] = E.cond_int[r];
        }
        E.marg_func.resize(H);
        E.marg_cdf.resize(H + 1);
        E.marg_int = dist_build(rowSums.data(), H, E.marg_func.data(), E.marg_cdf.data());
    }
    P.camera = d.camera;
    return ANA_OK;
}

}  // namespace ana
