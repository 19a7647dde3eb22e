// ============================================================================
// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT (see pt_oracle.h).
//
// Scene, acceleration, materials, lights and the Path integrator of the
// reference, restated in T = float / double, with a C API mirroring
// oracle/ref_harness.cpp so tests can drive both the same way.
// ============================================================================
#include "pt_oracle.h"

#include <array>
#include <atomic>
#include <type_traits>
#include <functional>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>

namespace po {

const uint32_t kPrimes[128] = {
    2,   3,   5,   7,   11,  13,  17,  19,  23,  29,  31,  37,  41,  43,  47,  53,
    59,  61,  67,  71,  73,  79,  83,  89,  97,  101, 103, 107, 109, 113, 127, 131,
    137, 139, 149, 151, 157, 163, 167, 173, 179, 181, 191, 193, 197, 199, 211, 223,
    227, 229, 233, 239, 241, 251, 257, 263, 269, 271, 277, 281, 283, 293, 307, 311,
    313, 317, 331, 337, 347, 349, 353, 359, 367, 373, 379, 383, 389, 397, 401, 409,
    419, 421, 431, 433, 439, 443, 449, 457, 461, 463, 467, 479, 487, 491, 499, 503,
    509, 521, 523, 541, 547, 557, 563, 569, 571, 577, 587, 593, 599, 601, 607, 613,
    617, 619, 631, 641, 643, 647, 653, 659, 661, 673, 677, 683, 691, 701, 709, 719};

template <class T> constexpr T kPi = T(3.14159265358979323846264338327950288L);
template <class T> constexpr T kInvPi = T(0.31830988618379067154L);
template <class T> constexpr T k2Pi = T(6.28318530717958647692L);
template <class T> T E(float f) { return T(f); }  // a reference float literal

void parallel_for(uint32_t n, int threads, const std::function<void(uint32_t)>& f) {
    unsigned nt = threads > 0 ? unsigned(threads) : std::max(1u, std::thread::hardware_concurrency());
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> ts;
    for (unsigned t = 0; t < nt; ++t)
        ts.emplace_back([&] {
            for (uint32_t i; (i = next.fetch_add(1)) < n;) f(i);
        });
    for (auto& t : ts) t.join();
}

// ---------------------------------------------------------------------------
// Geometry
// ---------------------------------------------------------------------------
template <class T>
struct Tri {
    V3<T> v0, e1, e2, n, sn0, sn1, sn2;
    uint32_t mesh, prim;
    bool objectSpace = false;  // a motion-blurred mesh's triangle (its keys: Scene::motion[mesh])
};

// Mat4f (include/anacapa/core/Types.h:144-229): the operations motion blur uses.
template <class T>
struct M4 {
    T m[4][4] = {};
    static M4 identity() {
        M4 r;
        for (int i = 0; i < 4; ++i) r.m[i][i] = T(1);
        return r;
    }
    V3<T> point(V3<T> p) const {
        T x = m[0][0] * p.x + m[0][1] * p.y + m[0][2] * p.z + m[0][3];
        T y = m[1][0] * p.x + m[1][1] * p.y + m[1][2] * p.z + m[1][3];
        T z = m[2][0] * p.x + m[2][1] * p.y + m[2][2] * p.z + m[2][3];
        T w = m[3][0] * p.x + m[3][1] * p.y + m[3][2] * p.z + m[3][3];
        return {x / w, y / w, z / w};
    }
    V3<T> vector(V3<T> v) const {
        return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
                m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
    }
    V3<T> normal(V3<T> n) const {  // the transpose, as transformNormal computes it
        return {m[0][0] * n.x + m[1][0] * n.y + m[2][0] * n.z, m[0][1] * n.x + m[1][1] * n.y + m[2][1] * n.z,
                m[0][2] * n.x + m[1][2] * n.y + m[2][2] * n.z};
    }
    static M4 lerp(const M4& a, const M4& b, T t) {
        M4 r;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) r.m[i][j] = a.m[i][j] * (T(1) - t) + b.m[i][j] * t;
        return r;
    }
    M4 inverse() const {  // Gauss-Jordan with partial pivoting; identity when singular
        T a[4][8];
        for (int i = 0; i < 4; ++i) {
            for (int j = 0; j < 4; ++j) a[i][j] = m[i][j];
            for (int j = 0; j < 4; ++j) a[i][j + 4] = (i == j) ? T(1) : T(0);
        }
        for (int col = 0; col < 4; ++col) {
            int pivot = col;
            for (int row = col + 1; row < 4; ++row)
                if (std::abs(a[row][col]) > std::abs(a[pivot][col])) pivot = row;
            if (pivot != col)
                for (int j = 0; j < 8; ++j) std::swap(a[col][j], a[pivot][j]);
            T diag = a[col][col];
            if (std::abs(diag) < T(1e-10f)) return identity();
            T invDiag = T(1) / diag;
            for (int j = 0; j < 8; ++j) a[col][j] *= invDiag;
            for (int row = 0; row < 4; ++row) {
                if (row == col) continue;
                T factor = a[row][col];
                for (int j = 0; j < 8; ++j) a[row][j] -= factor * a[col][j];
            }
        }
        M4 r;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) r.m[i][j] = a[i][j + 4];
        return r;
    }
};

// A motion key (MotionKey, GeometryPool.h:16-20).
template <class T>
struct Key {
    T time = 0;
    M4<T> o2w;
};

// MeshDesc::interpolateO2W (GeometryPool.h:51-65): piecewise-linear in the keys.
template <class T>
M4<T> interpO2W(const std::vector<Key<T>>& k, T t) {
    if (k.size() == 1) return k[0].o2w;
    if (t <= k.front().time) return k.front().o2w;
    if (t >= k.back().time) return k.back().o2w;
    size_t lo = 0, hi = k.size() - 1;
    while (hi - lo > 1) {
        size_t mid = (lo + hi) / 2;
        if (k[mid].time <= t) lo = mid;
        else hi = mid;
    }
    T alpha = (t - k[lo].time) / (k[hi].time - k[lo].time);
    return M4<T>::lerp(k[lo].o2w, k[hi].o2w, alpha);
}

template <class T>
struct Seg {
    V3<T> P[4];
    T hw0, hw3, v0, dv;
    uint32_t strand, seg, slot;
};

struct Node {  // binary BVH, median split on the longest centroid axis
    float lo[3], hi[3];
    uint32_t left, right, start, count;
};

template <class T>
struct Hit {
    bool hit = false;
    T t = 0, u = 0, v = 0;
    bool curve = false;
    uint32_t idx = 0;
    V3<T> tang;
    T tseg = 0;
};

enum { MAT_LAMBERT = 0, MAT_EMISSIVE = 1, MAT_STANDARD = 2, MAT_HAIR = 3 };

template <class T>
struct Mat {
    int type = 0;
    V3<T> albedo, emission;
    // standard_surface
    T base = 1, metal = 0, rough = 0.5, spec = 1, coat = 0, coatRough = T(0.1f), ior = T(1.5f);
    V3<T> specColor{1, 1, 1};
    T coatAlpha2 = 0, f0 = 0, coatF0 = 0;
    uint32_t flags = 0;
    bool delta = false;
    // glass and alpha masks (StandardSurface.h:197-218, 245-340, 410-462)
    T transmission = 0, opacity = 1;
    bool alphaMask = false;
    V3<T> tint;  // transmittanceColor: black = opaque to shadow rays
    // hair
    T eta = T(1.55f), bm = T(0.3f), bn = T(0.3f), alphaDeg = 2;
    V3<T> sigma;
    T v[3] = {0, 0, 0}, s = 0, ashift[3] = {0, 0, 0};
    int hairMode = 0;
};

template <class T>
struct Light {
    int type = 0;  // 0 area, 1 dome, 2 directional (n = direction toward it)
    V3<T> c, u, v, n, Le;
    T area = 1;
    T cosCone = 1;
};

template <class T>
struct Dist1D {  // DomeLight.h:146-182
    std::vector<T> func, cdf;
    T integral = 0;
    uint32_t n = 0;
    void build(const T* vals, uint32_t count) {
        n = count;
        func.assign(vals, vals + count);
        cdf.assign(count + 1, T(0));
        for (uint32_t i = 0; i < count; ++i) cdf[i + 1] = cdf[i] + func[i];
        integral = cdf[count];
        if (integral > T(0)) {
            T inv = T(1) / integral;
            for (auto& c : cdf) c *= inv;
        }
    }
    uint32_t sample(T u, T& pdf, T& ur) const {
        auto it = std::lower_bound(cdf.begin(), cdf.end(), u);
        int idx = int(it - cdf.begin()) - 1;
        idx = std::max(0, std::min(idx, int(n) - 1));
        T bw = cdf[idx + 1] - cdf[idx];
        ur = bw > T(1e-12f) ? (u - cdf[idx]) / bw : T(0);
        ur = std::max(T(0), std::min(ur, T(1) - T(1e-7f)));
        pdf = integral > T(0) ? func[idx] / integral : T(0);
        return uint32_t(idx);
    }
};

template <class T>
struct Scene {
    std::vector<Tri<T>> tris;
    std::vector<Seg<T>> segs;
    std::vector<V3<T>> strandColor;
    std::vector<Node> triNodes, segNodes;
    std::vector<uint32_t> triIdx, segIdx;
    std::vector<Mat<T>> mats;
    std::vector<int> slots;
    std::vector<Light<T>> lights;
    // dome
    bool dome = false;
    std::vector<T> env;
    uint32_t ew = 0, eh = 0;
    T intensity = 1;
    std::vector<Dist1D<T>> cond;
    Dist1D<T> marg;
    V3<T> envRadiance;
    bool transmit = false;  // a material passes shadow rays (non-black transmittanceColor)
    std::vector<std::vector<Key<T>>> motion;  // per meshID: its keys (empty: static)
    T shutterOpen = 0, shutterClose = 0;
    // camera (Camera::makePinhole, IIntegrator.h:49-74)
    V3<T> camO, camLL, camH, camV;
    uint32_t W = 0, H = 0;
    // pending strands (raw)
    struct RawStrand {
        std::vector<V3<T>> cps;
        std::vector<T> widths;
        uint32_t slot;
        V3<T> color;
    };
    std::vector<RawStrand> raw;
};

// BVH over boxes (own build: median split of centroids, leaves <= 4). Only
// the set of primitives a ray reaches matters for the closest hit.
template <class GetBox>
void build_bvh(uint32_t n, GetBox box, std::vector<Node>& nodes, std::vector<uint32_t>& idx) {
    nodes.clear();
    idx.resize(n);
    std::iota(idx.begin(), idx.end(), 0u);
    if (n == 0) return;
    std::vector<std::array<float, 6>> bb(n);
    for (uint32_t i = 0; i < n; ++i) box(i, bb[i].data());
    std::function<uint32_t(uint32_t, uint32_t)> rec = [&](uint32_t s, uint32_t e) -> uint32_t {
        uint32_t ni = uint32_t(nodes.size());
        nodes.push_back(Node{});
        Node nd{};
        for (int a = 0; a < 3; ++a) {
            nd.lo[a] = INFINITY;
            nd.hi[a] = -INFINITY;
        }
        float cl[3] = {INFINITY, INFINITY, INFINITY}, ch[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t i = s; i < e; ++i) {
            const auto& b = bb[idx[i]];
            for (int a = 0; a < 3; ++a) {
                nd.lo[a] = std::min(nd.lo[a], b[a]);
                nd.hi[a] = std::max(nd.hi[a], b[3 + a]);
                float c = 0.5f * (b[a] + b[3 + a]);
                cl[a] = std::min(cl[a], c);
                ch[a] = std::max(ch[a], c);
            }
        }
        if (e - s <= 4) {
            nd.start = s;
            nd.count = e - s;
            nodes[ni] = nd;
            return ni;
        }
        int ax = 0;
        for (int a = 1; a < 3; ++a)
            if (ch[a] - cl[a] > ch[ax] - cl[ax]) ax = a;
        uint32_t m = (s + e) / 2;
        std::nth_element(idx.begin() + s, idx.begin() + m, idx.begin() + e, [&](uint32_t a, uint32_t b) {
            return bb[a][ax] + bb[a][3 + ax] < bb[b][ax] + bb[b][3 + ax];
        });
        nd.count = 0;
        nd.left = rec(s, m);
        nd.right = rec(m, e);
        nodes[ni] = nd;
        return ni;
    };
    rec(0, n);
}

// Conservative node test in double (the accel only prunes; exactness lives in
// the primitive tests).
template <class T>
bool node_hit(const Node& nd, const Ray<T>& r, T tmax) {
    double t0 = double(r.tmin), t1 = double(tmax);
    for (int a = 0; a < 3; ++a) {
        double o = double(r.o[a]), d = double(r.d[a]);
        double lo = double(nd.lo[a]) - 1e-6 * (1.0 + std::fabs(nd.lo[a]));
        double hi = double(nd.hi[a]) + 1e-6 * (1.0 + std::fabs(nd.hi[a]));
        if (d == 0.0) {
            if (o < lo || o > hi) return false;
            continue;
        }
        double ta = (lo - o) / d, tb = (hi - o) / d;
        if (ta > tb) std::swap(ta, tb);
        t0 = std::max(t0, ta);
        t1 = std::min(t1, tb);
        if (t1 < t0) return false;
    }
    return true;
}

// BVHBackend::makeRay4 + intersectTriangle (BVHBackend.cpp:233-247, 264-283)
template <class T>
bool tri_hit(const Tri<T>& tr, const Ray<T>& r, T tmax, T& t, T& u, T& v) {
    auto safe = [](T x) { return std::abs(x) > T(1e-9f) ? x : T(1e-9f); };
    V3<T> inv(T(1) / safe(r.d.x), T(1) / safe(r.d.y), T(1) / safe(r.d.z));
    V3<T> dir(T(1) / inv.x, T(1) / inv.y, T(1) / inv.z);
    V3<T> h = cross(dir, tr.e2);
    T a = dot(tr.e1, h);
    if (std::abs(a) < T(1e-9f)) return false;
    T f = T(1) / a;
    V3<T> s = r.o - tr.v0;
    u = f * dot(s, h);
    if (u < T(0) || u > T(1)) return false;
    V3<T> q = cross(s, tr.e1);
    v = f * dot(dir, q);
    if (v < T(0) || u + v > T(1)) return false;
    t = f * dot(tr.e2, q);
    return t >= r.tmin && t <= tmax;
}

// ---- ray-ribbon (CurveBrute.cpp:29-234) -------------------------------------
template <class T>
struct Frame {
    V3<T> o, x, y, z;
    V3<T> project(V3<T> p) const {
        V3<T> q = p - o;
        return {dot(q, x), dot(q, y), dot(q, z)};
    }
};

template <class T>
V3<T> bezierTangent(V3<T> P0, V3<T> P1, V3<T> P2, V3<T> P3, T t) {
    T mt = T(1) - t;
    return (P1 - P0) * (T(3) * mt * mt) + (P2 - P1) * (T(6) * mt * t) + (P3 - P2) * (T(3) * t * t);
}

template <class T>
bool subdivide(const Frame<T>& f, V3<T> P0, V3<T> P1, V3<T> P2, V3<T> P3, T hw0, T hw3, T tOff, T tScale,
               T tmin, T& best, int depth, T& outTSeg, V3<T>& outTang) {
    V3<T> c0 = f.project(P0), c1 = f.project(P1), c2 = f.project(P2), c3 = f.project(P3);
    T maxHalfW = std::max(hw0, hw3);
    T zMin = std::min({c0.z, c1.z, c2.z, c3.z}), zMax = std::max({c0.z, c1.z, c2.z, c3.z});
    if (zMin - maxHalfW > best) return false;
    if (zMax + maxHalfW < tmin) return false;
    T xMin = std::min({c0.x, c1.x, c2.x, c3.x}), xMax = std::max({c0.x, c1.x, c2.x, c3.x});
    T yMin = std::min({c0.y, c1.y, c2.y, c3.y}), yMax = std::max({c0.y, c1.y, c2.y, c3.y});
    T cx = (T(0) < xMin) ? xMin : (T(0) > xMax ? xMax : T(0));
    T cy = (T(0) < yMin) ? yMin : (T(0) > yMax ? yMax : T(0));
    if (cx * cx + cy * cy > maxHalfW * maxHalfW) return false;
    if (depth == 0) {
        T ax = c0.x, ay = c0.y, bx = c3.x, by = c3.y;
        T dx = bx - ax, dy = by - ay;
        T lenSq = dx * dx + dy * dy;
        T tl = lenSq < T(1e-12f) ? T(0) : std::max(T(0), std::min(T(1), (-ax * dx - ay * dy) / lenSq));
        T px = ax + dx * tl, py = ay + dy * tl;
        T dist2 = px * px + py * py;
        T hw = hw0 * (T(1) - tl) + hw3 * tl;
        if (dist2 > hw * hw) return false;
        T tRay = c0.z + (c3.z - c0.z) * tl;
        if (tRay < tmin || tRay >= best) return false;
        V3<T> tg = bezierTangent(P0, P1, P2, P3, tl);
        if (tg.lengthSq() < T(1e-12f)) tg = P3 - P0;
        tg = safeNormalize(tg);
        best = tRay;
        outTSeg = tOff + tl * tScale;
        outTang = tg;
        return true;
    }
    V3<T> h = V3<T>(T(0.5f), T(0.5f), T(0.5f));
    V3<T> Q01 = (P0 + P1) * T(0.5f), Q12 = (P1 + P2) * T(0.5f), Q23 = (P2 + P3) * T(0.5f);
    V3<T> R01 = (Q01 + Q12) * T(0.5f), R12 = (Q12 + Q23) * T(0.5f), M = (R01 + R12) * T(0.5f);
    (void)h;
    T hwm = (hw0 + hw3) * T(0.5f), tsh = tScale * T(0.5f);
    bool hit = false;
    T ts;
    V3<T> tg;
    if (subdivide(f, P0, Q01, R01, M, hw0, hwm, tOff, tsh, tmin, best, depth - 1, ts, tg)) {
        outTSeg = ts;
        outTang = tg;
        hit = true;
    }
    if (subdivide(f, M, R12, Q23, P3, hwm, hw3, tOff + tsh, tsh, tmin, best, depth - 1, ts, tg)) {
        outTSeg = ts;
        outTang = tg;
        hit = true;
    }
    return hit;
}

// CurveBrute::trace (CurveBrute.cpp:398-440): triangles first, then strictly
// closer ribbon hits.
template <class T>
Hit<T> trace(const Scene<T>& S, const Ray<T>& r, bool any = false) {
    Hit<T> h;
    T closest = r.tmax;
    if (!S.triNodes.empty()) {
        uint32_t st[128];
        int sp = 0;
        st[sp++] = 0;
        while (sp) {
            const Node& nd = S.triNodes[st[--sp]];
            if (!node_hit(nd, r, closest)) continue;
            if (nd.count) {
                for (uint32_t i = nd.start; i < nd.start + nd.count; ++i) {
                    T t, u, v;
                    const Tri<T>& tr = S.tris[S.triIdx[i]];
                    bool ok;
                    if (tr.objectSpace) {  // BVHBackend.cpp:356-367
                        M4<T> w2o = interpO2W(S.motion[tr.mesh], r.time).inverse();
                        Ray<T> ro;
                        ro.o = w2o.point(r.o);
                        ro.d = w2o.vector(r.d);
                        ro.tmin = r.tmin;
                        ok = tri_hit(tr, ro, closest, t, u, v);
                    } else {
                        ok = tri_hit(tr, r, closest, t, u, v);
                    }
                    if (ok) {
                        closest = t;
                        h.hit = true;
                        h.t = t;
                        h.u = u;
                        h.v = v;
                        h.curve = false;
                        h.idx = S.triIdx[i];
                        if (any) return h;
                    }
                }
            } else {
                st[sp++] = nd.right;
                st[sp++] = nd.left;
            }
        }
    }
    if (!S.segNodes.empty()) {
        Frame<T> f;
        f.o = r.o;
        f.z = r.d;
        onb(f.z, f.x, f.y);
        T best = h.hit ? h.t : r.tmax;
        uint32_t st[128];
        int sp = 0;
        st[sp++] = 0;
        while (sp) {
            const Node& nd = S.segNodes[st[--sp]];
            if (!node_hit(nd, r, best)) continue;
            if (nd.count) {
                for (uint32_t i = nd.start; i < nd.start + nd.count; ++i) {
                    const Seg<T>& s = S.segs[S.segIdx[i]];
                    T ts;
                    V3<T> tg;
                    if (subdivide(f, s.P[0], s.P[1], s.P[2], s.P[3], s.hw0, s.hw3, s.v0, s.dv, r.tmin, best, 6, ts,
                                  tg)) {
                        h.hit = true;
                        h.curve = true;
                        h.t = best;
                        h.idx = S.segIdx[i];
                        h.tang = tg;
                        h.tseg = ts;
                        if (any) return h;
                    }
                }
            } else {
                st[sp++] = nd.right;
                st[sp++] = nd.left;
            }
        }
    }
    return h;
}

// SurfaceInteraction + ShadingContext (ShadingContext.h:28-59)
template <class T>
struct SI {
    V3<T> p, n, ng, dpdu, color{1, 1, 1};
    uint32_t slot = 0, mesh = 0, prim = 0, strand = ~0u;
    bool curve = false;
};

template <class T>
SI<T> surface(const Scene<T>& S, const Ray<T>& r, const Hit<T>& h) {
    SI<T> si;
    if (!h.curve) {  // fillSurfaceInteraction (BVHBackend.cpp:285-317)
        const Tri<T>& tr = S.tris[h.idx];
        T w = T(1) - h.u - h.v;
        if (tr.objectSpace) {  // the object-space triangle taken to the world at the ray's time
            M4<T> o2w = interpO2W(S.motion[tr.mesh], r.time);
            V3<T> pObj = tr.v0 + tr.e1 * h.u + tr.e2 * h.v;
            V3<T> nObj = safeNormalize(cross(tr.e1, tr.e2));
            V3<T> snObj = safeNormalize(tr.sn0 * w + tr.sn1 * h.u + tr.sn2 * h.v);
            si.p = o2w.point(pObj);
            si.ng = safeNormalize(o2w.normal(nObj));
            si.n = safeNormalize(o2w.normal(snObj));
            si.dpdu = o2w.vector(tr.e1);
        } else {
            si.p = tr.v0 + tr.e1 * h.u + tr.e2 * h.v;
            si.ng = tr.n;
            si.n = safeNormalize(tr.sn0 * w + tr.sn1 * h.u + tr.sn2 * h.v);
            si.dpdu = tr.e1;
        }
        if (dot(si.n, si.ng) < T(0)) si.n = -si.n;
        si.slot = tr.mesh;
        si.mesh = tr.mesh;
        si.prim = tr.prim;
    } else {  // intersectOneSegment (CurveBrute.cpp:209-233)
        const Seg<T>& s = S.segs[h.idx];
        Frame<T> f;
        f.z = r.d;
        onb(f.z, f.x, f.y);
        si.p = r.o + r.d * h.t;
        V3<T> nd = -r.d;
        V3<T> nrm = nd - h.tang * dot(nd, h.tang);
        nrm = safeNormalize(nrm, f.x);
        si.n = si.ng = nrm;
        si.dpdu = h.tang;
        si.slot = s.slot;
        si.mesh = s.slot;
        si.prim = s.seg;
        si.strand = s.strand;
        si.curve = true;
        si.color = S.strandColor[s.strand];
    }
    return si;
}

template <class T>
struct Ctx {
    V3<T> p, n, ng, t, bt, color;
    bool front;
    Ctx(const SI<T>& si, V3<T> rd) {
        p = si.p;
        color = si.color;
        front = dot(-rd, si.ng) > T(0);
        n = front ? si.n : -si.n;
        ng = front ? si.ng : -si.ng;
        if (si.curve) {
            t = si.dpdu;
            bt = safeNormalize(cross(n, t));
        } else {
            onb(n, t, bt);
        }
    }
    V3<T> toLocal(V3<T> v) const { return {dot(v, t), dot(v, bt), dot(v, n)}; }
    V3<T> toWorld(V3<T> v) const { return t * v.x + bt * v.y + n * v.z; }
};

template <class T>
struct BS {
    V3<T> f, wi;
    T pdf = 0;
    uint32_t flags = 0;
    bool valid() const { return pdf > T(0) && !f.black(); }
    bool delta() const { return (flags & 4u) != 0; }
};
template <class T>
struct BE {
    V3<T> f;
    T pdf = 0;
};

// ---- GGX helpers (StandardSurface.h:20-76) --------------------------------
template <class T> T D_GGX(T c, T a2) {
    if (c <= T(0)) return T(0);
    T d = c * c * (a2 - T(1)) + T(1);
    return a2 / (kPi<T> * d * d);
}
template <class T> T G1(T ac, T a2) {
    if (ac <= T(0)) return T(0);
    T c2 = ac * ac;
    return T(2) * ac / (ac + std::sqrt(a2 + (T(1) - a2) * c2));
}
template <class T> T G2(T co, T ci, T a2) { return G1(std::abs(co), a2) * G1(std::abs(ci), a2); }
template <class T> V3<T> sampleH(T ux, T uy, T a2) {
    T phi = T(2) * kPi<T> * ux;
    T ch2 = (T(1) - uy) / std::max(T(1) + (a2 - T(1)) * uy, T(1e-10f));
    T ch = std::sqrt(std::max(T(0), ch2));
    T sh = std::sqrt(std::max(T(0), T(1) - ch2));
    return {sh * std::cos(phi), sh * std::sin(phi), ch};
}
template <class T> T pdfRefl(T ch, T a2, T dvh) {
    if (ch <= T(0) || dvh <= T(0)) return T(0);
    return D_GGX(ch, a2) * ch / (T(4) * dvh);
}
template <class T> T schlickD(T c, T f0) {
    T x = T(1) - std::abs(c);
    T x5 = x * x * x * x * x;
    return f0 + (T(1) - f0) * x5;
}
template <class T> V3<T> schlickC(T c, V3<T> f0) {
    T x = T(1) - std::abs(c);
    T x5 = x * x * x * x * x;
    return f0 + (V3<T>(1, 1, 1) - f0) * x5;
}
template <class T> T fresnel(T ci, T eta) {
    T s2i = std::max(T(0), T(1) - ci * ci);
    T s2t = s2i / (eta * eta);
    if (s2t >= T(1)) return T(1);
    T ct = std::sqrt(T(1) - s2t);
    T rs = (ci - eta * ct) / (ci + eta * ct);
    T rp = (eta * ci - ct) / (eta * ci + ct);
    return T(0.5f) * (rs * rs + rp * rp);
}

template <class T>
struct W4 {
    T c, m, s, d;
};

template <class T>
bool ssWeights(const Mat<T>& m, T cosO, W4<T>& w) {  // StandardSurface.h:355-371
    T coatF = schlickD(cosO, m.coatF0);
    T specF = schlickD(cosO, m.f0);
    w.c = m.coat * coatF;
    w.m = m.metal * (T(1) - w.c);
    w.s = m.spec * (T(1) - m.metal) * specF * (T(1) - w.c);
    w.d = m.base * (T(1) - m.metal) * (T(1) - m.spec * specF) * (T(1) - w.c);
    T sum = w.c + w.m + w.s + w.d;
    if (sum <= T(0)) return false;
    T inv = T(1) / sum;
    w.c *= inv;
    w.m *= inv;
    w.s *= inv;
    w.d *= inv;
    return true;
}

template <class T>
V3<T> evalGGX(V3<T> wo, V3<T> wi, T a2, V3<T> F0, T& pdf) {  // StandardSurface.h:578-603
    pdf = 0;
    if (wo.z <= T(0) || wi.z <= T(0)) return {};
    V3<T> wh = safeNormalize(wo + wi);
    if (wh.z <= T(0)) return {};
    T dvh = std::max(T(0), dot(wo, wh));
    V3<T> F = schlickC(dvh, F0);
    T D = D_GGX(wh.z, a2), G = G2(wo.z, wi.z, a2);
    T co = std::abs(wo.z), ci = std::abs(wi.z);
    if (co < T(1e-6f) || ci < T(1e-6f)) return {};
    V3<T> b = F * (D * G / (T(4) * co * ci));
    pdf = pdfRefl(wh.z, a2, dvh);
    return b;
}

template <class T>
V3<T> ssCombined(const Mat<T>& m, V3<T> wo, V3<T> wi, const W4<T>& w, T& pdf) {  // :608-661
    V3<T> f;
    pdf = 0;
    if (!(wo.z * wi.z > T(0))) return f;
    if (w.c > T(0)) {
        T p;
        f = f + evalGGX(wo, wi, m.coatAlpha2, V3<T>(m.coatF0, m.coatF0, m.coatF0), p) * w.c;
        pdf += p * w.c;
    }
    T a = std::max(T(1e-4f), m.rough * m.rough), a2 = a * a;
    if (w.m > T(0)) {
        T p;
        f = f + evalGGX(wo, wi, a2, m.albedo * m.base, p) * w.m;
        pdf += p * w.m;
    }
    if (w.s > T(0)) {
        T p;
        f = f + evalGGX(wo, wi, a2, m.specColor * (m.spec * m.f0), p) * w.s;
        pdf += p * w.s;
    }
    if (w.d > T(0)) {
        T ci = std::abs(wi.z);
        f = f + m.albedo * m.base * kInvPi<T> * w.d;
        pdf += ci * kInvPi<T> * w.d;
    }
    return f;
}

template <class T>
bool ssSampleGGX(V3<T> wo, T ux, T uy, T a2, V3<T> F0, V3<T>& wi) {  // :516-549
    V3<T> wh = sampleH(ux, uy, a2);
    if (wh.z <= T(0)) return false;
    T dvh = dot(wo, wh);
    if (dvh <= T(0)) return false;
    wi = wh * (T(2) * dvh) - wo;
    if (wi.z <= T(0)) return false;
    V3<T> F = schlickC(dvh, F0);
    T D = D_GGX(wh.z, a2), G = G2(wo.z, wi.z, a2);
    T co = std::abs(wo.z), ci = std::abs(wi.z);
    if (co < T(1e-6f) || ci < T(1e-6f)) return false;
    V3<T> f = F * (D * G / (T(4) * co)) * ci;
    return pdfRefl(wh.z, a2, dvh) > T(0) && !f.black();
}

// Dielectric glass sampling (StandardSurface.h:245-340): smooth (delta) Fresnel
// reflection / Snell refraction, or a GGX half-vector then Fresnel reflection
// / Walter transmission with importance transport.
template <class T>
BS<T> glassSample(const Mat<T>& m, const Ctx<T>& c, V3<T> wol, T ux, T uy, T uc) {
    T eta = c.front ? m.ior : (T(1) / m.ior);
    T cosI = wol.z;
    BS<T> s;
    if (m.rough < T(0.001f)) {
        T Fr = fresnel(cosI, eta);
        if (uc < Fr) {
            s.wi = c.toWorld(V3<T>(-wol.x, -wol.y, wol.z));
            s.f = m.albedo * Fr;
            s.pdf = Fr;
            s.flags = 4u | 16u;
        } else {
            T sin2T = std::max(T(0), T(1) - cosI * cosI) / (eta * eta);
            T cosT = std::sqrt(std::max(T(0), T(1) - sin2T));
            s.wi = c.toWorld(V3<T>(-wol.x / eta, -wol.y / eta, -cosT));
            s.f = m.albedo * (T(1) - Fr);
            s.pdf = T(1) - Fr;
            s.flags = 4u | 8u;
        }
        return s;
    }
    T alpha = std::max(T(1e-4f), m.rough * m.rough);
    T alpha2 = alpha * alpha;
    V3<T> wh = sampleH(ux, uy, alpha2);
    if (wh.z <= T(0)) return {};
    T cosIH = std::max(T(0), dot(wol, wh));
    if (cosIH <= T(0)) return {};
    T Fr = fresnel(cosIH, eta);
    if (uc < Fr) {
        V3<T> wil = wh * (T(2) * cosIH) - wol;
        if (wil.z <= T(0)) return {};
        T D = D_GGX(wh.z, alpha2);
        T G = G2(wol.z, wil.z, alpha2);
        T cosO = wol.z;
        V3<T> bsdf = V3<T>(Fr, Fr, Fr) * (D * G / (T(4) * cosO));
        s.wi = c.toWorld(wil);
        s.f = bsdf * m.albedo;
        s.pdf = Fr * pdfRefl(wh.z, alpha2, cosIH);
        s.flags = 2u | 16u;
        return s;
    }
    T sin2T = std::max(T(0), T(1) - cosIH * cosIH) / (eta * eta);
    if (sin2T >= T(1)) return {};
    T cosTH = std::sqrt(T(1) - sin2T);
    V3<T> wil = wol * (T(-1) / eta) + wh * (cosIH / eta - cosTH);
    if (wil.z >= T(0)) return {};
    T cosO = wol.z, cosIt = std::abs(wil.z);
    T D = D_GGX(wh.z, alpha2);
    T G = G2(cosO, cosIt, alpha2);
    T denom = cosIH + eta * std::abs(dot(wil, wh));
    if (denom < T(1e-6f)) return {};
    T absCosTwh = std::abs(dot(wil, wh));
    T pdfWh = D * wh.z;
    T jac = eta * eta * absCosTwh / (denom * denom);
    s.wi = c.toWorld(wil);
    s.f = m.albedo * ((T(1) - Fr) * D * G * cosIH * absCosTwh / (cosO * denom * denom));
    s.pdf = (T(1) - Fr) * pdfWh * jac;
    s.flags = 2u | 8u;
    return s;
}

template <class T>
BS<T> ssSample(const Mat<T>& m, const Ctx<T>& c, V3<T> wo, T ux, T uy, T uc) {  // :231-405
    V3<T> wol = c.toLocal(wo);
    if (wol.z <= T(0)) return {};
    if (m.transmission > T(0.001f) && m.metal < T(0.001f)) return glassSample(m, c, wol, ux, uy, uc);
    W4<T> w;
    if (!ssWeights(m, wol.z, w)) return {};
    T a = std::max(T(1e-4f), m.rough * m.rough), a2 = a * a;
    V3<T> wil;
    bool ok;
    if (uc < w.c) ok = ssSampleGGX(wol, ux, uy, m.coatAlpha2, V3<T>(m.coatF0, m.coatF0, m.coatF0), wil);
    else if (uc < w.c + w.m) ok = ssSampleGGX(wol, ux, uy, a2, m.albedo * m.base, wil);
    else if (uc < w.c + w.m + w.s) ok = ssSampleGGX(wol, ux, uy, a2, m.specColor * (m.spec * m.f0), wil);
    else {  // sampleDiffuse :554-573
        T phi = T(2) * kPi<T> * ux, r = std::sqrt(uy), z = std::sqrt(std::max(T(0), T(1) - uy));
        wil = V3<T>(r * std::cos(phi), r * std::sin(phi), z);
        if (wol.z < T(0)) wil.z = -wil.z;
        T ci = std::abs(wil.z);
        V3<T> f = m.albedo * m.base * (kInvPi<T> * ci);
        ok = ci * kInvPi<T> > T(0) && !f.black();
    }
    if (!ok) return {};
    BS<T> s;
    s.wi = c.toWorld(wil);
    V3<T> wl2 = c.toLocal(s.wi);
    T pdf;
    V3<T> fc = ssCombined(m, wol, wl2, w, pdf);
    s.f = fc * std::abs(wl2.z);
    s.pdf = pdf;
    s.flags = m.flags;
    return s;
}

template <class T>
BE<T> ssEval(const Mat<T>& m, const Ctx<T>& c, V3<T> wo, V3<T> wi) {  // :410-504
    V3<T> wol = c.toLocal(wo), wil = c.toLocal(wi);
    BE<T> e;
    if (!(wol.z * wil.z > T(0))) {
        // rough dielectric transmission (StandardSurface.h:414-442): its alpha
        // is rough^4 without the 1e-4 clamp
        if (m.transmission < T(0.001f) || m.rough < T(0.001f) || m.metal > T(0.001f)) return e;
        T eta = c.front ? m.ior : (T(1) / m.ior);
        T alpha2 = m.rough * m.rough;
        alpha2 *= alpha2;
        V3<T> wh = safeNormalize(wol + wil * eta);
        if (wh.z < T(0)) wh = -wh;
        T cosIH = std::max(T(0), dot(wol, wh));
        T cosTH = std::abs(dot(wil, wh));
        T Fr = fresnel(cosIH, eta);
        T D = D_GGX(wh.z, alpha2);
        T G = G2(wol.z, std::abs(wil.z), alpha2);
        T denom = cosIH + eta * cosTH;
        if (denom < T(1e-6f)) return e;
        T bs = (T(1) - Fr) * D * G * cosIH * cosTH / (wol.z * std::abs(wil.z) * denom * denom);
        T jac = eta * eta * cosTH / (denom * denom);
        e.f = m.albedo * bs;
        e.pdf = (T(1) - Fr) * D * wh.z * jac;
        return e;
    }
    if (m.transmission > T(0.001f) && m.metal < T(0.001f)) {  // glass reflection (:455-473)
        if (m.rough < T(0.001f)) return e;
        T alpha = std::max(T(1e-4f), m.rough * m.rough);
        T alpha2 = alpha * alpha;
        T eta = c.front ? m.ior : (T(1) / m.ior);
        V3<T> wh = safeNormalize(wol + wil);
        if (wh.z < T(0)) return e;
        T cosIH = std::max(T(0), dot(wol, wh));
        T Fr = fresnel(cosIH, eta);
        T D = D_GGX(wh.z, alpha2);
        T G = G2(wol.z, wil.z, alpha2);
        T pdf = Fr > T(0) ? Fr * pdfRefl(wh.z, alpha2, cosIH) : T(0);
        e.f = m.albedo * (Fr * D * G / (T(4) * wol.z * wil.z));
        e.pdf = pdf;
        return e;
    }
    W4<T> w;
    if (!ssWeights(m, wol.z, w)) return e;
    e.f = ssCombined(m, wol, wil, w, e.pdf);
    return e;
}

// ---- hair (MarschnerHair.h) ---------------------------------------------------
template <class T> V3<T> hairSigma(const Mat<T>& m, V3<T> c) {  // :430-450
    if (c.x > T(0.98f) && c.y > T(0.98f) && c.z > T(0.98f)) return m.sigma;
    auto lin = [](T s) { return std::pow(std::max(s, T(0)), T(2.2f)); };
    T lr = lin(c.x), lg = lin(c.y), lb = lin(c.z);
    if (lr < T(0.01f) && lg < T(0.01f) && lb < T(0.01f)) return m.sigma;
    return {-std::log(std::max(lr, T(0.001f))), -std::log(std::max(lg, T(0.001f))),
            -std::log(std::max(lb, T(0.001f)))};
}
template <class T> BE<T> kkEval(const Mat<T>& m, const Ctx<T>& c, V3<T> wo, V3<T> wi) {  // :395-422
    V3<T> sa = hairSigma(m, c.color);
    V3<T> alb(std::exp(-sa.x), std::exp(-sa.y), std::exp(-sa.z));
    T dTL = dot(c.t, wi), dTV = dot(c.t, wo);
    T sTL = std::sqrt(std::max(T(0), T(1) - dTL * dTL)), sTV = std::sqrt(std::max(T(0), T(1) - dTV * dTV));
    V3<T> f = alb * kInvPi<T>;
    T sp = dTL * dTV + sTL * sTV;
    if (sp > T(0)) f = f + V3<T>(T(0.15f), T(0.15f), T(0.15f)) * (std::pow(sp, T(20)) * kInvPi<T>);
    BE<T> e;
    e.f = f;
    e.pdf = std::max(T(0), dot(wi, c.n)) * kInvPi<T>;
    return e;
}
template <class T> BS<T> kkSample(const Mat<T>& m, const Ctx<T>& c, V3<T> wo, T ux, T uy) {  // :267-282
    V3<T> t, b;
    onb(c.n, t, b);
    T phi = k2Pi<T> * ux, cT = std::sqrt(uy), sT = std::sqrt(T(1) - uy);
    V3<T> wi = safeNormalize(t * (sT * std::cos(phi)) + b * (sT * std::sin(phi)) + c.n * cT);
    BE<T> ev = kkEval(m, c, wo, wi);
    BS<T> s;
    s.wi = wi;
    s.f = ev.f * cT;
    s.pdf = cT * kInvPi<T>;
    s.flags = 1u | 16u;
    return s;
}
// Marschner lobes (MarschnerHair.h:49-185, 284-375, 457-556)
template <class T> T mhI0(T x) {
    T sum = 0, x2i = 1, den = 1;
    for (int i = 0; i < 12; ++i) {
        if (i > 0) {
            x2i *= x * x;
            den *= T(i) * T(i) * T(4);
        }
        sum += x2i / den;
    }
    return sum;
}
template <class T> T mhLogI0(T x) {
    if (x > T(12)) return x + T(0.5f) * (-std::log(k2Pi<T>) + std::log(T(1) / x) + T(1) / (T(8) * x));
    return std::log(mhI0(x));
}
template <class T> T mhMp(T cI, T sI, T cR, T sR, T v) {
    if (v < T(1e-5f)) v = T(1e-5f);
    T a = cI * cR / v, b = sI * sR / v;
    if (v <= T(0.1f)) return std::exp(mhLogI0(a) - b - T(1) / v + T(0.6931472f) + std::log(T(0.5f) / v));
    return std::exp(-b) * mhI0(a) / (T(2) * v * std::sinh(T(1) / v));
}
template <class T> T mhLog(T x, T s) {
    T ex = std::exp(-std::abs(x) / s);
    return ex / (s * (T(1) + ex) * (T(1) + ex));
}
template <class T> T mhCdf(T x, T s) { return T(1) / (T(1) + std::exp(-x / s)); }
template <class T> T mhTrim(T x, T s) { return mhLog(x, s) / (mhCdf(kPi<T>, s) - mhCdf(-kPi<T>, s)); }
template <class T> T mhSampleTrim(T u, T s) {
    T a = mhCdf(-kPi<T>, s), b = mhCdf(kPi<T>, s);
    T x = -s * std::log(T(1) / (a + u * (b - a)) - T(1));
    return std::clamp(x, -kPi<T>, kPi<T>);
}
template <class T> T mhPhi(int p, T gO, T gT) { return T(2) * T(p) * gT - T(2) * gO + T(p) * kPi<T>; }
template <class T> T mhWrap(T x) {
    while (x > kPi<T>) x -= k2Pi<T>;
    while (x < -kPi<T>) x += k2Pi<T>;
    return x;
}
template <class T> void mhAp(T cO, T eta, T h, V3<T> sa, V3<T> ap[3]) {
    T s2 = std::max(T(0), T(1) - cO * cO);
    T etaP = std::sqrt(std::max(T(0), eta * eta - s2)) / cO;
    T sGT = std::clamp(h / (etaP > T(1e-5f) ? etaP : T(1e-5f)), T(-1) + T(1e-5f), T(1) - T(1e-5f));
    T cGT = std::sqrt(std::max(T(0), T(1) - sGT * sGT));
    V3<T> Tt(std::exp(-sa.x * T(2) * cGT), std::exp(-sa.y * T(2) * cGT), std::exp(-sa.z * T(2) * cGT));
    T cGO = std::sqrt(std::max(T(0), T(1) - h * h));
    T fr = fresnel(std::max(T(0), cO * cGO), eta);
    ap[0] = V3<T>(fr, fr, fr);
    ap[1] = Tt * ((T(1) - fr) * (T(1) - fr));
    ap[2] = ap[1] * Tt * fr;
}
template <class T> void hairLong(V3<T> d, V3<T> t, T& s, T& c) {
    s = dot(d, t);
    c = std::sqrt(std::max(T(0), T(1) - s * s));
}
template <class T> T hairPhiF(V3<T> wo, V3<T> wi, V3<T> t, T sO, T sI) {
    V3<T> op = wo - t * sO, ip = wi - t * sI;
    T lo = op.length(), li = ip.length();
    if (lo < T(1e-5f) || li < T(1e-5f)) return T(0);
    op = op * (T(1) / lo);
    ip = ip * (T(1) / li);
    T c = std::clamp(dot(op, ip), T(-1), T(1));
    T s = dot(cross(ip, op), t);
    return std::atan2(s, c);
}
template <class T> T hairH(V3<T> wo, V3<T> t, V3<T> n, T sO) {
    V3<T> op = wo - t * sO;
    T lp = op.length();
    if (lp < T(1e-5f)) return T(0);
    return std::clamp(dot(op * (T(1) / lp), n), T(-1) + T(1e-5f), T(1) - T(1e-5f));
}
template <class T> void mhGammas(const Mat<T>& m, T cO, T h, T& gO, T& gT) {
    T s2 = T(1) - cO * cO;
    T etaP = std::sqrt(std::max(T(0), m.eta * m.eta - s2)) / cO;
    gO = std::asin(std::clamp(h, T(-1) + T(1e-5f), T(1) - T(1e-5f)));
    gT = std::asin(std::clamp(h / (etaP > T(1e-5f) ? etaP : T(1e-5f)), T(-1) + T(1e-5f), T(1) - T(1e-5f)));
}
template <class T> V3<T> mhLobes(const Mat<T>& m, T sO, T cO, T sI, T cI, T phi, T h, V3<T> sa) {
    T cD = std::sqrt(std::max(T(0), T(0.5f) * (T(1) + cO * cI + sO * sI)));
    T den = std::max(T(0.25f), cD * cD);
    T gO, gT;
    mhGammas(m, cO, h, gO, gT);
    V3<T> ap[3];
    mhAp(cO, m.eta, h, sa, ap);
    V3<T> fs;
    for (int p = 0; p < 3; ++p) {
        T sOs = sO * std::cos(T(2) * m.ashift[p]) + cO * std::sin(T(2) * m.ashift[p]);
        T cOs = std::sqrt(std::max(T(0), T(1) - sOs * sOs));
        fs = fs + ap[p] * (mhMp(cI, sI, cOs, sOs, m.v[p]) * mhTrim(mhWrap(phi - mhPhi(p, gO, gT)), m.s));
    }
    return fs * (T(1) / den);
}
template <class T> T mhPdf(const Mat<T>& m, T sO, T cO, T sI, T cI, T phi, T h, V3<T> sa) {
    T gO, gT;
    mhGammas(m, cO, h, gO, gT);
    V3<T> ap[3];
    mhAp(cO, m.eta, h, sa, ap);
    T w[3] = {luminance(ap[0]), luminance(ap[1]), luminance(ap[2])};
    T tot = w[0] + w[1] + w[2];
    if (tot < T(1e-8f)) return T(0);
    T pdf = 0;
    for (int p = 0; p < 3; ++p) {
        T sOs = sO * std::cos(T(2) * m.ashift[p]) + cO * std::sin(T(2) * m.ashift[p]);
        T cOs = std::sqrt(std::max(T(0), T(1) - sOs * sOs));
        pdf += (w[p] / tot) * (mhMp(cI, sI, cOs, sOs, m.v[p]) * cI) *
               mhTrim(mhWrap(phi - mhPhi(p, gO, gT)), m.s);
    }
    return std::max(T(0), pdf);
}
template <class T> BE<T> msEval(const Mat<T>& m, const Ctx<T>& c, V3<T> wo, V3<T> wi) {
    T sO, cO, sI, cI;
    hairLong(wo, c.t, sO, cO);
    hairLong(wi, c.t, sI, cI);
    T phi = hairPhiF(wo, wi, c.t, sO, sI), h = hairH(wo, c.t, c.n, sO);
    V3<T> sa = hairSigma(m, c.color);
    BE<T> e;
    e.f = mhLobes(m, sO, cO, sI, cI, phi, h, sa);
    e.pdf = mhPdf(m, sO, cO, sI, cI, phi, h, sa);
    return e;
}
template <class T> BS<T> msSample(const Mat<T>& m, const Ctx<T>& c, V3<T> wo, T ux, T uy, T uc) {
    T sO, cO;
    hairLong(wo, c.t, sO, cO);
    T h = hairH(wo, c.t, c.n, sO);
    V3<T> sa = hairSigma(m, c.color);
    V3<T> ap[3];
    mhAp(cO, m.eta, h, sa, ap);
    T w[3] = {luminance(ap[0]), luminance(ap[1]), luminance(ap[2])};
    T tot = w[0] + w[1] + w[2];
    if (tot < T(1e-8f)) return {};
    T inv = T(1) / tot, c0 = w[0] * inv, c1 = c0 + w[1] * inv, c2 = T(1);
    int lobe = 0;
    T ur = uc;
    if (uc < c0) ur = uc / c0;
    else if (uc < c1) { lobe = 1; ur = (uc - c0) / (c1 - c0); }
    else { lobe = 2; ur = (uc - c1) / (c2 - c1); }
    T thO = std::asin(std::clamp(sO, T(-1) + T(1e-5f), T(1) - T(1e-5f)));
    T z = std::sqrt(T(-2) * std::log(std::max(ux, T(1e-6f)))) * std::cos(k2Pi<T> * uy);
    T thI = std::clamp(thO + m.ashift[lobe] + z * std::sqrt(m.v[lobe]), -kPi<T> * T(0.5f), kPi<T> * T(0.5f));
    T sI = std::sin(thI), cI = std::cos(thI);
    T gO, gT;
    mhGammas(m, cO, h, gO, gT);
    T phiS = mhSampleTrim(ur, m.s) + mhPhi(lobe, gO, gT);
    V3<T> wop = safeNormalize(wo - c.t * sO);
    if (wop.lengthSq() < T(1e-8f)) {
        V3<T> d;
        onb(c.t, wop, d);
    }
    V3<T> ctp = cross(c.t, wop);
    V3<T> wi = safeNormalize(c.t * sI + wop * (cI * std::cos(phiS)) + ctp * (cI * std::sin(phiS)));
    T sIa, cIa;
    hairLong(wi, c.t, sIa, cIa);
    T phA = hairPhiF(wo, wi, c.t, sO, sIa);
    V3<T> f = mhLobes(m, sO, cO, sIa, cIa, phA, h, sa);
    T pd = mhPdf(m, sO, cO, sIa, cIa, phA, h, sa);
    if (pd < T(1e-8f)) return {};
    BS<T> s;
    s.wi = wi;
    s.f = f * std::abs(dot(wi, c.n));
    s.pdf = pd;
    s.flags = 2u | 16u | 8u;
    return s;
}

// ---- Lambert (Lambertian.h:12-82) ------------------------------------------------
template <class T> BS<T> lamSample(const Mat<T>& m, const Ctx<T>& c, V3<T> wo, T ux, T uy) {
    T r = std::sqrt(ux), phi = T(2) * kPi<T> * uy;
    V3<T> wl(r * std::cos(phi), r * std::sin(phi), std::sqrt(std::max(T(0), T(1) - ux)));
    if (c.toLocal(wo).z < T(0)) wl.z = -wl.z;
    BS<T> s;
    s.wi = c.toWorld(wl);
    s.pdf = std::max(T(0), std::abs(wl.z)) * kInvPi<T>;
    s.f = m.albedo * (kInvPi<T> * std::abs(wl.z));
    s.flags = 1u | 16u;
    return s;
}
template <class T> BE<T> lamEval(const Mat<T>& m, const Ctx<T>& c, V3<T> wo, V3<T> wi) {
    V3<T> wil = c.toLocal(wi), wol = c.toLocal(wo);
    BE<T> e;
    if (!(wil.z * wol.z > T(0))) return e;
    e.f = m.albedo * kInvPi<T>;
    e.pdf = std::max(T(0), std::abs(wil.z)) * kInvPi<T>;
    return e;
}

template <class T> BS<T> matSample(const Mat<T>& m, const Ctx<T>& c, V3<T> wo, T ux, T uy, T uc) {
    if (m.type == MAT_LAMBERT || m.type == MAT_EMISSIVE) return lamSample(m, c, wo, ux, uy);
    if (m.type == MAT_STANDARD) return ssSample(m, c, wo, ux, uy, uc);
    return m.hairMode == 1 ? msSample(m, c, wo, ux, uy, uc) : kkSample(m, c, wo, ux, uy);
}
template <class T> BE<T> matEval(const Mat<T>& m, const Ctx<T>& c, V3<T> wo, V3<T> wi) {
    if (m.type == MAT_LAMBERT || m.type == MAT_EMISSIVE) return lamEval(m, c, wo, wi);
    if (m.type == MAT_STANDARD) return ssEval(m, c, wo, wi);
    return m.hairMode == 1 ? msEval(m, c, wo, wi) : kkEval(m, c, wo, wi);
}

// ---- lights ----------------------------------------------------------------------
template <class T>
struct LS {
    V3<T> Li, wi;
    T pdf = 0, dist = 0;
};

template <class T> V3<T> envEval(const Scene<T>& S, V3<T> wo) {  // DomeLight.h:453-491
    T theta = std::acos(std::max(T(-1), std::min(T(1), wo.y)));
    T phi = std::atan2(wo.x, wo.z);
    if (phi < T(0)) phi += k2Pi<T>;
    T uu = phi / k2Pi<T>, v = theta / kPi<T>;
    T fc = uu * T(S.ew) - T(0.5f), fr = v * T(S.eh) - T(0.5f);
    int c0 = int(std::floor(fc)), r0 = int(std::floor(fr));
    T tc = fc - T(c0), tr = fr - T(r0);
    int W = int(S.ew), H = int(S.eh);
    auto wc = [&](int c) { return uint32_t((c % W + W) % W); };
    auto cr = [&](int r) { return uint32_t(std::max(0, std::min(r, H - 1))); };
    const T* p00 = &S.env[(size_t(cr(r0)) * S.ew + wc(c0)) * 3];
    const T* p01 = &S.env[(size_t(cr(r0)) * S.ew + wc(c0 + 1)) * 3];
    const T* p10 = &S.env[(size_t(cr(r0 + 1)) * S.ew + wc(c0)) * 3];
    const T* p11 = &S.env[(size_t(cr(r0 + 1)) * S.ew + wc(c0 + 1)) * 3];
    T s[3];
    for (int ch = 0; ch < 3; ++ch) {
        s[ch] = (T(1) - tr) * ((T(1) - tc) * p00[ch] + tc * p01[ch]) + tr * ((T(1) - tc) * p10[ch] + tc * p11[ch]);
        s[ch] = std::max(T(0), s[ch]);
    }
    return V3<T>(s[0], s[1], s[2]);
}
template <class T> V3<T> envLe(const Scene<T>& S, V3<T> d) {
    return S.dome ? envEval(S, d) * S.intensity : S.envRadiance;
}
template <class T> T envPdf(const Scene<T>& S, V3<T> wo) {  // DomeLight.h:427-448
    T theta = std::acos(std::max(T(-1), std::min(T(1), wo.y)));
    T phi = std::atan2(wo.x, wo.z);
    if (phi < T(0)) phi += k2Pi<T>;
    T uu = phi / k2Pi<T>, v = theta / kPi<T>;
    uint32_t col = std::min(uint32_t(uu * T(S.ew)), S.ew - 1u);
    uint32_t row = std::min(uint32_t(v * T(S.eh)), S.eh - 1u);
    T st = std::max(std::sin(theta), T(1e-6f));
    T pr = S.marg.integral > T(0) ? S.marg.func[row] / S.marg.integral : T(0);
    T pc = S.cond[row].integral > T(0) ? S.cond[row].func[col] / S.cond[row].integral : T(0);
    return (pr * pc * T(S.ew * S.eh)) / (k2Pi<T> * kPi<T> * st);
}
template <class T> LS<T> envSample(const Scene<T>& S, T ux, T uy) {  // DomeLight.h:244-256, 391-422
    T pR, pC, rR, rC;
    uint32_t row = S.marg.sample(uy, pR, rR);
    uint32_t col = S.cond[row].sample(ux, pC, rC);
    T v = (T(row) + rR) / T(S.eh), uu = (T(col) + rC) / T(S.ew);
    T theta = v * kPi<T>, phi = uu * k2Pi<T>;
    T st = std::sin(theta), ct = std::cos(theta);
    V3<T> dir(st * std::sin(phi), ct, st * std::cos(phi));
    T pdf = (pR * pC * T(S.ew * S.eh)) / (k2Pi<T> * kPi<T> * std::max(st, T(1e-6f)));
    LS<T> ls;
    if (pdf <= T(0)) return ls;
    ls.Li = envEval(S, dir) * S.intensity;
    ls.wi = dir;
    ls.pdf = pdf;
    ls.dist = T(1e10f);
    return ls;
}
template <class T> LS<T> areaSample(const Light<T>& L, V3<T> p, T ux, T uy) {  // AreaLight.h:32-56
    V3<T> pos = L.c + L.u * (T(2) * ux - T(1)) + L.v * (T(2) * uy - T(1));
    V3<T> tl = pos - p;
    T d2 = tl.lengthSq(), d = std::sqrt(d2);
    V3<T> wi = tl * (T(1) / d);
    T cosL = dot(-wi, L.n);
    LS<T> ls;
    if (cosL <= T(0)) return ls;
    ls.Li = L.Le;
    ls.wi = wi;
    ls.pdf = d2 / (cosL * L.area);
    ls.dist = d * (T(1) - T(1e-4f));
    return ls;
}
template <class T> T areaPdf(const Light<T>& L, V3<T> p, V3<T> wi) {  // AreaLight.h:58-79
    T den = dot(wi, -L.n);
    if (den < T(1e-6f)) return T(0);
    T t = dot(L.c - p, -L.n) / den;
    if (t <= T(0)) return T(0);
    V3<T> off = (p + wi * t) - L.c;
    T ul = L.u.length(), vl = L.v.length();
    T up = dot(off, L.u) / (ul * ul), vp = dot(off, L.v) / (vl * vl);
    if (std::abs(up) > T(1) || std::abs(vp) > T(1)) return T(0);
    return (t * t) / (den * L.area);
}

template <class T> T powerH(T f, T g) { return (f * f) / (f * f + g * g); }

// DirectionalLight::sample (DirectionalLight.h:52-78): delta, pdf 1, the
// direction toward the light jittered inside its cone when it has one.
template <class T> LS<T> dirSample(const Light<T>& L, T ux, T uy) {
    LS<T> ls;
    ls.Li = L.Le;
    ls.pdf = T(1);
    ls.dist = T(1e10f);
    if (L.cosCone >= T(1) - T(1e-6f)) {
        ls.wi = L.n;
    } else {
        T ct = T(1) - ux * (T(1) - L.cosCone);
        T st = std::sqrt(std::max(T(0), T(1) - ct * ct));
        T phi = T(2) * kPi<T> * uy;
        V3<T> t, bt;
        onb(L.n, t, bt);
        ls.wi = safeNormalize(t * (st * std::cos(phi)) + bt * (st * std::sin(phi)) + L.n * ct);
    }
    return ls;
}

template <class T> const Mat<T>* matOf(const Scene<T>& S, uint32_t slot) {
    if (slot >= S.slots.size() || S.slots[slot] < 0) return nullptr;
    return &S.mats[size_t(S.slots[slot])];
}

// shadowTransmittance (ShadowRay.h:26-61): closest hits through at most 8
// surfaces, multiplying their transmittanceColor; an opaque one blocks. In a
// scene without transmissive materials this is the any-hit query.
template <class T>
V3<T> shadowTr(const Scene<T>& S, Ray<T> r) {
    V3<T> Tr(1, 1, 1);
    if (!S.transmit) return trace(S, r, true).hit ? V3<T>() : Tr;
    for (int i = 0; i < 8; ++i) {
        Hit<T> h = trace(S, r);
        if (!h.hit) break;
        SI<T> si = surface(S, r, h);
        const Mat<T>* m = matOf(S, si.slot);
        if (!m) return {};
        if (m->tint.black()) return {};
        Tr = Tr * m->tint;
        if (Tr.black()) return {};
        T remaining = r.tmax - h.t;
        if (remaining <= T(1e-4f)) break;
        const T time = r.time;
        r = spawnRay(si.p, si.ng, r.d);
        r.tmax = remaining - T(1e-4f);
        r.time = time;
    }
    return Tr;
}

// PathIntegrator::Li + estimateDirect (PathIntegrator.cpp:71-265), static scenes
// (opaque, glass and alpha-masked materials).
template <class T>
V3<T> Li(const Scene<T>& S, Ray<T> r, Halton& smp, uint32_t maxDepth, uint32_t minDepth = 2) {
    const T time = r.time;  // every ray of the path sees the scene at the camera ray's time
    V3<T> L, beta(1, 1, 1);
    bool spec = false;
    const uint32_t nL = uint32_t(S.lights.size());
    auto u1 = [&]() { return T(smp.get1D()); };
    for (uint32_t bounce = 0; bounce <= maxDepth; ++bounce) {
        Hit<T> h = trace(S, r);
        if (!h.hit) {
            if (bounce == 0 || spec) L = L + beta * envLe(S, r.d);
            break;
        }
        SI<T> si = surface(S, r, h);
        const Mat<T>* m = matOf(S, si.slot);
        if (!m) break;
        V3<T> wo = -r.d;
        Ctx<T> c(si, r.d);
        // alpha test (PathIntegrator.cpp:103-118): a sample dimension only for
        // partial opacity; a cut-out point continues the ray, one bounce later
        if (m->opacity <= T(0) || (m->opacity < T(1) && T(smp.get1D()) >= m->opacity)) {
            r = spawnRay(si.p, si.ng, r.d);
            r.time = time;
            continue;
        }
        if (!m->emission.black() && (bounce == 0 || spec)) L = L + beta * m->emission;
        if (!m->delta && nL > 0) {
            uint32_t li = std::min(uint32_t(smp.get1D() * float(nL)), nL - 1);
            const Light<T>& lt = S.lights[li];
            V3<T> Ld;
            {
                T a = u1(), b = u1();
                LS<T> ls = lt.type == 0 ? areaSample(lt, si.p, a, b)
                           : lt.type == 2 ? dirSample(lt, a, b) : envSample(S, a, b);
                if (ls.pdf > T(0) && !ls.Li.black()) {
                    BE<T> be = matEval(*m, c, wo, ls.wi);
                    if (!be.f.black()) {
                        Ray<T> sr = spawnRayTo(si.p, si.n, si.p + ls.wi * ls.dist);
                        sr.time = time;
                        V3<T> Tr = shadowTr(S, sr);
                        if (!Tr.black()) {
                            T w = lt.type == 2 ? T(1) : powerH(ls.pdf, be.pdf);
                            T cosI = si.curve ? std::sqrt(std::max(T(0), T(1) - dot(ls.wi, c.t) * dot(ls.wi, c.t)))
                                              : std::abs(dot(ls.wi, si.n));
                            Ld = Ld + be.f * ls.Li * Tr * cosI * w / ls.pdf;
                        }
                    }
                }
            }
            if (lt.type != 2) {  // BSDF sampling for non-delta lights only (PathIntegrator.cpp:210)
                T uc = u1();  // right-to-left argument evaluation of sample(ctx, wo, get2D(), get1D())
                T a = u1(), b = u1();
                BS<T> bs = matSample(*m, c, wo, a, b, uc);
                if (bs.valid()) {
                    T lp = lt.type == 0 ? areaPdf(lt, si.p, bs.wi) : envPdf(S, bs.wi);
                    if (lp > T(0)) {
                        T w = bs.delta() ? T(1) : powerH(bs.pdf, lp);
                        Ray<T> mr = spawnRay(si.p, si.ng, bs.wi);
                        mr.tmax = T(1e10f);
                        mr.time = time;
                        // the first non-transmissive surface, through at most 8
                        // transmissive ones (PathIntegrator.cpp:220-244)
                        V3<T> Tr(1, 1, 1);
                        Hit<T> mh;
                        SI<T> ms;
                        for (int k = 0; k < 8; ++k) {
                            mh = trace(S, mr);
                            if (!mh.hit) break;
                            ms = surface(S, mr, mh);
                            const Mat<T>* tm = matOf(S, ms.slot);
                            if (!tm) {
                                Tr = V3<T>();
                                break;
                            }
                            if (tm->tint.black()) break;
                            Tr = Tr * tm->tint;
                            if (Tr.black()) break;
                            T remaining = mr.tmax - mh.t;
                            if (remaining <= T(1e-4f)) {
                                mh.hit = false;
                                break;
                            }
                            mr = spawnRay(ms.p, ms.ng, mr.d);
                            mr.tmax = remaining - T(1e-4f);
                            mr.time = time;
                        }
                        V3<T> Lm;
                        if (!mh.hit) Lm = envLe(S, bs.wi);
                        else {
                            const Mat<T>* hm = matOf(S, ms.slot);
                            if (hm) Lm = hm->emission;
                        }
                        if (!Lm.black() && !Tr.black())
                            Ld = Ld + bs.f * Lm * Tr * std::abs(dot(bs.wi, si.n)) * w / bs.pdf;
                    }
                }
            }
            L = L + beta * Ld * T(float(nL));
        }
        T uc = u1();
        T a = u1(), b = u1();
        BS<T> bs = matSample(*m, c, wo, a, b, uc);
        if (!bs.valid()) break;
        spec = bs.delta();
        beta = beta * (bs.f / bs.pdf);
        r = spawnRay(si.p, si.n, bs.wi);
        r.time = time;
        if (bounce >= minDepth) {
            T q = T(1) - std::min(beta.maxc(), T(0.95f));
            if (T(smp.get1D()) < q) break;
            beta = beta * (T(1) / (T(1) - q));
        }
    }
    return L;
}

// ---- FP64 reference adjoint (test infrastructure) ------------------------------
// dL/d theta of one path estimate by forward-mode accumulation along the path:
// d beta and d L are dense over the parameters (3 channels each), in double.
// Parameters: 8 per material (albedo rgb, roughness, emission rgb, -), then 4
// per light (Le rgb, -). Sampling decisions, pdfs, MIS weights and Russian
// roulette are held at the path's values: the estimator that a path-replay
// adjoint differentiates. The path itself is traced in T exactly as Li does;
// the local BSDF derivatives come from central differences of the BSDF value
// in double at the path's local directions (independent of any hand-written
// derivative).
template <class T> Mat<double> matD(const Mat<T>& m) {
    Mat<double> o;
    o.type = m.type;
    o.albedo = V3<double>(m.albedo.x, m.albedo.y, m.albedo.z);
    o.emission = V3<double>(m.emission.x, m.emission.y, m.emission.z);
    o.base = m.base;
    o.metal = m.metal;
    o.rough = m.rough;
    o.spec = m.spec;
    o.coat = m.coat;
    o.coatRough = m.coatRough;
    o.ior = m.ior;
    o.specColor = V3<double>(m.specColor.x, m.specColor.y, m.specColor.z);
    o.coatAlpha2 = m.coatAlpha2;
    o.f0 = m.f0;
    o.coatF0 = m.coatF0;
    o.flags = m.flags;
    o.delta = m.delta;
    return o;
}
// BSDF value in the local frame, double (Lambert, emissive, standard; hair: 0).
inline V3<double> bsdfLocal(const Mat<double>& m, V3<double> wo, V3<double> wi) {
    if (!(wo.z * wi.z > 0.0)) return {};
    if (m.type == MAT_LAMBERT || m.type == MAT_EMISSIVE) return m.albedo * kInvPi<double>;
    if (m.type != MAT_STANDARD) return {};
    W4<double> w;
    if (!ssWeights(m, wo.z, w)) return {};
    double pdf;
    return ssCombined(m, wo, wi, w, pdf);
}
// J[k] = d f / d theta_k for theta = (albedo r, g, b, roughness), f in double.
inline void bsdfJacobian(const Mat<double>& m0, V3<double> wo, V3<double> wi, V3<double> J[4]) {
    for (int k = 0; k < 4; ++k) {
        Mat<double> a = m0, b = m0;
        double h;
        if (k < 3) {
            h = 1e-4;
            double* pa = k == 0 ? &a.albedo.x : k == 1 ? &a.albedo.y : &a.albedo.z;
            double* pb = k == 0 ? &b.albedo.x : k == 1 ? &b.albedo.y : &b.albedo.z;
            *pa += h;
            *pb -= h;
        } else {
            h = 1e-5;
            a.rough += h;
            b.rough -= h;
        }
        J[k] = (bsdfLocal(a, wo, wi) - bsdfLocal(b, wo, wi)) * (0.5 / h);
    }
}

struct PathGrad {
    size_t P;
    std::vector<double> dbeta, dL;  // [param][channel]
    explicit PathGrad(size_t p) : P(p), dbeta(3 * p, 0.0), dL(3 * p, 0.0) {}
    // dL += dbeta * s (per channel)
    void addScaled(const double s[3]) {
        for (size_t k = 0; k < P; ++k)
            for (int c = 0; c < 3; ++c) dL[3 * k + c] += dbeta[3 * k + c] * s[c];
    }
};

template <class T>
V3<T> LiGrad(const Scene<T>& S, Ray<T> r, Halton& smp, uint32_t maxDepth, PathGrad& G, uint32_t minDepth = 2) {
    V3<T> L, beta(1, 1, 1);
    bool spec = false;
    const uint32_t nL = uint32_t(S.lights.size());
    const size_t lightBase = 8 * S.mats.size();
    auto u1 = [&]() { return T(smp.get1D()); };
    auto d3 = [](V3<T> v) { return V3<double>(double(v.x), double(v.y), double(v.z)); };
    // beta-weighted local derivative term: dL[param k of material mi] += beta * J_k * s
    auto addLocal = [&](uint32_t mi, const V3<double> J[4], const double s[3]) {
        const double b[3] = {double(beta.x), double(beta.y), double(beta.z)};
        for (int k = 0; k < 4; ++k)
            for (int c = 0; c < 3; ++c) G.dL[3 * (8 * mi + k) + c] += b[c] * J[k][c] * s[c];
    };
    for (uint32_t bounce = 0; bounce <= maxDepth; ++bounce) {
        Hit<T> h = trace(S, r);
        if (!h.hit) {
            if (bounce == 0 || spec) {
                V3<T> bg = envLe(S, r.d);
                const double s[3] = {double(bg.x), double(bg.y), double(bg.z)};
                G.addScaled(s);
                L = L + beta * bg;
            }
            break;
        }
        SI<T> si = surface(S, r, h);
        const Mat<T>* m = matOf(S, si.slot);
        if (!m) break;
        const uint32_t mi = uint32_t(m - S.mats.data());
        const Mat<double> mD = matD(*m);
        V3<T> wo = -r.d;
        Ctx<T> c(si, r.d);
        const V3<double> wol = d3(c.toLocal(wo));
        if (!m->emission.black() && (bounce == 0 || spec)) {
            const double s[3] = {double(m->emission.x), double(m->emission.y), double(m->emission.z)};
            G.addScaled(s);
            L = L + beta * m->emission;
        }
        if (m->type == MAT_EMISSIVE && (bounce == 0 || spec))
            for (int ch = 0; ch < 3; ++ch) G.dL[3 * (8 * mi + 4 + ch) + ch] += double(beta[ch]);
        if (!m->delta && nL > 0) {
            uint32_t li = std::min(uint32_t(smp.get1D() * float(nL)), nL - 1);
            const Light<T>& lt = S.lights[li];
            V3<T> Ld;
            {
                T a = u1(), b = u1();
                LS<T> ls = lt.type == 0 ? areaSample(lt, si.p, a, b)
                           : lt.type == 2 ? dirSample(lt, a, b) : envSample(S, a, b);
                if (ls.pdf > T(0) && !ls.Li.black()) {
                    BE<T> be = matEval(*m, c, wo, ls.wi);
                    if (!be.f.black()) {
                        Ray<T> sr = spawnRayTo(si.p, si.n, si.p + ls.wi * ls.dist);
                        if (!trace(S, sr, true).hit) {
                            T w = lt.type == 2 ? T(1) : powerH(ls.pdf, be.pdf);
                            T cosI = si.curve ? std::sqrt(std::max(T(0), T(1) - dot(ls.wi, c.t) * dot(ls.wi, c.t)))
                                              : std::abs(dot(ls.wi, si.n));
                            Ld = Ld + be.f * ls.Li * cosI * w / ls.pdf;
                            const double k = double(cosI) * double(w) / double(ls.pdf) * double(nL);
                            const double sf[3] = {double(be.f.x * ls.Li.x) * k, double(be.f.y * ls.Li.y) * k,
                                                  double(be.f.z * ls.Li.z) * k};
                            G.addScaled(sf);
                            V3<double> J[4];
                            bsdfJacobian(mD, wol, d3(c.toLocal(ls.wi)), J);
                            const double sl[3] = {double(ls.Li.x) * k, double(ls.Li.y) * k, double(ls.Li.z) * k};
                            addLocal(mi, J, sl);
                            if (lt.type == 0)
                                for (int ch = 0; ch < 3; ++ch)
                                    G.dL[3 * (lightBase + 4 * li + ch) + ch] += double(beta[ch]) * double(be.f[ch]) * k;
                        }
                    }
                }
            }
            if (lt.type != 2) {
                T uc = u1();
                T a = u1(), b = u1();
                BS<T> bs = matSample(*m, c, wo, a, b, uc);
                if (bs.valid()) {
                    T lp = lt.type == 0 ? areaPdf(lt, si.p, bs.wi) : envPdf(S, bs.wi);
                    if (lp > T(0)) {
                        T w = bs.delta() ? T(1) : powerH(bs.pdf, lp);
                        Ray<T> mr = spawnRay(si.p, si.ng, bs.wi);
                        mr.tmax = T(1e10f);
                        Hit<T> mh = trace(S, mr);
                        V3<T> Lm;
                        int hm = -1;
                        if (!mh.hit) Lm = envLe(S, bs.wi);
                        else {
                            SI<T> ms = surface(S, mr, mh);
                            const Mat<T>* hmat = matOf(S, ms.slot);
                            if (hmat) {
                                Lm = hmat->emission;
                                hm = int(hmat - S.mats.data());
                            }
                        }
                        const T cosN = std::abs(dot(bs.wi, si.n));
                        if (!Lm.black()) Ld = Ld + bs.f * Lm * cosN * w / bs.pdf;
                        const double k = double(cosN) * double(w) / double(bs.pdf) * double(nL);
                        if (!Lm.black()) {
                            const double sf[3] = {double(bs.f.x * Lm.x) * k, double(bs.f.y * Lm.y) * k,
                                                  double(bs.f.z * Lm.z) * k};
                            G.addScaled(sf);
                            const V3<double> wil = d3(c.toLocal(bs.wi));
                            V3<double> J[4];
                            bsdfJacobian(mD, wol, wil, J);
                            const double cl = std::abs(wil.z);
                            const double sl[3] = {double(Lm.x) * k * cl, double(Lm.y) * k * cl, double(Lm.z) * k * cl};
                            addLocal(mi, J, sl);
                        }
                        if (hm >= 0 && S.mats[size_t(hm)].type == MAT_EMISSIVE)
                            for (int ch = 0; ch < 3; ++ch)
                                G.dL[3 * (8 * size_t(hm) + 4 + ch) + ch] += double(beta[ch]) * double(bs.f[ch]) * k;
                    }
                }
            }
            L = L + beta * Ld * T(float(nL));
        }
        T uc = u1();
        T a = u1(), b = u1();
        BS<T> bs = matSample(*m, c, wo, a, b, uc);
        if (!bs.valid()) break;
        spec = bs.delta();
        // d beta' = d beta * (f/pdf) + beta * (d f / d theta) |cos| / pdf, then the roulette factor
        const V3<double> wil = d3(c.toLocal(bs.wi));
        V3<double> J[4];
        bsdfJacobian(mD, wol, wil, J);
        const double cl = std::abs(wil.z);
        const double wr[3] = {double(bs.f.x / bs.pdf), double(bs.f.y / bs.pdf), double(bs.f.z / bs.pdf)};
        const double bOld[3] = {double(beta.x), double(beta.y), double(beta.z)};
        for (size_t k = 0; k < G.P; ++k)
            for (int ch = 0; ch < 3; ++ch) G.dbeta[3 * k + ch] *= wr[ch];
        for (int k = 0; k < 4; ++k)
            for (int ch = 0; ch < 3; ++ch) G.dbeta[3 * (8 * mi + k) + ch] += bOld[ch] * J[k][ch] * cl / double(bs.pdf);
        beta = beta * (bs.f / bs.pdf);
        r = spawnRay(si.p, si.n, bs.wi);
        if (bounce >= minDepth) {
            T q = T(1) - std::min(beta.maxc(), T(0.95f));
            if (T(smp.get1D()) < q) break;
            const T rr = T(1) / (T(1) - q);
            beta = beta * rr;
            for (double& v : G.dbeta) v *= double(rr);
        }
    }
    return L;
}

// Camera::generateRay (IIntegrator.h:90-109), pinhole.
template <class T> Ray<T> cameraRay(const Scene<T>& S, uint32_t px, uint32_t py, T jx, T jy, T timeU = 0) {
    T s = (T(px) + jx) / T(S.W);
    T t = (T(S.H - 1 - py) + jy) / T(S.H);
    V3<T> target = S.camLL + S.camH * s + S.camV * t;
    Ray<T> r;
    r.o = S.camO;
    r.d = normalize(target - S.camO);
    r.time = S.shutterOpen + timeU * (S.shutterClose - S.shutterOpen);  // Camera::generateRay
    return r;
}

template <class T>
V3<T> sampleLi(const Scene<T>& S, uint32_t px, uint32_t py, uint32_t sIdx, uint32_t maxDepth, uint64_t seed) {
    Halton h;
    h.seed = seed;
    h.start(px, py, sIdx);
    T jx = T(h.get1D()), jy = T(h.get1D());
    h.get1D();
    h.get1D();
    T tu = T(h.get1D());
    return Li(S, cameraRay(S, px, py, jx, jy, tu), h, maxDepth);
}

// Per-row sums of the path gradients of a frame, weighted by dLoss/dL =
// dLoss/d pixel / spp for finite samples (the film drops the others).
template <class T>
void adjointRows(const Scene<T>& S, uint32_t W, uint32_t H, uint32_t spp, uint32_t s0, uint32_t maxDepth,
                 uint64_t seed, const float* dimage, int threads, size_t P, std::vector<std::vector<double>>& rows) {
    parallel_for(H, threads, [&](uint32_t py) {
        std::vector<double>& acc = rows[py];
        for (uint32_t px = 0; px < W; ++px) {
            const float* dI = dimage + 3 * (size_t(py) * W + px);
            for (uint32_t s = 0; s < spp; ++s) {
                Halton hs;
                hs.seed = seed;
                hs.start(px, py, s0 + s);
                T jx = T(hs.get1D()), jy = T(hs.get1D());
                hs.get1D();
                hs.get1D();
                hs.get1D();
                PathGrad G(P);
                V3<T> L = LiGrad(S, cameraRay(S, px, py, jx, jy), hs, maxDepth, G);
                if (!L.finite()) continue;
                for (size_t k = 0; k < P; ++k)
                    for (int c = 0; c < 3; ++c) acc[k] += double(dI[c]) / double(spp) * G.dL[3 * k + c];
            }
        }
    });
}

}  // namespace po

// ============================================================================
// C API
// ============================================================================
using namespace po;

namespace {

struct Handle {
    int precision;  // 32 or 64
    Scene<float> f;
    Scene<double> d;
};

template <class T> V3<T> ld(const float* p) { return V3<T>(T(p[0]), T(p[1]), T(p[2])); }

template <class T>
void add_mesh(Scene<T>& S, uint32_t meshID, const float* pos, const float* nrm, uint32_t nv,
              const uint32_t* idx, uint32_t ntri) {
    (void)nv;
    for (uint32_t t = 0; t < ntri; ++t) {  // BVHBackend::commit (BVHBackend.cpp:17-111)
        Tri<T> tr;
        V3<T> a = ld<T>(pos + 3 * idx[3 * t]), b = ld<T>(pos + 3 * idx[3 * t + 1]), c = ld<T>(pos + 3 * idx[3 * t + 2]);
        tr.v0 = a;
        tr.e1 = b - a;
        tr.e2 = c - a;
        tr.n = safeNormalize(cross(tr.e1, tr.e2));
        auto sn = [&](uint32_t i) { return nrm ? safeNormalize(ld<T>(nrm + 3 * i)) : tr.n; };
        tr.sn0 = sn(idx[3 * t]);
        tr.sn1 = sn(idx[3 * t + 1]);
        tr.sn2 = sn(idx[3 * t + 2]);
        tr.mesh = meshID;
        tr.prim = t;
        S.tris.push_back(tr);
    }
}

// A motion-blurred mesh (MeshDesc with motionKeys): object-space triangles
// and nkeys keys of 17 floats (time, objectToWorld row-major).
template <class T>
void add_mesh_motion(Scene<T>& S, uint32_t meshID, const float* pos, const float* nrm, uint32_t nv,
                     const uint32_t* idx, uint32_t ntri, const float* keys, uint32_t nkeys) {
    const size_t first = S.tris.size();
    add_mesh(S, meshID, pos, nrm, nv, idx, ntri);
    for (size_t i = first; i < S.tris.size(); ++i) S.tris[i].objectSpace = nkeys > 0;
    if (S.motion.size() <= meshID) S.motion.resize(meshID + 1);
    S.motion[meshID].clear();
    for (uint32_t k = 0; k < nkeys; ++k) {
        Key<T> key;
        key.time = T(keys[17 * k]);
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) key.o2w.m[i][j] = T(keys[17 * k + 1 + 4 * i + j]);
        S.motion[meshID].push_back(key);
    }
}

template <class T>
void commit(Scene<T>& S) {
    S.transmit = false;
    for (int slot : S.slots)
        if (slot >= 0 && size_t(slot) < S.mats.size() && !S.mats[size_t(slot)].tint.black()) S.transmit = true;
    build_bvh(uint32_t(S.tris.size()), [&](uint32_t i, float* b) {
        const Tri<T>& t = S.tris[i];
        V3<T> v[3] = {t.v0, t.v0 + t.e1, t.v0 + t.e2};
        if (!t.objectSpace) {
            for (int a = 0; a < 3; ++a) {
                b[a] = float(std::min({v[0][a], v[1][a], v[2][a]}));
                b[3 + a] = float(std::max({v[0][a], v[1][a], v[2][a]}));
            }
            return;
        }
        // a moving triangle: its world positions at every key bound it over
        // the shutter (the keys' matrices are affine and lerped, so each
        // vertex moves linearly between keys; BVHBackend.cpp:86-95)
        for (int a = 0; a < 3; ++a) {
            b[a] = INFINITY;
            b[3 + a] = -INFINITY;
        }
        for (const Key<T>& k : S.motion[t.mesh])
            for (const V3<T>& p : v) {
                V3<T> w = k.o2w.point(p);
                for (int a = 0; a < 3; ++a) {
                    b[a] = std::min(b[a], std::nextafter(float(w[a]), -INFINITY));
                    b[3 + a] = std::max(b[3 + a], std::nextafter(float(w[a]), INFINITY));
                }
            }
    }, S.triNodes, S.triIdx);
    S.segs.clear();
    S.strandColor.clear();
    for (uint32_t s = 0; s < S.raw.size(); ++s) {
        auto& R = S.raw[s];
        S.strandColor.push_back(R.color);
        uint32_t N = R.cps.size() < 4 ? 0 : uint32_t((R.cps.size() - 1) / 3);
        auto widthAt = [&](T v) -> T {  // CurvePool.h:45-54
            size_t n = R.widths.size();
            if (n == 0) return T(0.001f);
            if (n == 1) return R.widths[0];
            if (n == 2) return R.widths[0] * (T(1) - v) + R.widths[1] * v;
            T id = v * T(int(n) - 1);
            int lo = std::max(0, int(id)), hi = std::min(int(n) - 1, lo + 1);
            T fr = id - T(lo);
            return R.widths[lo] * (T(1) - fr) + R.widths[hi] * fr;
        };
        for (uint32_t k = 0; k < N; ++k) {
            Seg<T> g;
            for (int j = 0; j < 4; ++j) g.P[j] = R.cps[3 * k + j];
            g.v0 = T(float(k) / float(N));
            T v3 = T(float(k + 1) / float(N));
            g.dv = v3 - g.v0;
            g.hw0 = widthAt(g.v0) * T(0.5f);
            g.hw3 = widthAt(v3) * T(0.5f);
            g.strand = s;
            g.seg = k;
            g.slot = R.slot;
            S.segs.push_back(g);
        }
    }
    build_bvh(uint32_t(S.segs.size()), [&](uint32_t i, float* b) {
        const Seg<T>& g = S.segs[i];
        T mh = std::max(g.hw0, g.hw3);
        for (int a = 0; a < 3; ++a) {
            b[a] = float(std::min({g.P[0][a], g.P[1][a], g.P[2][a], g.P[3][a]}) - mh);
            b[3 + a] = float(std::max({g.P[0][a], g.P[1][a], g.P[2][a], g.P[3][a]}) + mh);
        }
    }, S.segNodes, S.segIdx);
}

template <class T>
void set_dome(Scene<T>& S, const float* rgb, uint32_t w, uint32_t h, float intensity) {
    S.dome = true;
    S.ew = w;
    S.eh = h;
    S.intensity = T(intensity);
    S.env.assign(size_t(w) * h * 3, T(0));
    for (size_t i = 0; i < S.env.size(); ++i) S.env[i] = T(rgb[i]);
    // DomeLight::buildDistribution (DomeLight.h:355-386)
    std::vector<T> rowSums(h), rowFunc(w);
    S.cond.assign(h, Dist1D<T>{});
    for (uint32_t r = 0; r < h; ++r) {
        T theta = kPi<T> * (T(r) + T(0.5f)) / T(h);
        T st = std::sin(theta);
        for (uint32_t c = 0; c < w; ++c) {
            const T* px = &S.env[(size_t(r) * w + c) * 3];
            T lum = T(0.2126f) * px[0] + T(0.7152f) * px[1] + T(0.0722f) * px[2];
            rowFunc[c] = lum * st;
        }
        S.cond[r].build(rowFunc.data(), w);
        rowSums[r] = S.cond[r].integral;
    }
    S.marg.build(rowSums.data(), h);
    Light<T> L;
    L.type = 1;
    S.lights.push_back(L);
}

template <class T>
void set_camera(Scene<T>& S, const float* from, const float* at, const float* up, float vfov, uint32_t w, uint32_t h) {
    // Camera::makePinhole (IIntegrator.h:49-74); float constants as the reference spells them
    T theta = T(vfov) * T(3.14159265f) / T(180.f);
    T hh = std::tan(theta * T(0.5f));
    T aspect = T(w) / T(h);
    V3<T> f = ld<T>(from), a = ld<T>(at), u0 = ld<T>(up);
    V3<T> ww = normalize(f - a), uu = normalize(cross(u0, ww)), vv = cross(ww, uu);
    T vpH = T(2) * hh, vpW = aspect * vpH;
    S.camO = f;
    S.camH = uu * vpW;
    S.camV = vv * vpH;
    S.camLL = f - uu * (vpW * T(0.5f)) - vv * (vpH * T(0.5f)) - ww;
    S.W = w;
    S.H = h;
}

template <class T>
void render(const Scene<T>& S, uint32_t W, uint32_t H, uint32_t spp, uint32_t s0, uint32_t maxDepth, int threads,
            uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1, uint64_t seed, double* rgbw, double* lumsq) {
    uint32_t rows = y1 - y0;
    parallel_for(rows, threads, [&](uint32_t ry) {
        uint32_t py = y0 + ry;
        for (uint32_t px = x0; px < x1; ++px) {  // PathIntegrator::renderTile (PathIntegrator.cpp:22-68)
            V3<T> acc;
            T lsq = 0;
            for (uint32_t s = 0; s < spp; ++s) {
                V3<T> L = sampleLi(S, px, py, s0 + s, maxDepth, seed);
                if (L.finite()) {
                    acc = acc + L;
                    T l = luminance(L);
                    lsq += l * l;
                }
            }
            T inv = T(1) / T(spp);
            size_t fi = size_t(py) * W + px;
            rgbw[4 * fi + 0] += double(acc.x * inv * T(spp));
            rgbw[4 * fi + 1] += double(acc.y * inv * T(spp));
            rgbw[4 * fi + 2] += double(acc.z * inv * T(spp));
            rgbw[4 * fi + 3] += double(spp);
            lumsq[fi] += double(lsq);
        }
    });
}

}  // namespace

#define BOTH(call) (h->precision == 64 ? (call<double>(h->d)) : (call<float>(h->f)))

extern "C" {

void* po_scene_new(int precision) {
    Handle* h = new Handle();
    h->precision = precision == 64 ? 64 : 32;
    return h;
}
void po_scene_free(void* p) { delete static_cast<Handle*>(p); }

void po_add_mesh(void* p, uint32_t meshID, const float* pos, const float* nrm, uint32_t nv, const uint32_t* idx,
                 uint32_t ntri) {
    Handle* h = static_cast<Handle*>(p);
    if (h->precision == 64) add_mesh(h->d, meshID, pos, nrm, nv, idx, ntri);
    else add_mesh(h->f, meshID, pos, nrm, nv, idx, ntri);
}

void po_add_mesh_motion(void* p, uint32_t meshID, const float* pos, const float* nrm, uint32_t nv,
                        const uint32_t* idx, uint32_t ntri, const float* keys, uint32_t nkeys) {
    Handle* h = static_cast<Handle*>(p);
    if (h->precision == 64) add_mesh_motion(h->d, meshID, pos, nrm, nv, idx, ntri, keys, nkeys);
    else add_mesh_motion(h->f, meshID, pos, nrm, nv, idx, ntri, keys, nkeys);
}

// Camera::shutterOpen / shutterClose (normalized): each path's time is
// shutterOpen + u * (shutterClose - shutterOpen), u its sample dimension 4.
void po_set_shutter(void* p, float open, float close) {
    Handle* h = static_cast<Handle*>(p);
    auto set = [&](auto& S) {
        using T = std::decay_t<decltype(S.env[0])>;
        S.shutterOpen = T(open);
        S.shutterClose = T(close);
    };
    if (h->precision == 64) set(h->d);
    else set(h->f);
}

void po_add_strand(void* p, const float* cps, uint32_t ncp, const float* widths, uint32_t nw, uint32_t slot,
                   const float* color) {
    Handle* h = static_cast<Handle*>(p);
    auto add = [&](auto& S) {
        using T = std::decay_t<decltype(S.env[0])>;
        typename std::decay_t<decltype(S)>::RawStrand R;
        for (uint32_t i = 0; i < ncp; ++i) R.cps.push_back(ld<T>(cps + 3 * i));
        for (uint32_t i = 0; i < nw; ++i) R.widths.push_back(T(widths[i]));
        R.slot = slot;
        R.color = color ? ld<T>(color) : V3<T>(1, 1, 1);
        S.raw.push_back(R);
    };
    if (h->precision == 64) add(h->d);
    else add(h->f);
}

// type: 0 lambert, 1 emissive, 2 standard (p18 packed as the reference harness), 3 hair
int po_add_material(void* p, int type, const float* a3, const float* e3, const float* p18, const float* hair8) {
    Handle* h = static_cast<Handle*>(p);
    auto add = [&](auto& S) {
        using T = std::decay_t<decltype(S.env[0])>;
        Mat<T> m;
        m.type = type;
        if (type == MAT_LAMBERT || type == MAT_EMISSIVE) {
            m.albedo = ld<T>(a3);
            m.flags = 1u | 16u;
            if (type == MAT_EMISSIVE) m.emission = ld<T>(e3);
        } else if (type == MAT_STANDARD) {  // StandardSurface.h:152-181
            m.albedo = ld<T>(p18);
            m.base = T(p18[3]);
            m.metal = T(p18[4]);
            m.rough = T(p18[5]);
            m.spec = T(p18[6]);
            m.specColor = ld<T>(p18 + 7);
            m.ior = T(p18[10]);
            m.coat = T(p18[11]);
            m.coatRough = T(p18[12]);
            if (p18[14] > 0.f) m.emission = ld<T>(p18 + 15) * T(p18[14]);
            T ca = std::max(T(1e-4f), m.coatRough * m.coatRough);
            m.coatAlpha2 = ca * ca;
            T r = (T(1) - m.ior) / (T(1) + m.ior);
            m.f0 = r * r;
            T rc = (T(1) - T(1.5f)) / (T(1) + T(1.5f));
            m.coatF0 = rc * rc;
            m.transmission = T(p18[13]);
            m.alphaMask = p18[18] != 0.f;
            m.opacity = m.alphaMask ? T(p18[19]) : T(1);
            if (m.alphaMask) {  // transmittanceColor (StandardSurface.h:207-218)
                T t = T(1) - m.opacity;
                if (t > T(0)) m.tint = V3<T>(t, t, t);
            } else if (m.transmission >= T(0.001f) && !(m.metal > T(0.001f))) {
                T Fr = fresnel(T(1), m.ior);
                m.tint = m.albedo * (m.transmission * (T(1) - Fr));
            }
            uint32_t f = 16u;
            if (m.transmission > T(0.001f)) f |= 8u;
            if (m.rough < T(0.001f)) f |= 4u;
            else if (m.rough < T(0.3f)) f |= 2u;
            else f |= 1u;
            m.flags = f;
            m.delta = (m.rough < T(0.001f) && m.transmission > T(0.001f) && m.metal < T(0.001f)) ||
                      (m.rough < T(0.001f) && (m.metal > T(0.999f) || m.spec > T(0)));
        } else {  // MarschnerHair.h:200-216
            m.eta = T(hair8[0]);
            m.sigma = ld<T>(hair8 + 1);
            m.bm = T(hair8[4]);
            m.bn = T(hair8[5]);
            m.alphaDeg = T(hair8[6]);
            m.hairMode = int(hair8[7]);
            T bm = std::clamp(m.bm, T(1e-3f), T(1)), bn = std::clamp(m.bn, T(1e-3f), T(1));
            T v0 = T(0.726f) * bm + T(0.812f) * bm * bm + T(3.7f) * std::pow(bm, T(20));
            m.v[0] = v0 * v0;
            m.v[1] = m.v[0] * T(0.25f);
            m.v[2] = m.v[0] * T(4);
            m.s = T(0.626657069f) * (T(0.265f) * bn + T(1.194f) * bn * bn + T(5.372f) * std::pow(bn, T(22)));
            m.ashift[0] = -m.alphaDeg * kPi<T> / T(180);
            m.ashift[1] = m.alphaDeg * kPi<T> / T(180) * T(0.5f);
            m.ashift[2] = -m.alphaDeg * kPi<T> / T(180) * T(1.5f);
            m.flags = 2u | 16u | 8u;
        }
        S.mats.push_back(m);
        return int(S.mats.size() - 1);
    };
    return h->precision == 64 ? add(h->d) : add(h->f);
}

void po_set_slots(void* p, const int32_t* slots, uint32_t n) {
    Handle* h = static_cast<Handle*>(p);
    h->f.slots.assign(slots, slots + n);
    h->d.slots.assign(slots, slots + n);
}

void po_light_area(void* p, const float* c, const float* u, const float* v, const float* Le) {
    Handle* h = static_cast<Handle*>(p);
    auto add = [&](auto& S) {
        using T = std::decay_t<decltype(S.env[0])>;
        Light<T> L;
        L.type = 0;
        L.c = ld<T>(c);
        L.u = ld<T>(u);
        L.v = ld<T>(v);
        L.Le = ld<T>(Le);
        L.n = safeNormalize(cross(L.u, L.v));
        L.area = cross(L.u, L.v).length() * T(4);
        S.lights.push_back(L);
    };
    if (h->precision == 64) add(h->d);
    else add(h->f);
}

void po_light_directional(void* p, const float* dir, const float* Le, float halfAngleDeg) {
    Handle* h = static_cast<Handle*>(p);
    auto add = [&](auto& S) {
        using T = std::decay_t<decltype(S.env[0])>;
        Light<T> L;
        L.type = 2;
        L.n = safeNormalize(ld<T>(dir));
        L.Le = ld<T>(Le);
        L.cosCone = T(std::cos(halfAngleDeg * 3.14159265358979323846f / 180.f));
        S.lights.push_back(L);
    };
    if (h->precision == 64) add(h->d);
    else add(h->f);
}

void po_light_dome(void* p, const float* rgb, uint32_t w, uint32_t hh, float intensity) {
    Handle* h = static_cast<Handle*>(p);
    if (h->precision == 64) set_dome(h->d, rgb, w, hh, intensity);
    else set_dome(h->f, rgb, w, hh, intensity);
}

void po_set_env_radiance(void* p, const float* rgb) {
    Handle* h = static_cast<Handle*>(p);
    h->f.envRadiance = ld<float>(rgb);
    h->d.envRadiance = ld<double>(rgb);
}

void po_set_camera(void* p, const float* from, const float* at, const float* up, float vfov, uint32_t w, uint32_t hh) {
    Handle* h = static_cast<Handle*>(p);
    if (h->precision == 64) set_camera(h->d, from, at, up, vfov, w, hh);
    else set_camera(h->f, from, at, up, vfov, w, hh);
}

void po_commit(void* p) {
    Handle* h = static_cast<Handle*>(p);
    if (h->precision == 64) commit(h->d);
    else commit(h->f);
}

// rays n x 8 floats; ids n x 4 (hit, meshID, primID, strandID); t in double
void po_trace(void* p, const float* rays, uint64_t n, int32_t* ids, double* tout, int threads) {
    Handle* h = static_cast<Handle*>(p);
    auto run = [&](auto& S) {
        using T = std::decay_t<decltype(S.env[0])>;
        parallel_for(uint32_t((n + 1023) / 1024), threads, [&](uint32_t c) {
            for (uint64_t i = uint64_t(c) * 1024; i < std::min<uint64_t>(n, uint64_t(c + 1) * 1024); ++i) {
                Ray<T> r;
                r.o = ld<T>(rays + 8 * i);
                r.tmin = T(rays[8 * i + 3]);
                r.d = ld<T>(rays + 8 * i + 4);
                r.tmax = T(rays[8 * i + 7]);
                Hit<T> hh = trace(S, r);
                ids[4 * i] = hh.hit ? 1 : 0;
                ids[4 * i + 1] = ids[4 * i + 2] = ids[4 * i + 3] = -1;
                tout[i] = 0;
                if (hh.hit) {
                    SI<T> si = surface(S, r, hh);
                    ids[4 * i + 1] = int32_t(si.mesh);
                    ids[4 * i + 2] = int32_t(si.prim);
                    ids[4 * i + 3] = si.curve ? int32_t(si.strand) : -1;
                    tout[i] = double(hh.t);
                }
            }
        });
    };
    if (h->precision == 64) run(h->d);
    else run(h->f);
}

void po_render(void* p, uint32_t W, uint32_t H, uint32_t spp, uint32_t s0, uint32_t maxDepth, int threads,
               uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1, uint64_t seed, double* rgbw, double* lumsq) {
    Handle* h = static_cast<Handle*>(p);
    if (h->precision == 64) render(h->d, W, H, spp, s0, maxDepth, threads, x0, y0, x1, y1, seed, rgbw, lumsq);
    else render(h->f, W, H, spp, s0, maxDepth, threads, x0, y0, x1, y1, seed, rgbw, lumsq);
}

void po_li(void* p, const uint32_t* q, uint64_t n, uint32_t maxDepth, uint64_t seed, double* out, int threads) {
    Handle* h = static_cast<Handle*>(p);
    auto run = [&](auto& S) {
        parallel_for(uint32_t(n), threads, [&](uint32_t i) {
            auto L = sampleLi(S, q[3 * i], q[3 * i + 1], q[3 * i + 2], maxDepth, seed);
            if (!L.finite()) L = decltype(L)();
            out[3 * i] = double(L.x);
            out[3 * i + 1] = double(L.y);
            out[3 * i + 2] = double(L.z);
        });
    };
    if (h->precision == 64) run(h->d);
    else run(h->f);
}

void po_halton(uint32_t px, uint32_t py, uint32_t s, uint64_t seed, uint32_t n, float* out) {
    Halton h;
    h.seed = seed;
    h.start(px, py, s);
    for (uint32_t i = 0; i < n; ++i) out[i] = h.get1D();
}

void po_pcg(uint64_t seed, uint32_t n, uint32_t* out) {
    Pcg r(seed);
    for (uint32_t i = 0; i < n; ++i) out[i] = r.next();
}

float po_ggx_D(float c, float a2) { return D_GGX<float>(c, a2); }

// Number of gradient entries of po_adjoint: 8 per material, 4 per light.
uint64_t po_num_params(void* p) {
    Handle* h = static_cast<Handle*>(p);
    return h->precision == 64 ? 8 * h->d.mats.size() + 4 * h->d.lights.size()
                              : 8 * h->f.mats.size() + 4 * h->f.lights.size();
}

// dLoss/d theta of a W x H x spp frame (samples s0 ..) given dLoss/d image
// (3 per pixel; the image is the film's mean over finite samples), in double.
// grad: po_num_params entries.
void po_adjoint(void* p, uint32_t W, uint32_t H, uint32_t spp, uint32_t s0, uint32_t maxDepth, uint64_t seed,
                const float* dimage, int threads, double* grad) {
    Handle* h = static_cast<Handle*>(p);
    const size_t P = po_num_params(p);
    std::vector<std::vector<double>> rows(H, std::vector<double>(P, 0.0));
    if (h->precision == 64) adjointRows(h->d, W, H, spp, s0, maxDepth, seed, dimage, threads, P, rows);
    else adjointRows(h->f, W, H, spp, s0, maxDepth, seed, dimage, threads, P, rows);
    for (size_t k = 0; k < P; ++k) {
        double s = 0.0;
        for (uint32_t y = 0; y < H; ++y) s += rows[y][k];
        grad[k] = s;
    }
}

// The Marschner lobe functions in float over rows of (cosI, sinI, cosR, sinR,
// v, x, s, u, h, cosO): the outputs of the reference harness's
// ref_mh_functions, in the same order (MarschnerHair.h:88-187).
void po_mh_functions(const float* in, uint32_t n, float eta, const float* sigma_a, float* out) {
    const V3<float> sa(sigma_a[0], sigma_a[1], sigma_a[2]);
    for (uint32_t k = 0; k < n; ++k) {
        const float* q = in + 10 * size_t(k);
        float* o = out + 16 * size_t(k);
        o[0] = mhMp(q[0], q[1], q[2], q[3], q[4]);
        o[1] = mhTrim(q[5], q[6]);
        o[2] = mhSampleTrim(q[7], q[6]);
        const float gO = std::asin(q[8]), gT = 0.3f * q[8];
        for (int p = 0; p < 3; ++p) o[3 + p] = mhTrim(mhWrap(q[5] - mhPhi(p, gO, gT)), q[6]);
        V3<float> ap[3];
        mhAp(q[9], eta, q[8], sa, ap);
        for (int p = 0; p < 3; ++p) {
            o[6 + 3 * p] = ap[p].x;
            o[7 + 3 * p] = ap[p].y;
            o[8 + 3 * p] = ap[p].z;
        }
        const float u2 = q[5] * 0.15915494f + 0.5f;
        o[15] = std::sqrt(-2.f * std::log(std::max(q[7], 1e-6f))) * std::cos(k2Pi<float> * u2);
    }
}

}  // extern "C"
