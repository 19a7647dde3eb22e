// ============================================================================
// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// CPU restatement of the reference renderer's unidirectional path-tracing hot
// path, templated on the arithmetic type T:
//   * T = float, compiled with -ffp-contract=off, reproduces the reference
//     built with the same flag operation for operation (same formulas, same
//     evaluation order, the same glibc libm calls), so sample values, hit ids
//     and per-sample radiance can be compared bit for bit;
//   * T = double is the FP64 oracle: converged reference images (RMSE) and the
//     reference adjoint for the gradient checks.
// Each function cites the reference file:line it follows (paths relative to
// the nhaflinger/anacapa tree). The sampler always produces the reference's
// float sample values; in double mode they are widened.
// ============================================================================
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

namespace po {

template <class T>
struct V3 {
    T x = 0, y = 0, z = 0;
    V3() = default;
    V3(T a, T b, T c) : x(a), y(b), z(c) {}
    V3 operator+(V3 o) const { return {x + o.x, y + o.y, z + o.z}; }
    V3 operator-(V3 o) const { return {x - o.x, y - o.y, z - o.z}; }
    V3 operator*(V3 o) const { return {x * o.x, y * o.y, z * o.z}; }
    V3 operator*(T s) const { return {x * s, y * s, z * s}; }
    V3 operator/(T s) const { return {x / s, y / s, z / s}; }
    V3 operator-() const { return {-x, -y, -z}; }
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    T lengthSq() const { return x * x + y * y + z * z; }
    T length() const { return std::sqrt(lengthSq()); }
    T maxc() const { return std::max({x, y, z}); }
    bool black() const { return x == 0 && y == 0 && z == 0; }
    bool finite() const { return std::isfinite(x) && std::isfinite(y) && std::isfinite(z); }
};
// Types.h:70-114
template <class T> T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> V3<T> normalize(V3<T> v) { return v * (T(1) / v.length()); }
template <class T> V3<T> safeNormalize(V3<T> v, V3<T> fb = V3<T>(0, 0, 1)) {
    T len = v.length();
    return len > T(1e-8f) ? v * (T(1) / len) : fb;
}
template <class T> void onb(V3<T> n, V3<T>& t, V3<T>& b) {
    T sign = std::copysign(T(1), n.z);
    T a = T(-1) / (sign + n.z);
    T bb = n.x * n.y * a;
    t = V3<T>(T(1) + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    b = V3<T>(bb, sign + n.y * n.y * a, -n.y);
}
template <class T> T luminance(V3<T> s) {
    return T(0.2722287f) * s.x + T(0.6740818f) * s.y + T(0.0536895f) * s.z;
}

template <class T>
struct Ray {
    V3<T> o, d;
    T tmin = T(1e-4f), tmax = std::numeric_limits<T>::infinity();
    T time = 0;  // normalized shutter time (motion-blurred meshes)
};

// spawnRay / spawnRayTo (Types.h:269-284)
template <class T> Ray<T> spawnRay(V3<T> p, V3<T> n, V3<T> d) {
    V3<T> off = n * T(1e-4f);
    if (dot(d, n) < T(0)) off = -off;
    Ray<T> r;
    r.o = p + off;
    r.d = d;
    return r;
}
template <class T> Ray<T> spawnRayTo(V3<T> p, V3<T> n, V3<T> target) {
    V3<T> d = target - p;
    T dist = d.length();
    d = d * (T(1) / dist);
    Ray<T> r = spawnRay(p, n, d);
    r.tmax = dist * (T(1) - T(1e-4f));
    return r;
}

// ---------------------------------------------------------------------------
// Sampler: PCGRng (src/sampling/PCGRng.h:15-52), HaltonSampler
// (src/sampling/HaltonSampler.h:20-113). Always float, as the reference.
// ---------------------------------------------------------------------------
struct Pcg {
    uint64_t state = 0x853c49e6748fea9bULL, inc = 0xda3e39cb94b95bdbULL;
    explicit Pcg(uint64_t seed) {
        state = 0;
        inc = (1ULL << 1u) | 1u;
        next();
        state += seed;
        next();
    }
    uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = uint32_t(old >> 59u);
        return (xs >> rot) | (xs << ((-rot) & 31));
    }
    float nextFloat() { return float(next()) * 2.3283064365386963e-10f; }
};

extern const uint32_t kPrimes[128];

inline float radicalInverse(uint32_t b, uint64_t n) {
    float invB = 1.f / float(b), invBN = 1.f, r = 0.f;
    while (n > 0) {
        uint64_t d = n % b;
        n /= b;
        invBN *= invB;
        r += float(d) * invBN;
    }
    return r;
}

struct Halton {
    uint64_t seed = 0;
    uint32_t px = 0, py = 0, index = 0, dim = 0;
    Pcg rng{0};
    void start(uint32_t x, uint32_t y, uint32_t s) {
        px = x;
        py = y;
        index = s;
        dim = 0;
        rng = Pcg(seed ^ (uint64_t(x) << 32 | y));
    }
    float get1D() {
        uint32_t d = dim++;
        if (d >= 128) return rng.nextFloat();
        Pcg r(seed ^ (uint64_t(px) * 2654435761ULL) ^ (uint64_t(py) * 805459861ULL) ^
              (uint64_t(d) * 999999893ULL));
        uint64_t scr = r.next();
        return radicalInverse(kPrimes[d], uint64_t(index) ^ scr);
    }
};

}  // namespace po
