// Motion blur on the device: MeshDesc::interpolateO2W (GeometryPool.h:51-65),
// Mat4f's lerp, Gauss-Jordan inverse and transforms (Types.h:144-229), each
// operation rounded on its own as the reference's float code runs, so object
// rays and the hits found with them match the reference's bit for bit.
#pragma once
#include "dmath.cuh"
#include "layout.h"

namespace ana {

struct M4 {
    float m[4][4];
};

__device__ __forceinline__ void m4_identity(M4& r) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) r.m[i][j] = i == j ? 1.f : 0.f;
}

__device__ __forceinline__ void m4_key(const float4* K, uint32_t k, M4& r) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float4 row = ldg4(K + 5 * size_t(k) + 1 + i);
        r.m[i][0] = row.x;
        r.m[i][1] = row.y;
        r.m[i][2] = row.z;
        r.m[i][3] = row.w;
    }
}

// objectToWorld of motion mesh `mm` at normalized time t: the first or last
// key outside the keys' range, else the lerp of the bracketing pair.
__device__ __forceinline__ void o2w_at(const DevScene& S, uint32_t mm, float t, M4& r) {
    const uint2 mk = S.mesh_motion[mm];
    const float4* K = S.motion_keys + 5 * size_t(mk.x);
    const uint32_t n = mk.y;
    if (n == 1 || t <= ldg4(K).x) {
        m4_key(K, 0, r);
        return;
    }
    if (t >= ldg4(K + 5 * size_t(n - 1)).x) {
        m4_key(K, n - 1, r);
        return;
    }
    uint32_t lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (ldg4(K + 5 * size_t(mid)).x <= t) lo = mid;
        else hi = mid;
    }
    const float t0 = ldg4(K + 5 * size_t(lo)).x, t1 = ldg4(K + 5 * size_t(hi)).x;
    const float alpha = xdiv(xsub(t, t0), xsub(t1, t0));
    M4 a, b;
    m4_key(K, lo, a);
    m4_key(K, hi, b);
    const float oneMinus = xsub(1.f, alpha);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) r.m[i][j] = xadd(xmul(a.m[i][j], oneMinus), xmul(b.m[i][j], alpha));
}

// Mat4f::inverse: Gauss-Jordan with partial pivoting; identity when a pivot
// is below 1e-10 in magnitude.
__device__ __forceinline__ void m4_inverse(const M4& M, M4& r) {
    float a[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            a[i][j] = M.m[i][j];
            a[i][j + 4] = i == j ? 1.f : 0.f;
        }
    }
#pragma unroll
    for (int col = 0; col < 4; ++col) {
        int pivot = col;
#pragma unroll
        for (int row = col + 1; row < 4; ++row)
            if (fabsf(a[row][col]) > fabsf(a[pivot][col])) pivot = row;
        if (pivot != col) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                // select rather than index with `pivot` so `a` stays in registers
                float p = a[col][j];
#pragma unroll
                for (int row = col + 1; row < 4; ++row)
                    if (row == pivot) {
                        const float q = a[row][j];
                        a[row][j] = p;
                        p = q;
                    }
                a[col][j] = p;
            }
        }
        const float diag = a[col][col];
        if (fabsf(diag) < 1e-10f) {
            m4_identity(r);
            return;
        }
        const float invDiag = xdiv(1.f, diag);
#pragma unroll
        for (int j = 0; j < 8; ++j) a[col][j] = xmul(a[col][j], invDiag);
#pragma unroll
        for (int row = 0; row < 4; ++row) {
            if (row == col) continue;
            const float factor = a[row][col];
#pragma unroll
            for (int j = 0; j < 8; ++j) a[row][j] = xsub(a[row][j], xmul(factor, a[col][j]));
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) r.m[i][j] = a[i][j + 4];
}

__device__ __forceinline__ float row_dot3(const M4& M, int i, float3 p) {
    return xadd(xadd(xmul(M.m[i][0], p.x), xmul(M.m[i][1], p.y)), xmul(M.m[i][2], p.z));
}
__device__ __forceinline__ float3 m4_point(const M4& M, float3 p) {
    const float x = xadd(row_dot3(M, 0, p), M.m[0][3]), y = xadd(row_dot3(M, 1, p), M.m[1][3]),
                z = xadd(row_dot3(M, 2, p), M.m[2][3]), w = xadd(row_dot3(M, 3, p), M.m[3][3]);
    return f3(xdiv(x, w), xdiv(y, w), xdiv(z, w));
}
__device__ __forceinline__ float3 m4_vector(const M4& M, float3 v) {
    return f3(row_dot3(M, 0, v), row_dot3(M, 1, v), row_dot3(M, 2, v));
}
// Mat4f::transformNormal: the transpose of M applied to n
__device__ __forceinline__ float3 m4_normal(const M4& M, float3 n) {
    return f3(xadd(xadd(xmul(M.m[0][0], n.x), xmul(M.m[1][0], n.y)), xmul(M.m[2][0], n.z)),
              xadd(xadd(xmul(M.m[0][1], n.x), xmul(M.m[1][1], n.y)), xmul(M.m[2][1], n.z)),
              xadd(xadd(xmul(M.m[0][2], n.x), xmul(M.m[1][2], n.y)), xmul(M.m[2][2], n.z)));
}

// safeNormalize (Types.h:80-89) with each operation rounded on its own
__device__ __forceinline__ float3 xsafe_normalize(float3 v) {
    const float len = __fsqrt_rn(xdot(v, v));
    return len > 1e-8f ? xmul3(v, xdiv(1.f, len)) : f3(0.f, 0.f, 1.f);
}

}  // namespace ana
