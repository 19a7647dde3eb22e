// Device vector math. Two flavours:
//   * plain operators (+, -, *) — the compiler may fuse a*b+c into one FMA;
//     used for shading, where results are compared statistically;
//   * the x-prefixed helpers, built on __fadd_rn/__fmul_rn/__fdiv_rn, which
//     never fuse and round each operation as IEEE-754 single precision does on
//     the host. They are used wherever the result must be bit-identical to the
//     reference's float code compiled without contraction: the triangle test,
//     the camera ray and the sampler.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ana {

__host__ __device__ inline float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__host__ __device__ inline float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ inline float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ inline float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ inline float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ inline float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ inline float3 operator*(float s, float3 a) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ inline float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ inline float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ inline float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ inline float length_sq(float3 v) { return dot(v, v); }
__device__ inline float length(float3 v) { return sqrtf(dot(v, v)); }
__device__ inline float3 normalize(float3 v) { return v * (1.f / length(v)); }
// Types.h:86-89
__device__ inline float3 safe_normalize(float3 v, float3 fb = {0.f, 0.f, 1.f}) {
    float len = length(v);
    return len > 1e-8f ? v * (1.f / len) : fb;
}
__device__ inline float absdot(float3 a, float3 b) { return fabsf(dot(a, b)); }
__device__ inline bool is_black(float3 s) { return s.x == 0.f && s.y == 0.f && s.z == 0.f; }
__device__ inline float max_comp(float3 s) { return fmaxf(s.x, fmaxf(s.y, s.z)); }
__device__ inline bool is_finite3(float3 s) { return isfinite(s.x) && isfinite(s.y) && isfinite(s.z); }
// ACEScg luminance, Types.h:245-248
__device__ inline float luminance(float3 s) {
    return 0.2722287f * s.x + 0.6740818f * s.y + 0.0536895f * s.z;
}

// ---- non-contracting IEEE helpers ------------------------------------------
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float3 xsub3(float3 a, float3 b) {
    return f3(xsub(a.x, b.x), xsub(a.y, b.y), xsub(a.z, b.z));
}
__device__ __forceinline__ float3 xadd3(float3 a, float3 b) {
    return f3(xadd(a.x, b.x), xadd(a.y, b.y), xadd(a.z, b.z));
}
__device__ __forceinline__ float3 xmul3(float3 a, float s) {
    return f3(xmul(a.x, s), xmul(a.y, s), xmul(a.z, s));
}
// (a.x*b.x + a.y*b.y) + a.z*b.z, each op rounded: Types.h:70-72
__device__ __forceinline__ float xdot(float3 a, float3 b) {
    return xadd(xadd(xmul(a.x, b.x), xmul(a.y, b.y)), xmul(a.z, b.z));
}
__device__ __forceinline__ float3 xcross(float3 a, float3 b) {
    return f3(xsub(xmul(a.y, b.z), xmul(a.z, b.y)), xsub(xmul(a.z, b.x), xmul(a.x, b.z)),
              xsub(xmul(a.x, b.y), xmul(a.y, b.x)));
}
__device__ __forceinline__ float3 xnormalize(float3 v) {
    float len = __fsqrt_rn(xdot(v, v));
    return xmul3(v, xdiv(1.f, len));
}

__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ int fbits_i(float f) { return __float_as_int(f); }
__device__ __forceinline__ uint32_t fbits_u(float f) { return __float_as_uint(f); }

}  // namespace ana
