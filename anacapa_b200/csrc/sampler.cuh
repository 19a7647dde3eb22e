// Scrambled Halton sampler and PCG32, restated for the device so that every
// sample value equals the reference's (src/sampling/HaltonSampler.h:20-113,
// src/sampling/PCGRng.h:15-52) bit for bit.
//
// The sampler is stateless per draw: dimension d of sample i of pixel (x, y)
// is a pure function of (seed, x, y, i, d). Dimensions below 128 use the
// radical inverse in base prime[d] of i XOR a 32-bit PCG scramble derived from
// (seed, x, y, d); dimensions from 128 on read the per-pixel PCG stream seeded
// with seed ^ (x << 32 | y), whose k-th output belongs to dimension 128 + k.
#pragma once
#include "dmath.cuh"

namespace ana {

constexpr uint64_t kPcgMult = 6364136223846793005ULL;
constexpr uint32_t kHaltonDims = 128;

__constant__ uint32_t c_primes[128] = {
    2,   3,   5,   7,   11,  13,  17,  19,  23,  29,  31,  37,  41,  43,  47,  53,
    59,  61,  67,  71,  73,  79,  83,  89,  97,  101, 103, 107, 109, 113, 127, 131,
    137, 139, 149, 151, 157, 163, 167, 173, 179, 181, 191, 193, 197, 199, 211, 223,
    227, 229, 233, 239, 241, 251, 257, 263, 269, 271, 277, 281, 283, 293, 307, 311,
    313, 317, 331, 337, 347, 349, 353, 359, 367, 373, 379, 383, 389, 397, 401, 409,
    419, 421, 431, 433, 439, 443, 449, 457, 461, 463, 467, 479, 487, 491, 499, 503,
    509, 521, 523, 541, 547, 557, 563, 569, 571, 577, 587, 593, 599, 601, 607, 613,
    617, 619, 631, 641, 643, 647, 653, 659, 661, 673, 677, 683, 691, 701, 709, 719};

// PCG32 output permutation (XSH RR) of a 64-bit state.
__device__ __forceinline__ uint32_t pcg_output(uint64_t old) {
    uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = uint32_t(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
}

// State of PCGRng{seed} (stream 1, inc = 3) right after its constructor:
// state = 0; step; state += seed; step.
__device__ __forceinline__ uint64_t pcg_seeded_state(uint64_t seed) {
    uint64_t s = 3ULL;  // 0 * mult + inc
    s += seed;
    return s * kPcgMult + 3ULL;
}

// First nextUint32() of PCGRng{seed}.
__device__ __forceinline__ uint32_t pcg_first(uint64_t seed) {
    return pcg_output(pcg_seeded_state(seed));
}

// radicalInverse(b, n) with the reference's float accumulation order.
__device__ __forceinline__ float radical_inverse(uint32_t b, uint32_t n) {
    const float invB = xdiv(1.f, __uint2float_rn(b));
    float invBN = 1.f, result = 0.f;
    while (n > 0) {
        uint32_t q = n / b;
        uint32_t d = n - q * b;
        n = q;
        invBN = xmul(invBN, invB);
        result = xadd(result, xmul(__uint2float_rn(d), invBN));
    }
    return result;
}

// HaltonSampler::get1D for dimension dim of (px, py, sampleIndex).
__device__ __forceinline__ float halton_sample(uint64_t seed, uint32_t px, uint32_t py,
                                               uint32_t sampleIndex, uint32_t dim) {
    if (dim < kHaltonDims) {
        uint64_t s = seed ^ (uint64_t(px) * 2654435761ULL) ^ (uint64_t(py) * 805459861ULL) ^
                     (uint64_t(dim) * 999999893ULL);
        uint32_t scramble = pcg_first(s);
        return radical_inverse(c_primes[dim], sampleIndex ^ scramble);
    }
    // PCG fallback stream: k-th draw past the Halton dimensions.
    uint64_t st = pcg_seeded_state(seed ^ ((uint64_t(px) << 32) | py));
    for (uint32_t k = kHaltonDims; k < dim; ++k) st = st * kPcgMult + 3ULL;
    return xmul(__uint2float_rn(pcg_output(st)), 2.3283064365386963e-10f);
}

// A path's sample stream: the pixel, sample index and next dimension.
struct SampleStream {
    uint64_t seed;
    uint32_t px, py, index, dim;
    __device__ __forceinline__ float next() { return halton_sample(seed, px, py, index, dim++); }
};

}  // namespace ana
