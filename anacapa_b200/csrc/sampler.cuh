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

// c_magic[d] = ceil(2^64 / c_primes[d]): for every 32-bit n, floor(n / b) is
// the high 64 bits of n * c_magic (M*b = 2^64 + e with e < b, so n*e < 2^64
// and the error term never reaches the next integer). The radical inverse's
// digits come from one multiply-high instead of a division by a variable.
__constant__ uint64_t c_magic[128] = {
    0x8000000000000000ULL, 0x5555555555555556ULL, 0x3333333333333334ULL, 0x2492492492492493ULL,
    0x1745D1745D1745D2ULL, 0x13B13B13B13B13B2ULL, 0x0F0F0F0F0F0F0F10ULL, 0x0D79435E50D79436ULL,
    0x0B21642C8590B217ULL, 0x08D3DCB08D3DCB09ULL, 0x0842108421084211ULL, 0x06EB3E45306EB3E5ULL,
    0x063E7063E7063E71ULL, 0x05F417D05F417D06ULL, 0x0572620AE4C415CAULL, 0x04D4873ECADE304EULL,
    0x0456C797DD49C342ULL, 0x04325C53EF368EB1ULL, 0x03D226357E16ECE6ULL, 0x039B0AD12073615BULL,
    0x0381C0E070381C0FULL, 0x033D91D2A2067B24ULL, 0x03159721ED7E7535ULL, 0x02E05C0B81702E06ULL,
    0x02A3A0FD5C5F02A4ULL, 0x0288DF0CAC5B3F5EULL, 0x027C45979C952050ULL, 0x02647C69456217EDULL,
    0x02593F69B02593F7ULL, 0x0243F6F0243F6F03ULL, 0x0204081020408103ULL, 0x01F44659E4A42716ULL,
    0x01DE5D6E3F8868A5ULL, 0x01D77B654B82C33AULL, 0x01B7D6C3DDA338B3ULL, 0x01B2036406C80D91ULL,
    0x01A16D3F97A4B01BULL, 0x01920FB49D0E228EULL, 0x01886E5F0ABB049AULL, 0x017AD2208E0ECC36ULL,
    0x016E1F76B4337C6DULL, 0x016A13CD15372905ULL, 0x01571ED3C506B39BULL, 0x015390948F40FEADULL,
    0x014CAB88725AF6E8ULL, 0x0149539E3B2D066FULL, 0x013698DF3DE0747AULL, 0x0125E22708092F12ULL,
    0x0120B470C67C0D89ULL, 0x011E2EF3B3FB8745ULL, 0x0119453808CA29C1ULL, 0x0112358E75D30337ULL,
    0x010FEF010FEF0110ULL, 0x0105197F7D734042ULL, 0x00FF00FF00FF0100ULL, 0x00F92FB2211855A9ULL,
    0x00F3A0D52CBA8724ULL, 0x00F1D48BCEE0D39AULL, 0x00EC979118F3FC4EULL, 0x00E939651FE2D8D4ULL,
    0x00E79372E225FE31ULL, 0x00DFAC1F74346C58ULL, 0x00D578E97C3F5FE6ULL, 0x00D2BA083B445251ULL,
    0x00D161543E28E503ULL, 0x00CEBCF8BB5B416AULL, 0x00C5FE740317F9D1ULL, 0x00C2780613C0309FULL,
    0x00BCDD535DB1CC5CULL, 0x00BBC8408CD6306AULL, 0x00B9A7862A0FF466ULL, 0x00B68D31340E4308ULL,
    0x00B2927C29DA551AULL, 0x00AFB321A1496FE0ULL, 0x00ACEB0F891E6552ULL, 0x00AB1CBDD3E29710ULL,
    0x00A87917088E262CULL, 0x00A513FD6BB00A52ULL, 0x00A36E71A2CB0332ULL, 0x00A03C1688732B31ULL,
    0x009C69169B30446EULL, 0x009BAADE8E4A2F6FULL, 0x00980E4156201302ULL, 0x00975A750FF68A59ULL,
    0x009548E4979E082AULL, 0x0093EFD1C50E726CULL, 0x0091F5BCB8BB02DAULL, 0x008F67A1E3FDC262ULL,
    0x008E2917E0E702C7ULL, 0x008D8BE33F95D716ULL, 0x008C55841C815ED6ULL, 0x0088D180CD3A4134ULL,
    0x00869222B1ACF1CFULL, 0x0085797B917765ACULL, 0x008355ACE3C897DCULL, 0x00824A4E60B3262CULL,
    0x0080C121B28BD1BBULL, 0x007DC9F3397D4C2AULL, 0x007D4ECE8FE8813AULL, 0x0079237D65BCCE51ULL,
    0x0077CF53C5F7936DULL, 0x0075A8ACCFBDD11FULL, 0x007467AC557C228FULL, 0x00732D70ED8DB8EAULL,
    0x0072C62A24C37980ULL, 0x007194A17F55A10EULL, 0x006FA549B41DA7E8ULL, 0x006E8419E6F61222ULL,
    0x006D68B5356C207CULL, 0x006D0B803685C01CULL, 0x006BF790A8B2D208ULL, 0x006AE907EF4B96C3ULL,
    0x006A37991A23AEAEULL, 0x0069DFBDD4295B67ULL, 0x0067DC4C45C8033FULL, 0x00663D80FF99C280ULL,
    0x0065EC17E3559949ULL, 0x00654AC835CFBA5DULL, 0x00645C854AE10773ULL, 0x006372990E5F9020ULL,
    0x006325913C07BEF0ULL, 0x006160FF9E9F0062ULL, 0x0060CDB520E5E88FULL, 0x005FF4017FD00600ULL,
    0x005ED79E31A4DCCEULL, 0x005D7D42D48AC5F0ULL, 0x005C6F35CCBA5029ULL, 0x005B2618EC6AD0A6ULL,
};

// c_inv_primes[d] = 1.f / c_primes[d], rounded to nearest as the reference's
// `1.f / static_cast<float>(b)` is.
__constant__ float c_inv_primes[128] = {
    0x1.0000000000000p-1f, 0x1.5555560000000p-2f, 0x1.99999a0000000p-3f, 0x1.24924a0000000p-3f,
    0x1.745d180000000p-4f, 0x1.3b13b20000000p-4f, 0x1.e1e1e20000000p-5f, 0x1.af286c0000000p-5f,
    0x1.642c860000000p-5f, 0x1.1a7b960000000p-5f, 0x1.0842100000000p-5f, 0x1.bacf920000000p-6f,
    0x1.8f9c180000000p-6f, 0x1.7d05f40000000p-6f, 0x1.5c98820000000p-6f, 0x1.3521d00000000p-6f,
    0x1.15b1e60000000p-6f, 0x1.0c97140000000p-6f, 0x1.e9131a0000000p-7f, 0x1.cd85680000000p-7f,
    0x1.c0e0700000000p-7f, 0x1.9ec8ea0000000p-7f, 0x1.8acb900000000p-7f, 0x1.702e060000000p-7f,
    0x1.51d07e0000000p-7f, 0x1.446f860000000p-7f, 0x1.3e22cc0000000p-7f, 0x1.323e340000000p-7f,
    0x1.2c9fb40000000p-7f, 0x1.21fb780000000p-7f, 0x1.0204080000000p-7f, 0x1.f4465a0000000p-8f,
    0x1.de5d6e0000000p-8f, 0x1.d77b660000000p-8f, 0x1.b7d6c40000000p-8f, 0x1.b203640000000p-8f,
    0x1.a16d400000000p-8f, 0x1.920fb40000000p-8f, 0x1.886e600000000p-8f, 0x1.7ad2200000000p-8f,
    0x1.6e1f760000000p-8f, 0x1.6a13ce0000000p-8f, 0x1.571ed40000000p-8f, 0x1.5390940000000p-8f,
    0x1.4cab880000000p-8f, 0x1.49539e0000000p-8f, 0x1.3698e00000000p-8f, 0x1.25e2280000000p-8f,
    0x1.20b4700000000p-8f, 0x1.1e2ef40000000p-8f, 0x1.1945380000000p-8f, 0x1.12358e0000000p-8f,
    0x1.0fef020000000p-8f, 0x1.0519800000000p-8f, 0x1.fe01fe0000000p-9f, 0x1.f25f640000000p-9f,
    0x1.e741aa0000000p-9f, 0x1.e3a9180000000p-9f, 0x1.d92f220000000p-9f, 0x1.d272ca0000000p-9f,
    0x1.cf26e60000000p-9f, 0x1.bf583e0000000p-9f, 0x1.aaf1d20000000p-9f, 0x1.a574100000000p-9f,
    0x1.a2c2a80000000p-9f, 0x1.9d79f20000000p-9f, 0x1.8bfce80000000p-9f, 0x1.84f00c0000000p-9f,
    0x1.79baa60000000p-9f, 0x1.7790820000000p-9f, 0x1.734f0c0000000p-9f, 0x1.6d1a620000000p-9f,
    0x1.6524f80000000p-9f, 0x1.5f66440000000p-9f, 0x1.59d6200000000p-9f, 0x1.56397c0000000p-9f,
    0x1.50f22e0000000p-9f, 0x1.4a27fa0000000p-9f, 0x1.46dce40000000p-9f, 0x1.40782e0000000p-9f,
    0x1.38d22e0000000p-9f, 0x1.3755be0000000p-9f, 0x1.301c820000000p-9f, 0x1.2eb4ea0000000p-9f,
    0x1.2a91ca0000000p-9f, 0x1.27dfa40000000p-9f, 0x1.23eb7a0000000p-9f, 0x1.1ecf440000000p-9f,
    0x1.1c52300000000p-9f, 0x1.1b17c60000000p-9f, 0x1.18ab080000000p-9f, 0x1.11a3020000000p-9f,
    0x1.0d24460000000p-9f, 0x1.0af2f80000000p-9f, 0x1.06ab5a0000000p-9f, 0x1.04949c0000000p-9f,
    0x1.0182440000000p-9f, 0x1.f727cc0000000p-10f, 0x1.f53b3a0000000p-10f, 0x1.e48df60000000p-10f,
    0x1.df3d500000000p-10f, 0x1.d6a2b40000000p-10f, 0x1.d19eb20000000p-10f, 0x1.ccb5c40000000p-10f,
    0x1.cb18a80000000p-10f, 0x1.c652860000000p-10f, 0x1.be95260000000p-10f, 0x1.ba10680000000p-10f,
    0x1.b5a2d40000000p-10f, 0x1.b42e000000000p-10f, 0x1.afde420000000p-10f, 0x1.aba4200000000p-10f,
    0x1.a8de640000000p-10f, 0x1.a77ef80000000p-10f, 0x1.9f71320000000p-10f, 0x1.98f6040000000p-10f,
    0x1.97b0600000000p-10f, 0x1.952b200000000p-10f, 0x1.9172160000000p-10f, 0x1.8dca640000000p-10f,
    0x1.8c96440000000p-10f, 0x1.8583fe0000000p-10f, 0x1.8336d40000000p-10f, 0x1.7fd0060000000p-10f,
    0x1.7b5e780000000p-10f, 0x1.75f50c0000000p-10f, 0x1.71bcd80000000p-10f, 0x1.6c98640000000p-10f,
};

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
__device__ __forceinline__ float radical_inverse(uint32_t b, float invB, uint64_t magic, uint32_t n) {
    float invBN = 1.f, result = 0.f;
    while (n > 0) {
        const uint32_t q = uint32_t(__umul64hi(uint64_t(n), magic));
        uint32_t d = n - q * b;
        n = q;
        invBN = xmul(invBN, invB);
        result = xadd(result, xmul(__uint2float_rn(d), invBN));
    }
    return result;
}

// HaltonSampler::get1D for dimension dim of (px, py, sampleIndex).
// Out of line: the shading kernel draws about ten samples per vertex, and one
// shared copy of the digit loop instead of ten inlined ones took the
// 1920x1080x64 throughput frame's shade stage from 77.3 to 76.2 ms (the dome
// lookups out of line as well measured 78.4 ms).
__device__ __noinline__ float halton_sample(uint64_t seed, uint32_t px, uint32_t py,
                                               uint32_t sampleIndex, uint32_t dim) {
    if (dim < kHaltonDims) {
        uint64_t s = seed ^ (uint64_t(px) * 2654435761ULL) ^ (uint64_t(py) * 805459861ULL) ^
                     (uint64_t(dim) * 999999893ULL);
        uint32_t scramble = pcg_first(s);
        return radical_inverse(c_primes[dim], c_inv_primes[dim], c_magic[dim], sampleIndex ^ scramble);
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
