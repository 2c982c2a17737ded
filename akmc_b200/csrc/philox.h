// Philox4x64-10 counter-based generator (Salmon, Moraes, Dror and Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC 2011) and the uniform doubles the library draws from it.
// The stream of key (k0, k1) and starting counter (c0, c1, 0, 0) is numpy.random.Philox's for
// the same key and counter: uniform q is word q % 4 of block q / 4, block b being the
// generator applied to the counter advanced by b + 1 (carry from the low word into the
// next); a uniform is the word's top 53 bits times 2^-53.
#pragma once

#include <cstdint>

namespace akmc {

// ten rounds of two 64x64 -> 128-bit multiplies with a Weyl key schedule
__device__ __forceinline__ void philox4x64_10(uint64_t c[4], uint64_t k0, uint64_t k1)
{
    const uint64_t M0 = 0xD2E7470EE14C6C93ull, M1 = 0xCA5A826395121157ull;
    const uint64_t W0 = 0x9E3779B97F4A7C15ull, W1 = 0xBB67AE8584CAA73Bull;
    #pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += W0;
            k1 += W1;
        }
        const uint64_t hi0 = __umul64hi(M0, c[0]), lo0 = M0 * c[0];
        const uint64_t hi1 = __umul64hi(M1, c[2]), lo1 = M1 * c[2];
        const uint64_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

// block b (four words) of the stream
__device__ __forceinline__ void philox_block(uint64_t k0, uint64_t k1, uint64_t c0, uint64_t c1,
                                             uint64_t b, uint64_t out[4])
{
    const uint64_t inc = b + 1;
    out[0] = c0 + inc;
    out[1] = c1 + (out[0] < inc ? 1 : 0);
    out[2] = 0;
    out[3] = 0;
    philox4x64_10(out, k0, k1);
}

__device__ __forceinline__ double philox_to_unit(uint64_t w) { return (double)(w >> 11) * 0x1.0p-53; }

// uniform q of the stream
__device__ __forceinline__ double philox_uniform(uint64_t k0, uint64_t k1, uint64_t c0, uint64_t c1, uint64_t q)
{
    uint64_t w[4];
    philox_block(k0, k1, c0, c1, q >> 2, w);
    return philox_to_unit(w[q & 3]);
}

}  // namespace akmc
