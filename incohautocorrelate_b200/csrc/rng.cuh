// rng.cuh -- counter-based random numbers for the simulator.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): ten rounds of two 32x32->64-bit multiplies with a Weyl
// key schedule.  Counter = (index, stream), key = seed; every draw is a pure
// function of its coordinates, so results do not depend on launch geometry.
// The oracle (oracle/iac_oracle.c, iaco_philox4x32_10 / iaco_uniform_double)
// is the same function.
#pragma once

#include <cstdint>

namespace iac {

__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = (uint32_t)p1;
        c[2] = n2;
        c[3] = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Two uniform doubles in [0, 1) with 53 random bits each, from the block at
// counter (idx, stream) under key seed.
__host__ __device__ __forceinline__ void uniform2(uint64_t seed, uint64_t stream, uint64_t idx,
                                                  double &u0, double &u1)
{
    uint32_t c[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), (uint32_t)stream, (uint32_t)(stream >> 32)};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t w0 = ((uint64_t)c[0] << 32) | c[1];
    const uint64_t w1 = ((uint64_t)c[2] << 32) | c[3];
    u0 = (double)(w0 >> 11) * (1.0 / 9007199254740992.0);
    u1 = (double)(w1 >> 11) * (1.0 / 9007199254740992.0);
}

// stream tags (top byte of the 64-bit stream word)
constexpr uint64_t RNG_POISSON = 0x01ull << 56;
constexpr uint64_t RNG_ROTATION = 0x02ull << 56;
constexpr uint64_t RNG_PHASE = 0x03ull << 56;
constexpr uint64_t RNG_YIELD = 0x04ull << 56;
constexpr uint64_t RNG_NOISE = 0x05ull << 56;

}  // namespace iac
