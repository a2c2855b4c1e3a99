// msgpu_philox.h -- counter-based random numbers shared by host and device.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define MSGPU_HD __host__ __device__ __forceinline__
#else
#define MSGPU_HD
#endif

namespace msgpu {

// ------------------------------------------------------------ Philox4x32-10
// Counter-based generator of Salmon, Moraes, Dror & Shaw, "Parallel random
// numbers: as easy as 1, 2, 3" (SC'11), 10 rounds with the published
// multipliers and Weyl key increments.
struct u32x4 { uint32_t x, y, z, w; };

MSGPU_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo)
{
    const uint64_t p = static_cast<uint64_t>(a) * static_cast<uint64_t>(b);
    hi = static_cast<uint32_t>(p >> 32);
    lo = static_cast<uint32_t>(p);
}

MSGPU_HD u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(M0, c.x, hi0, lo0);
        mulhilo32(M1, c.z, hi1, lo1);
        c = u32x4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// Uniform double in [0,1) with 53 random bits from the first two words.
MSGPU_HD double philox_uniform53(u32x4 r)
{
    const uint64_t a = r.x >> 5, b = r.y >> 6;  // 27 + 26 bits
    return static_cast<double>((a << 26) | b) * (1.0 / 9007199254740992.0);
}

// Bernoulli draw of the singlet-triplet flip for (trajectory, global step,
// half step) under a 64-bit seed.  The counter never depends on launch order,
// so a trajectory sees the same noise alone or batched with other work.
MSGPU_HD bool philox_flip(uint64_t seed, uint32_t traj, uint32_t step, uint32_t half,
                                                     double p)
{
    const u32x4 r = philox4x32_10(u32x4{traj, step, half, 0x53544e31u},
                                  static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
    return philox_uniform53(r) < p;
}

}  // namespace msgpu
