// philox.h -- counter-based random numbers for field generation.
//
// Philox4x32 with 10 rounds, as published by Salmon, Moraes, Dror and Shaw,
// "Parallel random numbers: as easy as 1, 2, 3" (SC11): two 32x32->64-bit
// multiplies per round with multipliers 0xD2511F53 / 0xCD9E8D57 and a Weyl
// key schedule 0x9E3779B9 / 0xBB67AE85. The same integer stream is produced
// on the host and on the device; doubles take 53 bits from two words and
// Gaussians use the Box-Muller transform.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace plqcd {

constexpr uint32_t kTagSpinor = 0x53500000u;
constexpr uint32_t kTagGauge = 0x47410000u;

struct u32x4 {
    uint32_t v[4];
};

__host__ __device__ inline void philox_mul(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
    uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

__host__ __device__ inline u32x4 philox4x32_10(u32x4 ctr, uint32_t k0, uint32_t k1) {
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int r = 0; r < 10; r++) {
        uint32_t hi0, lo0, hi1, lo1;
        philox_mul(0xD2511F53u, ctr.v[0], hi0, lo0);
        philox_mul(0xCD9E8D57u, ctr.v[2], hi1, lo1);
        u32x4 n;
        n.v[0] = hi1 ^ ctr.v[1] ^ k0;
        n.v[1] = lo1;
        n.v[2] = hi0 ^ ctr.v[3] ^ k1;
        n.v[3] = lo0;
        ctr = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return ctr;
}

__host__ __device__ inline double u01_from(uint32_t a, uint32_t b) {
    // 53 random bits -> [0, 1)
    return (double)(((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6)) * (1.0 / 9007199254740992.0);
}

// Two independent N(0,1) numbers for (seed, site, stream, index).
__host__ __device__ inline double2 philox_gaussian_pair(uint64_t seed, uint64_t site, uint32_t stream,
                                                        uint32_t index) {
    u32x4 c;
    c.v[0] = (uint32_t)site;
    c.v[1] = (uint32_t)(site >> 32);
    c.v[2] = stream;
    c.v[3] = index;
    u32x4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    double u1 = 1.0 - u01_from(r.v[0], r.v[1]);  // (0, 1]
    double u2 = u01_from(r.v[2], r.v[3]);
    double rad = sqrt(-2.0 * log(u1));
    double s, co;
#ifdef __CUDA_ARCH__
    sincospi(2.0 * u2, &s, &co);
#else
    s = sin(2.0 * 3.14159265358979323846 * u2);
    co = cos(2.0 * 3.14159265358979323846 * u2);
#endif
    return make_double2(rad * co, rad * s);
}

}  // namespace plqcd
