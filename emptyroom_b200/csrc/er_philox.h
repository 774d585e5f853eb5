// er_philox.h -- Philox4x32-10 counter-based generator, host and device.
//
// Written from Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as
// easy as 1, 2, 3" (SC'11): each round multiplies two counter words by the
// constants 0xD2511F53 / 0xCD9E8D57, swaps and xors the high halves with the
// key, and the key is bumped by the Weyl constants 0x9E3779B9 / 0xBB67AE85
// between rounds. It replaces the curand MTGP32 stream of src/henry.cu:111-126
// (seed 1234, 64 block states) with a stateless stream: insertion i of stream
// `seed` uses counters (i_lo, i_hi, 0, 0) and (i_lo, i_hi, 1, 0) under key
// (seed_lo, seed_hi), so any subset of insertions can be regenerated anywhere.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define ER_HD __host__ __device__ __forceinline__
#else
#define ER_HD inline
#endif

namespace er {

ER_HD void philox_mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#if defined(__CUDA_ARCH__)
    lo = a * b;
    hi = __umulhi(a, b);
#else
    uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
#endif
}

ER_HD void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        philox_mulhilo(0xD2511F53u, c0, hi0, lo0);
        philox_mulhilo(0xCD9E8D57u, c2, hi1, lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// 53 random bits -> [0, 1): (a >> 5) * 2^26 + (b >> 6), times 2^-53. Exact in double.
ER_HD double u53(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

ER_HD void insertion_point(uint64_t seed, uint64_t i, double out[3]) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t c[4] = {(uint32_t)i, (uint32_t)(i >> 32), 0u, 0u};
    uint32_t r[4], s[4];
    philox4x32_10(c, key, r);
    c[2] = 1u;
    philox4x32_10(c, key, s);
    out[0] = u53(r[0], r[1]);
    out[1] = u53(r[2], r[3]);
    out[2] = u53(s[0], s[1]);
}

}  // namespace er
