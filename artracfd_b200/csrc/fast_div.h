// Unsigned division by a divisor fixed at launch, as a multiply-high, a sum
// and a shift (the round-up method of Hacker's Delight, 2nd ed., 10-8): with
// l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
//     n / d = (umulhi(n, m) + n) >> l
// for every n < 2^32 when the sum is formed in 33 bits; kernels use it for
// n < 2^31, where the 32-bit sum cannot overflow.  A division by a run-time
// divisor costs about twenty instructions on the GPU, this one three.
// Host code builds the divisor (make_fast_div); both sides evaluate it.
#pragma once

#include <cstdint>

struct FastDiv {
    uint32_t m;  // multiplier, m < 2^32
    uint32_t l;  // shift, ceil(log2 d)
};

inline FastDiv make_fast_div(uint32_t d)
{
    uint32_t l = 0;
    while (l < 32 && (1ull << l) < d) ++l;
    const uint64_t m = (((1ull << 32) * ((1ull << l) - d)) / d) + 1;
    return FastDiv{(uint32_t)m, l};
}

#ifdef __CUDACC__
__host__ __device__
#endif
inline uint32_t fast_div(uint32_t n, FastDiv f)
{
#ifdef __CUDA_ARCH__
    const uint32_t t = __umulhi(n, f.m);
#else
    const uint32_t t = (uint32_t)(((uint64_t)n * f.m) >> 32);
#endif
    return (t + n) >> f.l;
}
