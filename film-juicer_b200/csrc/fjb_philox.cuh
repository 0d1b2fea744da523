// fjb_philox.cuh -- the counter-based generator shared by grain and scanner glare.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fjb {

// Philox4x32-10 (Salmon et al. 2011) in the openrand arrangement: key = seed hi/lo,
// counter = {ctr0, ctr1, global seed, draw index}, first output word per draw.
struct Philox {
    uint32_t k0, k1, c0, c1, c2, n;
    __device__ Philox(uint64_t seed, uint32_t ctr0, uint32_t global, uint32_t ctr1)
        : k0((uint32_t)(seed >> 32)), k1((uint32_t)seed), c0(ctr0), c1(ctr1), c2(global), n(0) {}
    __device__ __forceinline__ uint32_t next() {
        uint32_t x0 = c0, x1 = c1, x2 = c2, x3 = n;
        uint32_t a = k0, b = k1;
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            if (r > 0) {
                a += 0x9E3779B9u;
                b += 0xBB67AE85u;
            }
            const uint32_t hi0 = __umulhi(0xD2511F53u, x0), lo0 = 0xD2511F53u * x0;
            const uint32_t hi1 = __umulhi(0xCD9E8D57u, x2), lo1 = 0xCD9E8D57u * x2;
            const uint32_t y0 = hi1 ^ x1 ^ a, y2 = hi0 ^ x3 ^ b;
            x0 = y0;
            x1 = lo1;
            x2 = y2;
            x3 = lo0;
        }
        ++n;
        return x0;
    }
};

// Uniform in (0, 1) from one 32-bit draw: x 2^-32 + 2^-33 (the product is exact, so
// the fused multiply-add is too).
__device__ __forceinline__ float philox_u01(uint32_t x) {
    return __fmaf_rn((float)x, 1.0f / 4294967296.0f, 0.5f / 4294967296.0f);
}

} // namespace fjb
