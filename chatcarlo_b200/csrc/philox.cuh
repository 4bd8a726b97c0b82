// Philox4x32-10 counter-based generator (J.K. Salmon, M.A. Moraes,
// R.O. Dror, D.E. Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11).  Each photon history owns the stream keyed by the run seed with
// the history index in the upper counter words, so any history can be
// replayed independently of launch shape and of every other history.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define CC_HD __host__ __device__ __forceinline__
#define CC_HD_NOINLINE __host__ __device__ __noinline__
#else
#define CC_HD inline
#define CC_HD_NOINLINE inline
#endif

namespace cc {

struct u32x4 { uint32_t x, y, z, w; };

CC_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#ifdef __CUDA_ARCH__
    hi = __umulhi(a, b);
    lo = a * b;
#else
    uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
#endif
}

// Round multipliers and Weyl increments of Philox4x32 from the SC'11 paper.
constexpr uint32_t PHILOX_M0 = 0xD2511F53u;
constexpr uint32_t PHILOX_M1 = 0xCD9E8D57u;
constexpr uint32_t PHILOX_W0 = 0x9E3779B9u;
constexpr uint32_t PHILOX_W1 = 0xBB67AE85u;

CC_HD u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(PHILOX_M0, c.x, hi0, lo0);
        mulhilo32(PHILOX_M1, c.z, hi1, lo1);
        u32x4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
    return c;
}

// One counter block, kept out of line: the generator is drawn from at many
// places of the transport kernel and each inlined copy of the ten rounds
// would cost instruction-cache space.
CC_HD_NOINLINE u32x4 philox_block(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                  uint32_t k1) {
    u32x4 c = {c0, c1, c2, c3};
    return philox4x32_10(c, k0, k1);
}

// (0, 1] with 2^-32 resolution; safe for -log().
CC_HD float u01_oc(uint32_t x) { return ((float)x + 1.0f) * 2.3283064365386963e-10f; }

// Per-history stream: counter = (draw block, stream tag, history lo, history hi).
struct HistoryRng {
    uint32_t k0, k1;       // seed
    uint32_t h0, h1;       // history index
    uint32_t block;        // next counter block
    uint32_t tag;          // stream tag (0 = transport)
    u32x4 buf;
    int avail;

    CC_HD void init(uint64_t seed, uint64_t history, uint32_t stream_tag) {
        k0 = (uint32_t)seed;
        k1 = (uint32_t)(seed >> 32);
        h0 = (uint32_t)history;
        h1 = (uint32_t)(history >> 32);
        block = 0;
        tag = stream_tag;
        avail = 0;
    }
    CC_HD uint32_t next_u32() {
        if (avail == 0) {
            buf = philox_block(block, tag, h0, h1, k0, k1);
            ++block;
            avail = 4;
        }
        uint32_t r;
        switch (avail) {
            case 4: r = buf.x; break;
            case 3: r = buf.y; break;
            case 2: r = buf.z; break;
            default: r = buf.w; break;
        }
        --avail;
        return r;
    }
    CC_HD float uniform() { return u01_oc(next_u32()); }   // (0, 1]
    // the same draw as an FP64 uniform in (0, 1] (exact: 32 bits fit a double)
    CC_HD double uniform_d() { return ((double)next_u32() + 1.0) * 2.3283064365386963e-10; }
};

}  // namespace cc
