// Counter-based random numbers for the simulation core.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11).  Stateless: a POISSON neuron's draw at a step is
// a pure function of (seed, neuron, step), which is what lets a run be split,
// resumed, captured in a graph or replayed and still draw the same numbers.
// It replaces the reference's per-neuron XORWOW state
// (src/simulator/mgsim/adj/mgcore.cu:123 curand_uniform, :449-455
// curand_init).
//
// Counter layout:
//   key     = (seed lo, seed hi)
//   counter = (step lo, step hi, neuron >> 2, TAG)   word = neuron & 3
//   u       = ((word >> 8) + 1) * 2^-24 in (0, 1], exact in fp32
#pragma once
#include <cstdint>

namespace mgc {

constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;
constexpr uint32_t kTagPoisson = 0x504F4953u;  // "POIS"
constexpr uint32_t kTagConn = 0x434F4E4Eu;     // "CONN"

struct U32x4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ U32x4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                        uint32_t c3, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        const uint32_t hi0 = __umulhi(kPhiloxM0, c0), lo0 = kPhiloxM0 * c0;
        const uint32_t hi1 = __umulhi(kPhiloxM1, c2), lo1 = kPhiloxM1 * c2;
#else
        const uint64_t p0 = (uint64_t)kPhiloxM0 * c0, p1 = (uint64_t)kPhiloxM1 * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
    }
    return U32x4{c0, c1, c2, c3};
}

__host__ __device__ __forceinline__ uint32_t pick(const U32x4& r, int i)
{
    return i == 0 ? r.x : (i == 1 ? r.y : (i == 2 ? r.z : r.w));
}

// (0, 1] with 24 random bits: an integer in [1, 2^24] scaled by 2^-24.
__host__ __device__ __forceinline__ float unit_open0(uint32_t x)
{
    return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f);
}

__host__ __device__ __forceinline__ float poisson_uniform(uint64_t seed, int64_t neuron, int64_t step)
{
    const uint64_t st = (uint64_t)step;
    const U32x4 r = philox4x32_10((uint32_t)st, (uint32_t)(st >> 32), (uint32_t)((uint64_t)neuron >> 2),
                                  kTagPoisson, (uint32_t)seed, (uint32_t)(seed >> 32));
    return unit_open0(pick(r, (int)(neuron & 3)));
}

// The draws of four consecutive neurons first, first+1, .., first+3 at a
// step, equal to poisson_uniform of each: one Philox block when the four
// share one (first % 4 == 0), else two.
__host__ __device__ __forceinline__ void poisson_uniform4(uint64_t seed, int64_t first, int64_t step, float u[4])
{
    const uint64_t st = (uint64_t)step;
    const uint32_t blk = (uint32_t)((uint64_t)first >> 2);
    const int off = (int)(first & 3);
    U32x4 r = philox4x32_10((uint32_t)st, (uint32_t)(st >> 32), blk, kTagPoisson, (uint32_t)seed,
                            (uint32_t)(seed >> 32));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int w = off + k;
        if (w == 4)  // the next neurons' block
            r = philox4x32_10((uint32_t)st, (uint32_t)(st >> 32), blk + 1u, kTagPoisson, (uint32_t)seed,
                              (uint32_t)(seed >> 32));
        u[k] = unit_open0(pick(r, w & 3));
    }
}

// Draw for synapse k of target t in projection r of the fixed in-degree
// generator: x = source pick, y = delay pick.
__host__ __device__ __forceinline__ U32x4 conn_draw(uint64_t conn_seed, uint32_t t, uint32_t k, uint32_t r)
{
    return philox4x32_10(t, k, r, kTagConn, (uint32_t)conn_seed, (uint32_t)(conn_seed >> 32));
}

// floor(x * span / 2^32): an integer in [0, span).
__host__ __device__ __forceinline__ uint32_t scale_u32(uint32_t x, uint32_t span)
{
    return (uint32_t)(((uint64_t)x * (uint64_t)span) >> 32);
}

}  // namespace mgc
