/*
 * Test infrastructure (oracle side): counter-based Poisson draws.
 *
 * Philox4x32-10 as published by Salmon, Moraes, Dror and Shaw, "Parallel
 * random numbers: as easy as 1, 2, 3" (SC'11), restated from the paper.
 * It replaces the reference's per-neuron cuRAND XORWOW state
 * (src/simulator/mgsim/adj/mgcore.cu:123 curand_uniform, :449-455 curand_init)
 * so that the oracle, the shimmed reference kernels and the CUDA core draw
 * the same number for (seed, neuron, step).
 *
 * Counter layout (shared contract with mgbrain_b200/csrc/philox.cuh):
 *   key     = (seed & 0xffffffff, seed >> 32)
 *   counter = (step & 0xffffffff, step >> 32, neuron >> 2, MGB_TAG_POISSON)
 *   word    = neuron & 3
 *   u       = ((word >> 8) + 1) * 2^-24          in (0, 1], exact in fp32
 * A POISSON neuron fires when rate > u (mgcore.cu:124).
 *
 * Usable from C (oracle), C++ and CUDA device code (reference shim).
 */
#ifndef MGB_PHILOX_H
#define MGB_PHILOX_H
#include <stdint.h>

#if defined(__CUDACC__)
#define MGB_HD __host__ __device__ __forceinline__
#else
#define MGB_HD static inline
#endif

#define MGB_PHILOX_M0 0xD2511F53u
#define MGB_PHILOX_M1 0xCD9E8D57u
#define MGB_PHILOX_W0 0x9E3779B9u
#define MGB_PHILOX_W1 0xBB67AE85u
#define MGB_TAG_POISSON 0x504F4953u /* "POIS" */

typedef struct { uint32_t v[4]; } mgb_u32x4;

MGB_HD mgb_u32x4 mgb_philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                   uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)MGB_PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)MGB_PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += MGB_PHILOX_W0;
        k1 += MGB_PHILOX_W1;
    }
    mgb_u32x4 out;
    out.v[0] = c0; out.v[1] = c1; out.v[2] = c2; out.v[3] = c3;
    return out;
}

/* u32 -> (0,1] float, exact: an integer in [1, 2^24] times 2^-24. */
MGB_HD float mgb_u32_to_unit(uint32_t x)
{
    return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f);
}

MGB_HD float mgb_poisson_uniform(uint64_t seed, int64_t neuron, int64_t step)
{
    uint64_t st = (uint64_t)step;
    mgb_u32x4 r = mgb_philox4x32_10((uint32_t)st, (uint32_t)(st >> 32),
                                    (uint32_t)((uint64_t)neuron >> 2), MGB_TAG_POISSON,
                                    (uint32_t)seed, (uint32_t)(seed >> 32));
    return mgb_u32_to_unit(r.v[neuron & 3]);
}

#endif
