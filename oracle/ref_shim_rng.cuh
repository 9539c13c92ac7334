/*
 * Test infrastructure: force-included (nvcc -include) when the reference's
 * src/simulator/mgsim/adj/mgcore.cu is compiled into oracle/_ref/.
 * Replaces the XORWOW Poisson draws (mgcore.cu:123 curand_uniform,
 * :449-455 curand_init, :665-669 srand(time(0)); rand()) with the
 * counter-based draw of mgb_philox.h, so the reference kernels, the oracle
 * and the CUDA core see the same numbers.  The curandState keeps
 * d = neuron index (the subsequence curand_init receives), v[0..1] = seed,
 * v[2..3] = draws so far (= step, since a POISSON neuron draws every step).
 * The seed comes from MGB_REF_SEED.
 */
#pragma once
#include <vector>
#include <chrono>
#include <random>
#include <cstdlib>
#include <cstdio>
#include <ctime>
#include <algorithm>
#include <cmath>
#include <iostream>
#include <string>
#include <array>
#include <curand_kernel.h>
#include "mgb_philox.h"

static inline unsigned long mgb_ref_seed_value()
{
    const char* s = getenv("MGB_REF_SEED");
    return s ? strtoul(s, nullptr, 10) : 1UL;
}

__device__ __forceinline__ void mgb_ref_init(unsigned long long seed, unsigned long long sub,
                                             unsigned long long, curandStateXORWOW_t* st)
{
    st->d = (unsigned int)sub;
    st->v[0] = (unsigned int)seed;
    st->v[1] = (unsigned int)(seed >> 32);
    st->v[2] = 0;
    st->v[3] = 0;
    st->v[4] = 0;
}

__device__ __forceinline__ float mgb_ref_uniform(curandStateXORWOW_t* st)
{
    unsigned long long seed = (unsigned long long)st->v[0] | ((unsigned long long)st->v[1] << 32);
    unsigned long long n = (unsigned long long)st->v[2] | ((unsigned long long)st->v[3] << 32);
    float u = mgb_poisson_uniform(seed, (int64_t)st->d, (int64_t)n);
    ++n;
    st->v[2] = (unsigned int)n;
    st->v[3] = (unsigned int)(n >> 32);
    return u;
}

#define curand_init(seed, sub, off, st) mgb_ref_init((seed), (sub), (off), (st))
#define curand_uniform(st) mgb_ref_uniform(st)
#define rand() mgb_ref_seed_value()
