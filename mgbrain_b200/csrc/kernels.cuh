// Device kernels of the simulation core (sm_100a).
//
// One simulation step is two or three launches on the handle's stream:
//   k_neuron  neuron update of every neuron + spike compaction
//   k_push    event delivery from the spiking rows into the delay ring
//   k_stdp    (Config::STDP) weight update over the spikers' rows
// The step number lives in device memory and the last block of the step's
// last kernel advances it, so the launch sequence of every step is
// identical and a run of steps can be captured once as a CUDA graph and
// replayed.
//
// Arithmetic follows the reference kernels operation by operation
// (src/simulator/mgsim/adj/mgcore.cu); the library is compiled with
// --fmad=false and the float expressions use explicit round-to-nearest
// intrinsics, so nothing is contracted into an fma.
#pragma once
#include <cstdint>

#include "philox.cuh"

namespace mgc {

enum : int { kRAW = 0, kLIF0 = 1, kPOISSON = 2, kLIF = 3, kLIFE = 4, kLIFB = 5 };

// Device status bits, read back by mgc_sync / mgc_read_raster.
enum : int { kStatusRasterIds = 1, kStatusRasterSteps = 2 };

constexpr int kNeuronBlock = 256;
constexpr int kPushBlock = 256;
constexpr int kChunk = 128;           // synapses per warp task (4 per lane)

struct StepArgs {
    int32_t n;            // neurons
    int32_t M;            // ring slots = max_delay + 1
    int32_t tbits;        // target bits in a packed CSR word
    uint32_t tmask;
    uint64_t seed;        // POISSON draw key
    int32_t refrac_steps; // round(t_ref/DT) - 1, mgcore.cu:184
    float lifb_leak;      // 0.005f (mgcore.cu:190) unless lifconst[9] != 0
    float C[30];          // LIFECONSTS
    float P[6];           // STDPCONSTS
    int32_t chunks_per_spike;
    int32_t stdp;
    int32_t record;       // raster recording on
    // neuron state
    const int8_t* type;
    const float* rate;
    float* V;
    float* Iexc;
    float* Iinh;
    int32_t* refrac;
    int32_t* last_fired;
    int32_t* fire_cnt;
    float* ring_e;        // [M][n]
    float* ring_i;        // [M][n]
    // synapses: CSR by source; word .x = target | delay << tbits, .y = weight bits
    const int64_t* row_ptr;
    uint2* syn;
    const int32_t* csr_src;   // STDP only
    const uint8_t* plastic;   // STDP only, may be null (all plastic)
    const int64_t* dend_off;  // STDP only: incoming lists
    const int64_t* dend_pos;  //   (CSR positions)
    // step bookkeeping
    int32_t* spk;             // spike ids of the current step
    int32_t* spk_count;
    int64_t* step;
    unsigned int* done;       // blocks finished in the step's last kernel
    unsigned long long* events;
    int32_t* raster_ids;
    int64_t raster_ids_cap;
    int32_t* raster_counts;
    int64_t raster_steps_cap;
    int64_t* raster_pos;
    int64_t* raster_step0;
    int32_t* status;
};

__device__ __forceinline__ float as_f(uint32_t u) { return __uint_as_float(u); }
__device__ __forceinline__ uint32_t as_u(float f) { return __float_as_uint(f); }

// ---------------------------------------------------------------------------
// Step epilogue: run by the last block to finish the step's last kernel.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool last_block(unsigned int* done)
{
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int prev = atomicAdd(done, 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    return is_last;
}

__device__ __forceinline__ void step_epilogue(const StepArgs& a)
{
    if (threadIdx.x != 0) return;
    __threadfence();
    const int64_t s = *a.step;
    const int32_t nspk = *(volatile int32_t*)a.spk_count;
    if (a.record) {
        const int64_t idx = s - *a.raster_step0;
        if (idx < a.raster_steps_cap)
            a.raster_counts[idx] = nspk;
        else
            atomicOr(a.status, kStatusRasterSteps);
        const int64_t pos = *a.raster_pos;
        if (pos + nspk > a.raster_ids_cap) atomicOr(a.status, kStatusRasterIds);
        *a.raster_pos = pos + nspk;
    }
    *a.spk_count = 0;
    *a.done = 0;
    __threadfence();
    *a.step = s + 1;
}

// ---------------------------------------------------------------------------
// Neuron update, mgsim_neus_core (mgcore.cu:116-234), plus compaction of
// the spiking ids (warp ballot, one atomic per warp).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kNeuronBlock) k_neuron(StepArgs a)
{
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t s = *a.step;
    bool fired = false;
    if (i < a.n) {
        const int t = a.type[i];
        if (t == kPOISSON) {
            // mgcore.cu:121-131
            const float u = poisson_uniform(a.seed, i, s);
            fired = a.rate[i] > u;
            if (fired) {
                a.fire_cnt[i] += 1;
                a.last_fired[i] = (int32_t)s;
            }
        } else if (t == kLIF || t == kLIFB || t == kLIFE) {
            const int32_t slot = (int32_t)(s % a.M);
            const size_t loc = (size_t)slot * (size_t)a.n + (size_t)i;
            const float re = a.ring_e[loc];
            const float ri = a.ring_i[loc];
            // every LIF-family path clears slot s%M (getInput/clearInput, :94-103)
            a.ring_e[loc] = 0.0f;
            a.ring_i[loc] = 0.0f;
            int32_t rf = a.refrac[i];
            float v = a.V[i];
            if (t == kLIFB) {
                // mgcore.cu:164-196: threshold on the old V, then leak + input
                if (rf > 0) {
                    --rf;
                } else if (v >= a.C[4]) {
                    fired = true;
                    v = a.C[3];
                    rf = a.refrac_steps;
                } else {
                    const float in = __fadd_rn(re, ri);
                    const float lk = __fmul_rn(a.lifb_leak, v);
                    v = __fadd_rn(v, __fsub_rn(in, lk));
                }
            } else if (t == kLIF) {
                // mgcore.cu:132-163: exponential integration, then threshold
                if (rf > 0) {
                    --rf;
                } else {
                    float ie = a.Iexc[i], ii = a.Iinh[i];
                    float nv = __fmul_rn(a.C[17], v);
                    nv = __fadd_rn(nv, a.C[14]);
                    nv = __fadd_rn(nv, __fmul_rn(ie, a.C[12]));
                    nv = __fadd_rn(nv, __fmul_rn(ii, a.C[13]));
                    ie = __fmul_rn(ie, a.C[15]);
                    ii = __fmul_rn(ii, a.C[16]);
                    if (nv >= a.C[4]) {
                        fired = true;
                        nv = a.C[3];
                        rf = a.refrac_steps;
                    } else {
                        ie = __fadd_rn(ie, re);
                        ii = __fadd_rn(ii, ri);
                    }
                    v = nv;
                    a.Iexc[i] = ie;
                    a.Iinh[i] = ii;
                }
            } else {
                // LIFE, mgcore.cu:197-233: conductances decay every step
                const float ie = __fadd_rn(re, __fmul_rn(a.Iexc[i], 0.98f));
                const float ii = __fadd_rn(-ri, __fmul_rn(a.Iinh[i], 0.99f));
                a.Iexc[i] = ie;
                a.Iinh[i] = ii;
                if (rf > 0) {
                    --rf;
                } else if (v >= a.C[4]) {
                    fired = true;
                    v = a.C[3];
                    rf = a.refrac_steps;
                } else {
                    float sum = __fsub_rn(-0.06f, v);
                    sum = __fadd_rn(sum, __fmul_rn(ie, __fsub_rn(0.0f, v)));
                    sum = __fadd_rn(sum, __fmul_rn(ii, __fsub_rn(-0.08f, v)));
                    sum = __fadd_rn(sum, 0.02f);
                    v = __fadd_rn(v, __fmul_rn(sum, 0.005f));
                }
            }
            if (fired) {
                a.fire_cnt[i] += 1;
                a.last_fired[i] = (int32_t)s;
            }
            a.V[i] = v;
            a.refrac[i] = rf;
        }
        // RAW and LIF0 have no branch in the reference: never update, never fire.
    }
    const unsigned int m = __ballot_sync(0xffffffffu, fired);
    if (m) {
        const int lane = threadIdx.x & 31;
        int32_t base = 0;
        if (lane == 0) base = atomicAdd(a.spk_count, __popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (fired) a.spk[base + __popc(m & ((1u << lane) - 1u))] = i;
    }
}

// ---------------------------------------------------------------------------
// Event push, mgsim_syn_fast_core + pushInnerSpike (mgcore.cu:271-305,
// :112-115): every synapse of a spiking neuron adds its weight to
// ring[(s + delay) % M][target], the exc ring when weight > 0, else inh.
// Work unit: one warp per (spike, 128-synapse chunk of its row).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kPushBlock) k_push(StepArgs a)
{
    const int64_t s = *a.step;
    const int32_t cnt = *(volatile int32_t*)a.spk_count;
    const int32_t slot0 = (int32_t)(s % a.M);
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t tasks = (int64_t)cnt * a.chunks_per_spike;
    unsigned long long ev = 0;
    const int64_t rpos = a.record ? *a.raster_pos : 0;
    for (int64_t task = warp; task < tasks; task += nwarps) {
        const int32_t j = (int32_t)(task / a.chunks_per_spike);
        const int32_t c = (int32_t)(task - (int64_t)j * a.chunks_per_spike);
        const int32_t nid = a.spk[j];
        if (c == 0 && lane == 0 && a.record && rpos + j < a.raster_ids_cap) a.raster_ids[rpos + j] = nid;
        const int64_t rb = a.row_ptr[nid], re = a.row_ptr[nid + 1];
        const int64_t b = rb + (int64_t)c * kChunk;
        if (b >= re) continue;
        const int64_t e = min(re, b + (int64_t)kChunk);
        if (lane == 0) ev += (unsigned long long)(e - b);
        uint2 w[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t k = b + lane + 32 * u;
            w[u] = k < e ? a.syn[k] : make_uint2(0u, 0u);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (b + lane + 32 * u >= e) continue;
            const uint32_t tgt = w[u].x & a.tmask;
            int32_t slot = slot0 + (int32_t)(w[u].x >> a.tbits);
            if (slot >= a.M) slot -= a.M;
            const float wt = as_f(w[u].y);
            float* ring = wt > 0.0f ? a.ring_e : a.ring_i;
            atomicAdd(ring + (size_t)slot * (size_t)a.n + tgt, wt);
        }
    }
    if (lane == 0 && ev) atomicAdd(a.events, ev);
    if (!a.stdp) {
        if (last_block(a.done)) step_epilogue(a);
    }
}

// stdp_cal_weight, mgcore.cu:346-364 (dt in steps, nearest-spike pairing).
__device__ __forceinline__ float stdp_weight(int32_t dt, float w, const float* P)
{
    float dw = 0.0f;
    if (dt < 0)
        dw = __fmul_rn(P[0], expf(__fdiv_rn((float)dt, P[2])));
    else if (dt > 0)
        dw = __fmul_rn(P[1], expf(__fdiv_rn((float)(-dt), P[3])));
    float nw = __fadd_rn(w, dw);
    nw = (nw > P[4]) ? P[4] : ((nw < P[5]) ? P[5] : nw);
    return nw;
}

// ---------------------------------------------------------------------------
// STDP, mgsim_stdp_core (mgcore.cu:365-412): for each spiking neuron its
// outgoing synapses (dt = last_fired[self] - last_fired[target]) then its
// incoming ones (dt = last_fired[source] - last_fired[self]).  A synapse is
// touched by two warps only when both ends spiked this step; then dt = 0
// on both sides and both store the same clipped weight.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kPushBlock) k_stdp(StepArgs a)
{
    const int32_t cnt = *(volatile int32_t*)a.spk_count;
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t j = warp; j < cnt; j += nwarps) {
        const int32_t nid = a.spk[j];
        const int32_t lfn = a.last_fired[nid];
        for (int64_t k = a.row_ptr[nid] + lane; k < a.row_ptr[nid + 1]; k += 32) {
            if (a.plastic && !a.plastic[k]) continue;
            const uint2 e = a.syn[k];
            const int32_t dt = lfn - a.last_fired[e.x & a.tmask];
            a.syn[k].y = as_u(stdp_weight(dt, as_f(e.y), a.P));
        }
        for (int64_t q = a.dend_off[nid] + lane; q < a.dend_off[nid + 1]; q += 32) {
            const int64_t k = a.dend_pos[q];
            if (a.plastic && !a.plastic[k]) continue;
            const int32_t dt = a.last_fired[a.csr_src[k]] - lfn;
            a.syn[k].y = as_u(stdp_weight(dt, as_f(a.syn[k].y), a.P));
        }
    }
    if (last_block(a.done)) step_epilogue(a);
}

}  // namespace mgc
