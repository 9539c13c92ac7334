// Device kernels of the simulation core (sm_100a).
//
// Two delivery methods compute the same input currents:
//  ring (immediate push; needed when weights are plastic):
//   k_neuron  neuron update reading ring slot s % M, spike compaction
//   k_push    event push from the spiking rows into ring slots (s+d) % M
//             (k_push_stdp with Config::STDP: push and both STDP sides)
//  deferred (static weights):
//   k_deliver events whose arrival step is s: for every delay d, the
//             spikes of step s-d push their delay-d row segment (rows are
//             bucketed by delay) into one accumulator per neuron, which
//             stays resident in L2 instead of an M-slot ring in HBM
//   k_neuron  neuron update reading and clearing the accumulators; spikes
//             go to the history slot s % H.
// A ring slot receives exactly the events whose arrival step is that of the
// slot (delays are 1..M-1), so both methods hand every neuron the same sum;
// with equal weights per sign the fp32 sums are identical in any order.
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
enum : int { kStatusRasterIds = 1, kStatusRasterSteps = 2, kStatusBarrier = 4, kStatusExchange = 8,
             kStatusBounds = 16 };

constexpr int kNeuronBlock = 256;
constexpr int kPushBlock = 256;
constexpr int kChunk = 128;           // synapses per warp task (4 per lane)
constexpr int kMaxBuckets = 2048;     // delay values the deferred method handles
constexpr int kTracePops = 4;         // schedule trace: populations counted per step
constexpr int kTraceCols = kTracePops + 1;  // ... plus the events delivered
constexpr int kTraceSteps = 1024;     // rows of the per-step trace ring

struct StepArgs {
    int32_t n;            // neurons
    int32_t ns;           // neuron arrays' length: n rounded up to a multiple of 4
    int32_t n_src;        // CSR rows (spike sources): n, or the whole network's neurons
                          // when this handle simulates one partition of it
    int32_t src_base;     // id of local neuron 0 in the spike history and raster
    int32_t deliver_blocks;  // fused step kernel: blocks that deliver
    int32_t M;            // ring slots = max_delay + 1
    int32_t tbits;        // target bits in a packed CSR word
    uint32_t tmask;
    uint64_t seed;        // POISSON draw key
    int32_t id_offset;    // added to neuron ids in the POISSON draws
    int32_t refrac_steps; // round(t_ref/DT) - 1, mgcore.cu:184
    float lifb_leak;      // 0.005f (mgcore.cu:190) unless lifconst[9] != 0
    float C[30];          // LIFECONSTS
    float P[6];           // STDPCONSTS
    int32_t chunks_per_spike;
    int32_t chunks_in_per_spike;  // ring method with STDP: 128-entry chunks of the longest incoming list
    int32_t has_cur;      // some neuron is LIF or LIFE: the update loads Iexc/Iinh with the group
                          // (k_fused is instantiated for each case)
    int32_t stdp;
    int32_t record;       // raster recording on
    int32_t deferred;     // deferred delivery (else ring)
    int32_t dmin;         // deferred: delay of bucket 0
    int32_t D;            //   number of delay buckets per row
    int32_t H;            //   history slots: dmax + max(4, longest window) (step groups clear the
                          //   slots of the next steps up to a window ahead)
    int32_t bucket_chunks;//   delivery tasks per (spike, delay) segment
    int32_t chunk_len;    //   synapses per task: segment positions [c*len, (c+1)*len)
    int32_t* hist_ids;    //   [H][n_src] spike ids per step
    int32_t* hist_cnt;    //   [H]
    const int64_t* bucket;   // [n_src*D + 1] CSR position of (source, bucket)
    float* acc_e;         //   [4 or 8][ns] input arriving at step s in buffer s & acc_mask
    float* acc_i;         //   (fixed-point accumulation: 64-bit integers, 8 bytes an entry)
    int32_t acc_mask;     //   3, or 7 while windows of more than 4 steps run (8 buffers allocated)
    int32_t fx;           // fixed-point accumulation (deferred and ring methods)
    float fx_scale;       //   2^fx_shift: a weight w is added as the integer rint(w * fx_scale)
    float fx_unscale;     //   2^-fx_shift: an input sum is float(sum) * fx_unscale
    int32_t pull;         // pull method (per-target pass at emission, STDP fused)
    uint32_t* fired_bits; //   [ns/32] spikes of the current step (also the ring method with STDP)
    const int64_t* in_ptr;//   [n+1] incoming rows (by target)
    uint2* in_ent;        //   [S] {source | delay << tbits, weight bits}, rows sorted by
                          //   (delay, source, synapse-list order)
    const uint8_t* in_plastic;  // [S] or null
    // neuron state
    const int8_t* type;
    const float* rate;    // POISSON per-step probabilities (staging; the update reads them from V)
    float* V;             // V; for POISSON neurons their probability
    float* Iexc;
    float* Iinh;
    int32_t* refrac;
    int32_t* last_fired;
    int32_t* fire_cnt;
    float* ring_e;        // [M][ns] (fixed-point accumulation: 64-bit integers)
    float* ring_i;        // [M][ns]
    // synapses: CSR by source; word .x = target | delay << tbits, .y = weight bits
    const int64_t* row_ptr;
    uint2* syn;
    int64_t n_syn;            // synapses in the CSR
    const int32_t* csr_src;   // STDP only
    const uint8_t* plastic;   // STDP only, may be null (all plastic)
    const int64_t* dend_off;  // STDP only: incoming lists
    const int64_t* dend_pos;  //   (CSR positions)
    // step bookkeeping
    int32_t* spk;             // spike ids of the current step
    int32_t* spk_count;
    int64_t* step;            // steps done; step[1] packs the slots below
    int32_t* slots;           // [0] = step % M (ring slot), [1] = step % H (history slot)
    unsigned int* done;       // blocks finished in the step's last kernel
    unsigned long long* events;
    int32_t* raster_ids;
    int64_t raster_ids_cap;
    int32_t* raster_counts;
    int64_t raster_steps_cap;
    int64_t* raster_pos;
    int64_t* raster_step0;
    int32_t* status;
    // schedule trace (fused method): row s % kTraceSteps holds step s's spikes
    // per trace population and the events its kernel delivered
    const uint8_t* tpop;      // [ns] trace population of each neuron (< kTracePops)
    float* trace;             // [kTraceSteps][kTraceCols]
    unsigned long long* ev_mark;  // events counter at the previous step's end
    unsigned int* bar;        // [4] step-group barriers: arrivals + generation (k_steps, k_steps1),
                              //     phase arrival counters (k_pipe)
    // deferred method, pull steps of the windowed group (mgc_set_pull): the
    // incoming rows in_ptr / in_ent (by target, synapse-CSR order inside) and
    // the spikes of every history slot as a bitmap, which that group writes
    uint32_t* hist_bits;      // [H][bits_words] bit i of the slot: neuron i spiked at its step
    int32_t bits_words;       // words per slot (4 per 32 neuron groups)
    int32_t pull_min;         // a step whose arrivals come from at least this many (spike, delay)
                              //   pairs is delivered by pull (0: never)
    int64_t* bits_span;       // [2] the steps [from, end) whose bitmaps the group wrote, one run
                              //   of groups without other step forms between them
    int64_t upd_rot;          // windowed update without pull steps: the lane at position p of a
                              //   pass updates neuron group (p + upd_rot) mod groups
};

__device__ __forceinline__ float as_f(uint32_t u) { return __uint_as_float(u); }

// Checked build (-DMGC_CHECKED, the library libmgbrain_b200_checked.so): every
// index the kernels take from memory (a spike id, a CSR position, a target,
// a delay, a history slot) is tested before it is used; a failed test sets
// kStatusBounds, which mgc_sync reports, and the access is skipped.  In the
// normal build the tests compile away.
#ifdef MGC_CHECKED
#define MGC_OK_INDEX(cond) mgc_check_index(a, (cond))
__device__ __forceinline__ bool mgc_check_index(const struct StepArgs& a, bool ok);
#else
#define MGC_OK_INDEX(cond) true
#endif

// Fire-and-forget fp32 reduction into global memory (PTX red.add.f32: the
// same rounding and subnormal flushing as atomicAdd, but no value comes back,
// so the issuing warp never waits on it).
__device__ __forceinline__ void red_add(float* p, float v)
{
    asm volatile("red.relaxed.gpu.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ uint32_t as_u(float f) { return __float_as_uint(f); }

// The same reduction with an L2 evict-last hint: the deferred method's
// accumulators (a few MB per step buffer) keep their L2 lines while the
// synapse words stream through L2 evict-first, so a reduction finds its line
// in L2 instead of fetching the sector from DRAM.
__device__ __forceinline__ void red_add_keep(float* p, float v)
{
    asm volatile(
        "{\n\t.reg .b64 pol;\n\t"
        "createpolicy.fractional.L2::evict_last.b64 pol, 1.0;\n\t"
        "red.relaxed.gpu.global.add.L2::cache_hint.f32 [%0], %1, pol;\n\t}" ::"l"(p), "f"(v) : "memory");
}

// ---------------------------------------------------------------------------
// Fixed-point accumulation (FX), for networks in which some neuron receives
// unequal weights of one sign.  fp32 additions of unequal values depend on
// their order, and the order in which scattered reductions land is not
// fixed, so such a neuron's input would change in the last bits from run to
// run (the reference's atomicAdd, mgcore.cu:112-115, has the same property).
// Instead every weight is added as the integer rint(w * 2^shift) into a
// 64-bit accumulator: integer addition is associative, so the sum does not
// depend on the order, and the neuron update converts it to fp32 once
// (round to nearest) and scales it back by 2^-shift (exact).  The builder
// picks the shift so that every weight of the network is an exact multiple
// of 2^-shift whenever the sums still fit 63 bits; the input is then the
// exact sum of the arriving fp32 weights, rounded once.  Only the final
// sum must fit: partial sums that wrap cancel in two's complement.
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long to_fx(float w, float scale) { return __float2ll_rn(__fmul_rn(w, scale)); }
__device__ __forceinline__ float from_fx(long long x, float unscale) { return __fmul_rn(__ll2float_rn(x), unscale); }
__device__ __forceinline__ void red_add_fx(unsigned long long* p, long long v)
{
    asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void red_add_fx_keep(unsigned long long* p, long long v)
{
    asm volatile(
        "{\n\t.reg .b64 pol;\n\t"
        "createpolicy.fractional.L2::evict_last.b64 pol, 1.0;\n\t"
        "red.relaxed.gpu.global.add.L2::cache_hint.u64 [%0], %1, pol;\n\t}" ::"l"(p), "l"(v) : "memory");
}

// The accumulator entries of one step: fp32, or 64-bit fixed point.
template <bool FX> struct AccT { using type = float; };
template <> struct AccT<true> { using type = unsigned long long; };

// One group of four neurons' input of one step, loaded with the group
// (16-byte loads; two of them for fixed point) and read as fp32.
template <bool FX> struct In4;
template <> struct In4<false> {
    float4 v;
    __device__ __forceinline__ void zero() { v = make_float4(0.f, 0.f, 0.f, 0.f); }
    __device__ __forceinline__ void load(const void* base, int64_t g) { v = reinterpret_cast<const float4*>(base)[g]; }
    __device__ __forceinline__ float4 get(const StepArgs&) const { return v; }
    __device__ __forceinline__ static void clear(void* base, int64_t g)
    {
        reinterpret_cast<float4*>(base)[g] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
};
template <> struct In4<true> {
    longlong2 lo, hi;
    __device__ __forceinline__ void zero() { lo = hi = make_longlong2(0, 0); }
    __device__ __forceinline__ void load(const void* base, int64_t g)
    {
        lo = reinterpret_cast<const longlong2*>(base)[2 * g];
        hi = reinterpret_cast<const longlong2*>(base)[2 * g + 1];
    }
    __device__ __forceinline__ float4 get(const StepArgs& a) const
    {
        return make_float4(from_fx(lo.x, a.fx_unscale), from_fx(lo.y, a.fx_unscale), from_fx(hi.x, a.fx_unscale),
                           from_fx(hi.y, a.fx_unscale));
    }
    __device__ __forceinline__ static void clear(void* base, int64_t g)
    {
        reinterpret_cast<longlong2*>(base)[2 * g] = make_longlong2(0, 0);
        reinterpret_cast<longlong2*>(base)[2 * g + 1] = make_longlong2(0, 0);
    }
};

#ifdef MGC_CHECKED
__device__ __forceinline__ bool mgc_check_index(const StepArgs& a, bool ok)
{
    if (!ok) atomicOr(a.status, kStatusBounds);
    return ok;
}
#endif

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

__device__ __forceinline__ int32_t* step_count(const StepArgs& a, int32_t hslot)
{
    return a.deferred ? a.hist_cnt + hslot : a.spk_count;
}

__device__ __forceinline__ int32_t* step_ids(const StepArgs& a, int32_t hslot)
{
    return a.deferred ? a.hist_ids + (size_t)hslot * (size_t)a.n_src : a.spk;
}

__device__ __forceinline__ void step_epilogue(const StepArgs& a)
{
    if (threadIdx.x != 0) return;
    __threadfence();
    const int64_t s = *a.step;
    const int32_t slot = a.slots[0], hslot = a.slots[1];
    const int32_t nspk = *(volatile int32_t*)step_count(a, hslot);
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
    if (a.trace) {
        const unsigned long long ev = *(volatile unsigned long long*)a.events;
        a.trace[(s & (kTraceSteps - 1)) * kTraceCols + kTracePops] = (float)(ev - *a.ev_mark);
        *a.ev_mark = ev;
        float* nxt = a.trace + ((s + 1) & (kTraceSteps - 1)) * kTraceCols;
        for (int c = 0; c < kTraceCols; ++c) nxt[c] = 0.f;
    }
    const int32_t next_h = hslot + 1 == a.H ? 0 : hslot + 1;
    if (a.deferred)
        a.hist_cnt[next_h] = 0;  // held step s+1-H, no longer read
    else
        *a.spk_count = 0;
    *a.done = 0;
    a.slots[0] = slot + 1 == a.M ? 0 : slot + 1;
    a.slots[1] = next_h;
    __threadfence();
    *a.step = s + 1;
}

// ---------------------------------------------------------------------------
// Neuron update, mgsim_neus_core (mgcore.cu:116-234).  One thread updates a
// group of 4 consecutive neurons with 16-byte loads and stores (arrays are
// padded to a multiple of 4 with RAW neurons, which never change); spiking
// ids are compacted in neuron order within a warp, one atomic per warp.
// ---------------------------------------------------------------------------
// One neuron of a group; ie_io/ii_io (LIF and LIFE currents) were loaded
// with the group when the network has such neurons and are stored back with it.
// u: the neuron's POISSON draw of this step (poisson_uniform), computed for
// its group of four.
template <bool BOOK = true>
__device__ __forceinline__ bool update_one(const StepArgs& a, int t, int32_t i, int64_t s, float& v, int32_t& rf,
                                           float re, float ri, float& ie_io, float& ii_io, float u)
{
    bool fired = false;
    if (t == kPOISSON) {
        // mgcore.cu:121-131: fires when the per-step probability beats the
        // draw.  A POISSON neuron's V is never used, so its V slot holds the
        // probability (mgc_set_rates writes it there): it arrives with the
        // group's loads instead of a second, dependent load.
        fired = v > u;
    } else if (t == kLIFB) {
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
            float ie = ie_io, ii = ii_io;
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
            ie_io = ie;
            ii_io = ii;
        }
    } else if (t == kLIFE) {
        // mgcore.cu:197-233: conductances decay every step
        const float ie = __fadd_rn(re, __fmul_rn(ie_io, 0.98f));
        const float ii = __fadd_rn(-ri, __fmul_rn(ii_io, 0.99f));
        ie_io = ie;
        ii_io = ii;
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
    // RAW and LIF0 have no branch in the reference: never update, never fire.
    if (BOOK && fired) {
        atomicAdd(a.fire_cnt + i, 1);  // a reduction: the update does not wait on the count
        a.last_fired[i] = (int32_t)s;
    }
    return fired;
}

// update_one's LIFB branch without branches (the same operations, selected):
// the windowed group runs it for groups of four LIFB neurons, where the
// per-neuron type and refractory branches would otherwise split the warp.
// Returns whether the neuron fired; its fire count and last spike are the
// caller's to record.
__device__ __forceinline__ bool lifb_step(const StepArgs& a, float& v, int32_t& rf, float re, float ri)
{
    const bool ref = rf > 0;
    const bool fire = !ref && v >= a.C[4];
    const float nv = __fadd_rn(v, __fsub_rn(__fadd_rn(re, ri), __fmul_rn(a.lifb_leak, v)));
    v = ref ? v : (fire ? a.C[3] : nv);
    rf = ref ? rf - 1 : (fire ? a.refrac_steps : rf);
    return fire;
}

// Updates the neuron groups with a warp-strided loop; `warp`/`nwarps` index
// the warps taking part.  Each lane takes G groups per pass (groups
// gb + h*32 + lane, h < G), all of whose loads are issued before the first
// update, so a warp waits for memory once per pass.  Input of this step is
// read from (and cleared in) in_e/in_i, which point at the ring slot or the
// accumulator buffer.  Spiking ids are compacted in neuron order within the
// pass, one atomic per warp.
template <int G, bool CUR, bool FX>
__device__ __forceinline__ void neuron_groups(const StepArgs& a, int64_t s, int32_t hslot, void* in_e, void* in_i,
                                              int64_t warp, int64_t nwarps, int64_t rbase, int* pop_cnt = nullptr,
                                              bool raster = true)
{
    static_assert(G == 1 || G == 2, "one or two groups per lane");
    const int lane = threadIdx.x & 31;
    const int64_t ngroups = a.ns >> 2;
    int32_t* ids = step_ids(a, hslot);
    int32_t* cnt = step_count(a, hslot);
    const bool rec = raster && (a.deferred || a.pull) && a.record;  // no push kernel to record

    for (int64_t gb = warp * 32 * G; gb < ngroups; gb += nwarps * 32 * G) {
        char4 t4[G];
        float4 v4[G], ce4[G], ci4[G];
        In4<FX> e4[G], i4[G];
        int4 r4[G];
#pragma unroll
        for (int h = 0; h < G; ++h) {
            const int64_t g = gb + h * 32 + lane;
            ce4[h] = ci4[h] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (g < ngroups) {
                t4[h] = __ldg(reinterpret_cast<const char4*>(a.type) + g);
                v4[h] = reinterpret_cast<float4*>(a.V)[g];
                r4[h] = reinterpret_cast<int4*>(a.refrac)[g];
                e4[h].load(in_e, g);
                i4[h].load(in_i, g);
                if (CUR) {  // in flight with the rest of the group
                    ce4[h] = reinterpret_cast<float4*>(a.Iexc)[g];
                    ci4[h] = reinterpret_cast<float4*>(a.Iinh)[g];
                }
            }
        }
        unsigned fmask[G];
        unsigned lifbm = 0;  // bit h: pass h's group is four LIFB neurons (branch-free update)
#pragma unroll
        for (int h = 0; h < G; ++h) {
            const int64_t g = gb + h * 32 + lane;
            fmask[h] = 0;
            if (g < ngroups) {
                const int32_t i0 = (int32_t)(g << 2);
                const float4 e = e4[h].get(a), ii = i4[h].get(a);
                if (t4[h].x == kLIFB && t4[h].y == kLIFB && t4[h].z == kLIFB && t4[h].w == kLIFB) {
                    lifbm |= 1u << h;
                    fmask[h] |= lifb_step(a, v4[h].x, r4[h].x, e.x, ii.x) ? 1u : 0u;
                    fmask[h] |= lifb_step(a, v4[h].y, r4[h].y, e.y, ii.y) ? 2u : 0u;
                    fmask[h] |= lifb_step(a, v4[h].z, r4[h].z, e.z, ii.z) ? 4u : 0u;
                    fmask[h] |= lifb_step(a, v4[h].w, r4[h].w, e.w, ii.w) ? 8u : 0u;
                } else {
                    // one Philox block serves the group's four POISSON draws
                    float u[4] = {0.f, 0.f, 0.f, 0.f};
                    if (t4[h].x == kPOISSON || t4[h].y == kPOISSON || t4[h].z == kPOISSON || t4[h].w == kPOISSON)
                        poisson_uniform4(a.seed, (int64_t)i0 + a.id_offset, s, u);
                    fmask[h] |= update_one(a, t4[h].x, i0 + 0, s, v4[h].x, r4[h].x, e.x, ii.x, ce4[h].x, ci4[h].x, u[0]) ? 1u : 0u;
                    fmask[h] |= update_one(a, t4[h].y, i0 + 1, s, v4[h].y, r4[h].y, e.y, ii.y, ce4[h].y, ci4[h].y, u[1]) ? 2u : 0u;
                    fmask[h] |= update_one(a, t4[h].z, i0 + 2, s, v4[h].z, r4[h].z, e.z, ii.z, ce4[h].z, ci4[h].z, u[2]) ? 4u : 0u;
                    fmask[h] |= update_one(a, t4[h].w, i0 + 3, s, v4[h].w, r4[h].w, e.w, ii.w, ce4[h].w, ci4[h].w, u[3]) ? 8u : 0u;
                }
                // the input is cleared only after it was used: a store issued
                // while the load of the same line is in flight stalls the
                // memory pipeline (measured 4-6x slower once the state
                // leaves L2)
                In4<FX>::clear(in_e, g);
                In4<FX>::clear(in_i, g);
                reinterpret_cast<float4*>(a.V)[g] = v4[h];
                reinterpret_cast<int4*>(a.refrac)[g] = r4[h];
                if (CUR) {
                    reinterpret_cast<float4*>(a.Iexc)[g] = ce4[h];
                    reinterpret_cast<float4*>(a.Iinh)[g] = ci4[h];
                }
            }
            if (a.fired_bits) {
                // bitmap of this step's spikes (pull method, ring method with
                // STDP): 8 lanes (32 neurons) per word
                unsigned wv = fmask[h] << (4 * (lane & 7));
                wv |= __shfl_xor_sync(0xffffffffu, wv, 1);
                wv |= __shfl_xor_sync(0xffffffffu, wv, 2);
                wv |= __shfl_xor_sync(0xffffffffu, wv, 4);
                if ((lane & 7) == 0 && gb + h * 32 < ngroups) a.fired_bits[((gb + h * 32) >> 3) + (lane >> 3)] = wv;
            }
        }
        // compaction in neuron order: one warp scan of the per-pass counts
        // (pass h in bits 8h.., at most 128 spikes each); none when no lane
        // of the warp spiked (most passes of a quiet step)
        int c = 0;
#pragma unroll
        for (int h = 0; h < G; ++h) c |= __popc(fmask[h]) << (8 * h);
        if (!__any_sync(0xffffffffu, c != 0)) continue;
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int packed = __shfl_sync(0xffffffffu, incl, 31);
        int total = 0;
#pragma unroll
        for (int h = 0; h < G; ++h) total += (packed >> (8 * h)) & 0xff;
        if (total) {
            int32_t base = 0;
            if (lane == 31) base = atomicAdd(cnt, total);
            base = __shfl_sync(0xffffffffu, base, 31);
#pragma unroll
            for (int h = 0; h < G; ++h) {
                const int ch = (c >> (8 * h)) & 0xff;
                int32_t pos = base + ((incl >> (8 * h)) & 0xff) - ch;
                base += (packed >> (8 * h)) & 0xff;
                const int32_t i0 = (int32_t)((gb + h * 32 + lane) << 2);
                for (int k = 0; k < 4; ++k) {
                    if (fmask[h] & (1u << k)) {
                        if ((lifbm >> h) & 1u) {  // (update_one records the others' itself)
                            atomicAdd(a.fire_cnt + i0 + k, 1);
                            a.last_fired[i0 + k] = (int32_t)s;
                        }
                        if (!MGC_OK_INDEX(pos < (a.deferred ? a.n_src : a.n))) break;
                        ids[pos] = a.src_base + i0 + k;
                        if (pop_cnt) atomicAdd(pop_cnt + a.tpop[i0 + k], 1);
                        if (rec && rbase + pos < a.raster_ids_cap) a.raster_ids[rbase + pos] = a.src_base + i0 + k;
                        ++pos;
                    }
                }
            }
        }
    }
}

// Raster position of the current step's first spike id (when this kernel records).
__device__ __forceinline__ int64_t raster_base(const StepArgs& a)
{
    return (a.deferred || a.pull) && a.record ? *a.raster_pos : 0;
}

// Accumulator buffer of the input arriving at step s: four buffers in use
// (s & 3), so the pipelined step group can deliver two steps ahead while the
// oldest buffer is still being read, and a window of up to 4 steps holds its
// steps' inputs at once; eight (s & 7) while windows of 5 to 8 steps run.
// The eight are allocated only for a minimum delay >= 5; the smaller cycle is
// kept otherwise because it touches half the memory each 4 steps.
constexpr int kAccBuffers = 4;
constexpr int kAccBuffersWide = 8;

// MASK: the cycle when the kernel fixes it at compile time (the windowed
// groups: 3 up to 4 steps, 7 above; the host launches them only in that
// cycle), 0 for the handle's current one.
template <bool FX = false, int MASK = 0>
__device__ __forceinline__ typename AccT<FX>::type* acc_buf(const StepArgs& a, float* base, int64_t s)
{
    const int64_t m = MASK ? MASK : a.acc_mask;
    return reinterpret_cast<typename AccT<FX>::type*>(base) + (size_t)(s & m) * (size_t)a.ns;
}

template <bool FX>
__global__ void __launch_bounds__(kNeuronBlock) k_neuron(StepArgs a)
{
    const int64_t s = *a.step;
    const int32_t slot = a.slots[0], hslot = a.slots[1];
    void *in_e, *in_i;
    if (a.deferred) {
        in_e = acc_buf<FX>(a, a.acc_e, s);
        in_i = acc_buf<FX>(a, a.acc_i, s);
    } else {
        in_e = reinterpret_cast<typename AccT<FX>::type*>(a.ring_e) + (size_t)slot * (size_t)a.ns;
        in_i = reinterpret_cast<typename AccT<FX>::type*>(a.ring_i) + (size_t)slot * (size_t)a.ns;
    }
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    if (a.has_cur)
        neuron_groups<1, true, FX>(a, s, hslot, in_e, in_i, warp, nwarps, raster_base(a));
    else
        neuron_groups<1, false, FX>(a, s, hslot, in_e, in_i, warp, nwarps, raster_base(a));
    if (a.deferred) {
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

__device__ __forceinline__ bool bit_of(const uint32_t* bits, int32_t i) { return (bits[i >> 5] >> (i & 31)) & 1u; }

// ---------------------------------------------------------------------------
// Deferred delivery of the events that arrive at step sa: for each delay d
// of the buckets, the spikes of step sa-d send the delay-d segment of their
// row into the accumulator of step sa.  Task f enumerates (d, spike)
// through a prefix sum over the per-delay spike counts held in shared
// memory.  A warp takes up to 32 tasks at once: each lane fetches one segment
// header, a warp scan lays the 32 segments end to end, and the lanes then
// stride over the concatenated synapses (owner segment found by a 5-step
// shuffle search), so all synapse loads of the batch are independent and
// in flight together instead of one dependent chain per segment.
// ---------------------------------------------------------------------------
constexpr int kDeliverUnroll = 4;

// History slot of step sa, given the current step s and its slot.
__device__ __forceinline__ int32_t hist_slot(const StepArgs& a, int64_t sa, int64_t s, int32_t hslot)
{
    int32_t hs = hslot + (int32_t)(sa - s);
    return hs >= a.H ? hs - a.H : hs;
}

// pre[k] = spikes of the delays before bucket k that arrive at step sa
// (pre[D] = tasks in all); run by the block's first warp.
__device__ __forceinline__ void deliver_prefix(const StepArgs& a, int64_t sa, int64_t s, int32_t hslot, int64_t* pre)
{
    const int D = a.D;
    const int32_t hs = hist_slot(a, sa, s, hslot);
    const int lane = threadIdx.x & 31;
    int64_t carry = 0;
    if (lane == 0) pre[0] = 0;
    for (int base = 0; base < D; base += 32) {
        const int k = base + lane;
        int64_t c = 0;
        if (k < D && sa - (a.dmin + k) >= 0) {
            int32_t h = hs - (a.dmin + k);  // slot of step sa - d, d < H
            if (h < 0) h += a.H;
            c = (int64_t)a.hist_cnt[h];
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t v = __shfl_up_sync(0xffffffffu, c, o);
            if (lane >= o) c += v;
        }
        if (k < D) pre[k + 1] = carry + c;
        carry += __shfl_sync(0xffffffffu, c, 31);
    }
}

// The tasks themselves, after deliver_prefix and a block barrier.
// blk_ev: when given, the warps add their delivered events into this block
// counter (shared memory) instead of the global one.  NMAX > 1: the tasks of
// the n <= NMAX consecutive arrival steps sa, sa+1, ... as one task space
// (step k's prefixes at pre + k*(D+1)), so that a warp's lanes fetch the
// segments of several steps in one batch.  MASK: as for acc_buf.
template <bool FX, int NMAX = 1, int MASK = 0>
__device__ __forceinline__ void deliver_tasks(const StepArgs& a, int64_t sa, int64_t s, int32_t hslot,
                                              const int64_t* pre, int64_t warp, int64_t nwarps,
                                              unsigned long long* blk_ev = nullptr, int n = 1)
{
    const int D = a.D;
    const int CH = a.bucket_chunks;
    int64_t first[NMAX + 1];  // task offset of each step
    first[0] = 0;
#pragma unroll
    for (int k = 0; k < NMAX; ++k) first[k + 1] = first[k] + (k < n ? pre[(size_t)k * (D + 1) + D] * CH : 0);
    const int64_t total = first[NMAX];  // (spike, delay) segments x chunks
    const int lane = threadIdx.x & 31;
    unsigned long long ev = 0;
    // tasks per warp: 32, or fewer when the grid has more lanes than tasks,
    // so that a small step spreads over all warps instead of a few
    const int64_t need = (total + nwarps - 1) / nwarps;
    const int per = need >= 32 ? 32 : (need < 1 ? 1 : (int)need);
    // tasks start at the last warp: the neuron update gives the first warps
    // its extra passes, so a step with few tasks lands on the least busy ones
    const int64_t rw = nwarps - 1 - warp;
    for (int64_t fb = rw * per; fb < total; fb += nwarps * per) {
        // 1. this lane's segment header
        const int64_t f = fb + lane;
        int64_t b = 0;
        int32_t len = 0;
        int step = 0;  // arrival step sa + step of the lane's task
        if (lane < per && f < total) {
            int64_t f0 = 0;
#pragma unroll
            for (int k = 1; k < NMAX; ++k)
                if (f >= first[k]) {
                    step = k;
                    f0 = first[k];
                }
            const int64_t* pk = pre + (size_t)step * (D + 1);
            const int32_t hs = hist_slot(a, sa + step, s, hslot);
            const int64_t fl = f - f0;
            const int64_t fs = fl / CH;               // segment task
            const int32_t c = (int32_t)(fl - fs * CH);  // chunk of it
            int lo = 0, hi = D - 1;  // last k with pk[k] <= fs
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (pk[mid] <= fs) lo = mid; else hi = mid - 1;
            }
            const int k = lo;
            const int32_t j = (int32_t)(fs - pk[k]);
            int32_t h = hs - (a.dmin + k);
            if (h < 0) h += a.H;
            const int32_t src = a.hist_ids[(size_t)h * (size_t)a.n_src + j];
            if (MGC_OK_INDEX(h >= 0 && h < a.H && j < a.n_src && src >= 0 && src < a.n_src)) {
                const int64_t* bk = a.bucket + (size_t)src * D + k;  // segment [bk[0], bk[1])
                const int64_t b0 = __ldg(bk);
                const int64_t seg = __ldg(bk + 1) - b0;
                const int64_t c0 = (int64_t)c * a.chunk_len;
                if (MGC_OK_INDEX(b0 >= 0 && seg >= 0 && b0 + seg <= a.n_syn)) {
                    b = b0 + c0;
                    len = seg > c0 ? (int32_t)(seg - c0 < a.chunk_len ? seg - c0 : a.chunk_len) : 0;
                }
            }
        }
        // 2. segments end to end: exclusive offsets
        int32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int32_t excl = incl - len;
        const int32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        if (lane == 0) ev += (unsigned long long)tot;
        // 3. all lanes over the concatenated synapses
        for (int32_t base = 0; base < tot; base += 32 * kDeliverUnroll) {
            uint2 w[kDeliverUnroll];
            int st_of[kDeliverUnroll];
#pragma unroll
            for (int u = 0; u < kDeliverUnroll; ++u) {
                const int32_t idx = base + u * 32 + lane;
                int L = 0;  // last lane whose segment starts at or before idx
#pragma unroll
                for (int st = 16; st >= 1; st >>= 1) {
                    const int32_t e = __shfl_sync(0xffffffffu, excl, L + st);
                    if (e <= idx) L += st;
                }
                const int64_t bl = __shfl_sync(0xffffffffu, b, L);
                const int32_t el = __shfl_sync(0xffffffffu, excl, L);
                if (NMAX > 1) st_of[u] = __shfl_sync(0xffffffffu, step, L);
                w[u] = idx < tot ? __ldcs(a.syn + bl + (idx - el)) : make_uint2(0u, 0u);
            }
#pragma unroll
            for (int u = 0; u < kDeliverUnroll; ++u) {
                if (base + u * 32 + lane >= tot) continue;
                if (!MGC_OK_INDEX((w[u].x & a.tmask) < (uint32_t)a.ns)) continue;
                const float wt = as_f(w[u].y);
                const int64_t sx = sa + (NMAX > 1 ? st_of[u] : 0);
                if (FX)
                    red_add_fx_keep(acc_buf<true, MASK>(a, wt > 0.0f ? a.acc_e : a.acc_i, sx) + (w[u].x & a.tmask),
                                    to_fx(wt, a.fx_scale));
                else
                    red_add_keep(acc_buf<false, MASK>(a, wt > 0.0f ? a.acc_e : a.acc_i, sx) + (w[u].x & a.tmask), wt);
            }
        }
    }
    if (ev) atomicAdd(blk_ev ? blk_ev : a.events, ev);
}

template <bool FX>
__device__ __forceinline__ void deliver_arrivals(const StepArgs& a, int64_t sa, int64_t* pre, int64_t warp,
                                                 int64_t nwarps)
{
    const int64_t s = *a.step;
    const int32_t hslot = a.slots[1];
    if (threadIdx.x < 32) deliver_prefix(a, sa, s, hslot, pre);
    __syncthreads();
    deliver_tasks<FX>(a, sa, s, hslot, pre, warp, nwarps);
}

// Arrivals of the current step (used when the minimum delay is one step).
template <bool FX>
__global__ void __launch_bounds__(kPushBlock) k_deliver(StepArgs a)
{
    __shared__ int64_t pre[kMaxBuckets + 1];
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    deliver_arrivals<FX>(a, *a.step, pre, warp, nwarps);
}

// One launch per step when the minimum delay is >= 2: the arrivals of step
// s+1 depend only on spikes of steps <= s-1, so every warp updates its
// share of the neurons for step s and then delivers its share of those
// arrivals into the other accumulator buffer; the memory-latency chains of
// different warps overlap on each SM.
// MINB: resident blocks per SM the kernel is compiled for (its register
// budget); the schedule chooses between the instantiations.
template <bool CUR, int MINB, bool FX>
__global__ void __launch_bounds__(kPushBlock, MINB) k_fused(StepArgs a)
{
    __shared__ int64_t pre[kMaxBuckets + 1];
    __shared__ int pop_cnt[kTracePops];
    const int64_t s = *a.step;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    if (threadIdx.x < kTracePops) pop_cnt[threadIdx.x] = 0;
    __syncthreads();
    // the first warp sums the spike counts per delay while all warps update
    // their neurons; the barrier then publishes the sums for the delivery
    const int32_t hslot = a.slots[1];
    if (threadIdx.x < 32) deliver_prefix(a, s + 1, s, hslot, pre);
    neuron_groups<2, CUR, FX>(a, s, hslot, acc_buf<FX>(a, a.acc_e, s), acc_buf<FX>(a, a.acc_i, s), warp, nwarps, raster_base(a),
                          a.trace ? pop_cnt : nullptr);
    __syncthreads();
    if (a.trace && threadIdx.x < kTracePops && pop_cnt[threadIdx.x])
        atomicAdd(a.trace + (s & (kTraceSteps - 1)) * kTraceCols + threadIdx.x, (float)pop_cnt[threadIdx.x]);
    deliver_tasks<FX>(a, s + 1, s, hslot, pre, warp, nwarps);
    if (last_block(a.done)) step_epilogue(a);
}

// ---------------------------------------------------------------------------
// Persistent step group: the fused step for `nsteps` consecutive steps in
// one cooperative launch (all blocks resident), a grid barrier between
// steps.  Step, slots and raster position live in registers; block 0 keeps
// the bookkeeping the epilogue does (clearing the next history slot during
// the step, which no delivery of this step reads; recording the finished
// step after the barrier) and writes the clock back at the end.  Every
// barrier wait is bounded: on time-out the kernel sets kStatusBarrier and
// all blocks return.
// ---------------------------------------------------------------------------
constexpr unsigned int kBarrierSpins = 1u << 21;

// Arrivals count up on a.bar[0], which is cleared before every launch: a
// block's arrival returns the count before it, from which it knows the
// total that completes this barrier (the next multiple of gridDim.x), so the
// last block to arrive releases the others by its arrival alone.
__device__ __forceinline__ bool grid_barrier(const StepArgs& a, int* abort_flag)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int before = atomicAdd(a.bar, 1u);
        const unsigned int target = (before / gridDim.x + 1u) * gridDim.x;
        if (before + 1u != target) {
            volatile unsigned int* arrived = a.bar;
            unsigned int it = 0;
            while (*arrived < target) {
                if (++it > kBarrierSpins) {
                    atomicOr(a.status, kStatusBarrier);
                    *abort_flag = 1;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *abort_flag == 0;
}

template <bool CUR, int MINB, bool FX>
__global__ void __launch_bounds__(kPushBlock, MINB) k_steps(StepArgs a, int32_t nsteps)
{
    __shared__ int64_t pre[kMaxBuckets + 1];
    __shared__ int pop_cnt[kTracePops];
    __shared__ int abort_flag;
    __shared__ unsigned long long blk_ev;  // without the trace: the block's events, added once at the end
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    int64_t s = *a.step;
    int32_t slot = a.slots[0], hslot = a.slots[1];
    int64_t rbase = a.record ? *a.raster_pos : 0;
    const int64_t rstep0 = *a.raster_step0;
    if (threadIdx.x == 0) {
        abort_flag = 0;
        blk_ev = 0;
    }
    for (int32_t i = 0; i < nsteps; ++i) {
        const int32_t next_h = hslot + 1 == a.H ? 0 : hslot + 1;
        if (lead) {
            a.hist_cnt[next_h] = 0;  // step s+1's slot held step s+1-H; no delivery of step s reads it
            if (a.trace) {
                float* nxt = a.trace + ((s + 1) & (kTraceSteps - 1)) * kTraceCols;
                for (int c = 0; c < kTraceCols; ++c) nxt[c] = 0.f;
            }
        }
        if (threadIdx.x < kTracePops) pop_cnt[threadIdx.x] = 0;
        __syncthreads();
        if (threadIdx.x < 32) deliver_prefix(a, s + 1, s, hslot, pre);
        neuron_groups<2, CUR, FX>(a, s, hslot, acc_buf<FX>(a, a.acc_e, s), acc_buf<FX>(a, a.acc_i, s), warp, nwarps,
                              a.record ? rbase : 0, a.trace ? pop_cnt : nullptr);
        __syncthreads();
        if (a.trace && threadIdx.x < kTracePops && pop_cnt[threadIdx.x])
            atomicAdd(a.trace + (s & (kTraceSteps - 1)) * kTraceCols + threadIdx.x, (float)pop_cnt[threadIdx.x]);
        deliver_tasks<FX>(a, s + 1, s, hslot, pre, warp, nwarps, a.trace ? nullptr : &blk_ev);
        if (!a.trace && i == nsteps - 1) {  // the block's events, before the last barrier
            __syncthreads();
            if (threadIdx.x == 0 && blk_ev) atomicAdd(a.events, blk_ev);
        }
        if (!grid_barrier(a, &abort_flag)) return;
        // step s is complete on every block
        const int32_t nspk = *(volatile int32_t*)(a.hist_cnt + hslot);
        if (lead) {
            if (a.record) {
                const int64_t idx = s - rstep0;
                if (idx < a.raster_steps_cap)
                    a.raster_counts[idx] = nspk;
                else
                    atomicOr(a.status, kStatusRasterSteps);
                if (rbase + nspk > a.raster_ids_cap) atomicOr(a.status, kStatusRasterIds);
            }
            if (a.trace) {
                const unsigned long long ev = *(volatile unsigned long long*)a.events;
                a.trace[(s & (kTraceSteps - 1)) * kTraceCols + kTracePops] = (float)(ev - *a.ev_mark);
                *a.ev_mark = ev;
            }
        }
        if (a.record) rbase += nspk;
        s += 1;
        hslot = next_h;
        slot = slot + 1 == a.M ? 0 : slot + 1;
    }
    if (lead) {
        if (a.record) *a.raster_pos = rbase;
        *a.ev_mark = *(volatile unsigned long long*)a.events;  // every block's events are in
        a.slots[0] = slot;
        a.slots[1] = hslot;
        __threadfence();
        *a.step = s;
    }
}

// ---------------------------------------------------------------------------
// Windowed step group (window W <= minimum delay, W <= 8).  The inputs of
// the W steps of a window arrive from spikes of steps before the window, so
// all of them are delivered before it, and then every neuron advances W
// steps in registers: its state is loaded and stored once per window, its W
// input slots are loaded together, and the blocks meet twice per window (after
// the update, after the next window's deliveries) instead of at every step.
// The arithmetic of each step is that of the single-step update, step by
// step, so the results are the same bits.  Accumulator buffers: step x in
// x & acc_mask (the 8-buffer cycle for W > 4 keeps a window's buffers
// distinct); history: H >= max delay + W, so the slots cleared for the next
// window hold steps no delivery of this window reads.  WMAX (4 or 8) is the
// longest window an instantiation runs: the 4-step one keeps the smaller
// per-task step table of the delivery.  The group starts and ends in the
// state of the single-step kernels (arrivals of its first step delivered,
// nothing later).  Waits are bounded (kStatusBarrier).
// ---------------------------------------------------------------------------
constexpr int kMaxWindow = 8;
constexpr int kWinLoad = 4;  // input slots a lane holds at once

// Neurons [first group, ...) advanced through the window's wl steps.  One
// group of four neurons per lane per pass: its state is loaded once, its
// input slots four steps at a time, the steps run in registers, the state is
// stored once, and the pass's spikes of all its steps are compacted into the
// steps' history slots together at the end.  The lane at position p of a
// pass takes group (p + upd_rot) mod groups (the host's rotation puts the
// POISSON groups on lanes without an extra pass).
template <bool CUR, bool FX, int WMAX, bool PULL>
__device__ __forceinline__ void neuron_window(const StepArgs& a, int64_t w0, int wl, int32_t hs0, int64_t warp,
                                              int64_t nwarps)
{
    const int lane = threadIdx.x & 31;
    const int64_t ngroups = a.ns >> 2;
    for (int64_t gb = warp * 32; gb < ngroups; gb += nwarps * 32) {
        const bool have = gb + lane < ngroups;
        int64_t g = gb + lane + (PULL ? 0 : a.upd_rot);  // the bitmaps' words follow the positions
        if (g >= ngroups) g -= ngroups;
        char4 t4 = make_char4(0, 0, 0, 0);
        float4 v4 = make_float4(0.f, 0.f, 0.f, 0.f), ce4 = v4, ci4 = v4;
        int4 r4 = make_int4(0, 0, 0, 0);
        if (have) {
            t4 = __ldg(reinterpret_cast<const char4*>(a.type) + g);
            v4 = reinterpret_cast<float4*>(a.V)[g];
            r4 = reinterpret_cast<int4*>(a.refrac)[g];
            if (CUR) {
                ce4 = reinterpret_cast<float4*>(a.Iexc)[g];
                ci4 = reinterpret_cast<float4*>(a.Iinh)[g];
            }
        }
        const int32_t i0 = (int32_t)(g << 2);
        const bool pois = t4.x == kPOISSON || t4.y == kPOISSON || t4.z == kPOISSON || t4.w == kPOISSON;
        const bool lifb4 = t4.x == kLIFB && t4.y == kLIFB && t4.z == kLIFB && t4.w == kLIFB;
        // four POISSON neurons ignore their input and keep their state (V holds
        // the probability): no input slot is cleared, no state stored
        const bool pois4 = t4.x == kPOISSON && t4.y == kPOISSON && t4.z == kPOISSON && t4.w == kPOISSON;
        unsigned fms = 0;  // the pass's spikes: bits 4j..4j+3 for step w0 + j
        // the window's steps four at a time: their input slots loaded at once
        // (one copy of the update in the code; the loop forms keep the
        // 3-blocks-per-SM instantiations within their 80 registers)
#pragma unroll 1
        for (int h = 0; h < (WMAX > kWinLoad ? wl : WMAX); h += kWinLoad) {
            if (h >= wl) break;
            In4<FX> e4[kWinLoad], i4[kWinLoad];
#pragma unroll
            for (int k = 0; k < kWinLoad; ++k) {
                e4[k].zero();
                i4[k].zero();
                if (have && !pois4 && h + k < wl) {
                    e4[k].load(acc_buf<FX, WMAX - 1>(a, a.acc_e, w0 + h + k), g);
                    i4[k].load(acc_buf<FX, WMAX - 1>(a, a.acc_i, w0 + h + k), g);
                }
            }
#pragma unroll
            for (int k = 0; k < kWinLoad; ++k) {
                if (h + k >= wl) break;
                const int64_t s = w0 + h + k;
                unsigned fm = 0;
                if (have) {
                    const float4 e = e4[k].get(a), ii = i4[k].get(a);
                    if (lifb4) {
                        fm |= lifb_step(a, v4.x, r4.x, e.x, ii.x) ? 1u : 0u;
                        fm |= lifb_step(a, v4.y, r4.y, e.y, ii.y) ? 2u : 0u;
                        fm |= lifb_step(a, v4.z, r4.z, e.z, ii.z) ? 4u : 0u;
                        fm |= lifb_step(a, v4.w, r4.w, e.w, ii.w) ? 8u : 0u;
                        // (fire counts and last spikes of every group: after the pass)
                    } else {
                        float u[4] = {0.f, 0.f, 0.f, 0.f};
                        if (pois) poisson_uniform4(a.seed, (int64_t)i0 + a.id_offset, s, u);
                        fm |= update_one<false>(a, t4.x, i0 + 0, s, v4.x, r4.x, e.x, ii.x, ce4.x, ci4.x, u[0]) ? 1u : 0u;
                        fm |= update_one<false>(a, t4.y, i0 + 1, s, v4.y, r4.y, e.y, ii.y, ce4.y, ci4.y, u[1]) ? 2u : 0u;
                        fm |= update_one<false>(a, t4.z, i0 + 2, s, v4.z, r4.z, e.z, ii.z, ce4.z, ci4.z, u[2]) ? 4u : 0u;
                        fm |= update_one<false>(a, t4.w, i0 + 3, s, v4.w, r4.w, e.w, ii.w, ce4.w, ci4.w, u[3]) ? 8u : 0u;
                    }
                    // the step's input was used: its slot is cleared for step s + acc_mask + 1
                    if (!pois4) {
                        In4<FX>::clear(acc_buf<FX, WMAX - 1>(a, a.acc_e, s), g);
                        In4<FX>::clear(acc_buf<FX, WMAX - 1>(a, a.acc_i, s), g);
                    }
                }
                if (PULL) {  // the step's spikes as a bitmap (pull steps read it)
                    int32_t hb = hs0 + h + k;
                    if (hb >= a.H) hb -= a.H;
                    unsigned wv = fm << (4 * (lane & 7));
                    wv |= __shfl_xor_sync(0xffffffffu, wv, 1);
                    wv |= __shfl_xor_sync(0xffffffffu, wv, 2);
                    wv |= __shfl_xor_sync(0xffffffffu, wv, 4);
                    if ((lane & 7) == 0 && gb < ngroups)
                        a.hist_bits[(size_t)hb * (size_t)a.bits_words + (gb >> 3) + (lane >> 3)] = wv;
                }
                fms |= fm << (4 * (h + k));
            }
        }
        // the pass's spikes into their steps' history slots, in neuron order
        // within the warp: one scan for all steps (a warp's count of a step is
        // at most 128, so four steps share a word, a byte each), the steps'
        // positions reserved by lanes 0..wl-1 at once
        if (__any_sync(0xffffffffu, fms != 0)) {
            uint32_t ca = 0, cb = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                ca |= (uint32_t)__popc((fms >> (4 * j)) & 15u) << (8 * j);
                cb |= (uint32_t)__popc((fms >> (4 * j + 16)) & 15u) << (8 * j);
            }
            uint32_t ia = ca, ib = cb;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t va = __shfl_up_sync(0xffffffffu, ia, o), vb = __shfl_up_sync(0xffffffffu, ib, o);
                if (lane >= o) {
                    ia += va;
                    ib += vb;
                }
            }
            const uint32_t ta = __shfl_sync(0xffffffffu, ia, 31), tb = __shfl_sync(0xffffffffu, ib, 31);
            ia -= ca;  // exclusive
            ib -= cb;
            int32_t base = 0;
            if (lane < wl) {
                const int32_t tot = (int32_t)(((lane < 4 ? ta : tb) >> (8 * (lane & 3))) & 255u);
                if (tot) {
                    int32_t hs = hs0 + lane;
                    if (hs >= a.H) hs -= a.H;
                    base = atomicAdd(a.hist_cnt + hs, tot);
                }
            }
            for (int j = 0; j < wl; ++j) {
                const int32_t bj = __shfl_sync(0xffffffffu, base, j);
                const unsigned f = (fms >> (4 * j)) & 15u;
                if (!f) continue;
                int32_t pos = bj + (int32_t)(((j < 4 ? ia : ib) >> (8 * (j & 3))) & 255u);
                int32_t hs = hs0 + j;
                if (hs >= a.H) hs -= a.H;
                int32_t* ids = a.hist_ids + (size_t)hs * (size_t)a.n_src;
                for (int q = 0; q < 4; ++q)
                    if (f & (1u << q)) {
                        if (!MGC_OK_INDEX(pos < a.n_src)) break;
                        ids[pos++] = a.src_base + i0 + q;
                    }
            }
            // each neuron's spikes of the pass: its count added once, its last step stored once
            for (int q = 0; q < 4; ++q) {
                const unsigned fq = fms & (0x11111111u << q);
                if (fq) {
                    atomicAdd(a.fire_cnt + i0 + q, __popc(fq));
                    a.last_fired[i0 + q] = (int32_t)(w0 + ((31 - __clz(fq)) >> 2));
                }
            }
        }
        if (have && !pois4) {
            reinterpret_cast<float4*>(a.V)[g] = v4;
            reinterpret_cast<int4*>(a.refrac)[g] = r4;
            if (CUR) {
                reinterpret_cast<float4*>(a.Iexc)[g] = ce4;
                reinterpret_cast<float4*>(a.Iinh)[g] = ci4;
            }
        }
    }
}

// The arrivals of steps [sa0, sa0 + n) (n <= WMAX), from spikes of steps
// before sa0: the prefixes of the n steps by the first n warps, then every
// warp through the n steps' tasks without a barrier between them.  s, hslot:
// a step and its history slot, for the slot arithmetic.
constexpr int kPullUnroll = 8;  // incoming entries a lane loads at once in a pull step

// fp32 addition with the rounding and subnormal flushing of red.add.f32
__device__ __forceinline__ float fadd_ftz(float x, float y)
{
    float r;
    asm("add.rn.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(x), "f"(y));
    return r;
}

// Pull delivery of the arrivals of the steps in `mask` (bit k: step sa0 + k):
// one warp per (step x, target t) walks t's incoming row and adds the
// weights of the synapses whose source spiked at step x - delay (the history
// slots' bitmaps), then stores the sums into the accumulators of step x,
// which nothing else writes for a pulled step.  No atomics, and the sum is
// the one the push computes: with fixed-point accumulation the exact integer
// sum; with fp32 sums every neuron receives one weight per sign (the handle
// refuses pull steps otherwise), and k additions of one weight give the same
// bits in any order, here a chain of k additions from zero with red.add's
// rounding (lane 0 the exc sum, lane 1 the inh).  Work starts at the first
// warp (push tasks start at the last).
template <bool FX, int MASK>
__device__ __forceinline__ void pull_steps(const StepArgs& a, int64_t sa0, unsigned mask, int64_t s, int32_t hslot,
                                           int64_t warp, int64_t nwarps, unsigned long long* blk_ev)
{
    const int lane = threadIdx.x & 31;
    const int64_t n = a.n;
    const int64_t total = (int64_t)__popc(mask) * n;
    unsigned long long ev = 0;
    for (int64_t it = warp; it < total; it += nwarps) {
        const int j = (int)(it / n);  // the j-th pulled step
        const int32_t t = (int32_t)(it - (int64_t)j * n);
        unsigned m = mask;
        for (int q = 0; q < j; ++q) m &= m - 1;
        const int64_t x = sa0 + (__ffs(m) - 1);
        const int32_t hx = hist_slot(a, x, s, hslot);
        const int64_t rb = a.in_ptr[t], re = a.in_ptr[t + 1];
        int ce = 0, ci = 0;
        long long fe = 0, fi = 0;
        float we = 0.f, wi = 0.f;
        for (int64_t q0 = rb; q0 < re; q0 += 32 * kPullUnroll) {
            uint2 e[kPullUnroll];
#pragma unroll
            for (int u = 0; u < kPullUnroll; ++u) {
                const int64_t q = q0 + u * 32 + lane;
                // (cached normally: the rows stay in L2 for the next pulled
                // step while the push's synapse words stream past evict-first)
                e[u] = q < re ? __ldcg(a.in_ent + q) : make_uint2(0u, 0u);
            }
#pragma unroll
            for (int u = 0; u < kPullUnroll; ++u) {
                if (q0 + u * 32 + lane >= re) continue;
                const int32_t src = (int32_t)(e[u].x & a.tmask);
                const int32_t d = (int32_t)(e[u].x >> a.tbits);
                if (!MGC_OK_INDEX(src < a.n && d >= a.dmin && d < a.dmin + a.D)) continue;
                int32_t h = hx - d;
                if (h < 0) h += a.H;
                if (!((a.hist_bits[(size_t)h * (size_t)a.bits_words + (src >> 5)] >> (src & 31)) & 1u)) continue;
                const float w = as_f(e[u].y);
                if (w > 0.0f) {
                    ++ce;
                    we = w;
                    if (FX) fe += to_fx(w, a.fx_scale);
                } else {
                    ++ci;
                    wi = w;
                    if (FX) fi += to_fx(w, a.fx_scale);
                }
            }
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            ce += __shfl_xor_sync(0xffffffffu, ce, o);
            ci += __shfl_xor_sync(0xffffffffu, ci, o);
            if (FX) {
                fe += __shfl_xor_sync(0xffffffffu, fe, o);
                fi += __shfl_xor_sync(0xffffffffu, fi, o);
            }
        }
        if (!FX) {  // the weight of each sign (the same on every lane that saw one)
            const unsigned he = __ballot_sync(0xffffffffu, we != 0.0f), hi = __ballot_sync(0xffffffffu, wi != 0.0f);
            we = he ? __shfl_sync(0xffffffffu, we, __ffs(he) - 1) : 0.0f;
            wi = hi ? __shfl_sync(0xffffffffu, wi, __ffs(hi) - 1) : 0.0f;
        }
        if (lane == 0) ev += (unsigned long long)(ce + ci);
        if (lane < 2 && (lane == 0 ? ce : ci)) {
            float* base = lane == 0 ? a.acc_e : a.acc_i;
            if (FX) {
                acc_buf<true, MASK>(a, base, x)[t] = (unsigned long long)(lane == 0 ? fe : fi);
            } else {
                const float w = lane == 0 ? we : wi;
                const int c = lane == 0 ? ce : ci;
                float v = 0.0f;
                for (int r = 0; r < c; ++r) v = fadd_ftz(v, w);
                acc_buf<false, MASK>(a, base, x)[t] = v;
            }
        }
    }
    if (lane == 0 && ev) atomicAdd(blk_ev ? blk_ev : a.events, ev);
}

template <bool FX, int WMAX, bool PULL>
__device__ __forceinline__ void deliver_window(const StepArgs& a, int64_t sa0, int n, int64_t s, int32_t hslot,
                                               int64_t* pre, int64_t warp, int64_t nwarps, unsigned long long* blk_ev,
                                               int64_t bits_from)
{
    const int wib = threadIdx.x >> 5;
    for (int k = wib; k < n; k += blockDim.x >> 5) deliver_prefix(a, sa0 + k, s, hslot, pre + (size_t)k * (a.D + 1));
    __syncthreads();
    unsigned pull = 0;
    if (PULL && a.pull_min > 0) {
        // the steps delivered by pull: many arriving (spike, delay) pairs, and
        // every step they come from has its bitmap (every block takes the
        // same decision from the same counts)
        const int64_t dmax = (int64_t)a.dmin + a.D - 1;
        for (int k = 0; k < n; ++k)
            if (pre[(size_t)k * (a.D + 1) + a.D] >= a.pull_min && sa0 + k - dmax >= bits_from) pull |= 1u << k;
        if (pull) {  // their push tasks emptied
            __syncthreads();
            for (int k = 0; k < n; ++k)
                if ((pull >> k) & 1u)
                    for (int j = threadIdx.x; j <= a.D; j += blockDim.x) pre[(size_t)k * (a.D + 1) + j] = 0;
            __syncthreads();
        }
    }
    deliver_tasks<FX, WMAX, WMAX - 1>(a, sa0, s, hslot, pre, warp, nwarps, blk_ev, n);
    if (PULL && pull) pull_steps<FX, WMAX - 1>(a, sa0, pull, s, hslot, warp, nwarps, blk_ev);
}

__device__ __forceinline__ void raster_copy(const StepArgs& a, int64_t sc, int32_t hs, int64_t rstep0,
                                            int64_t& rbase);

template <bool CUR, int MINB, bool FX, int WMAX, bool PULL>
__global__ void __launch_bounds__(kPushBlock, MINB) k_window(StepArgs a, int32_t nsteps, int32_t W)
{
    extern __shared__ int64_t wpre[];   // [WMAX][D + 1]
    __shared__ int abort_flag;
    __shared__ unsigned long long blk_ev;  // the block's delivered events, added once at the end
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    const int64_t s0 = *a.step;
    const int32_t slot0 = a.slots[0], h0 = a.slots[1];
    const bool rec = a.record != 0;
    int64_t rbase = rec ? *a.raster_pos : 0;
    const int64_t rstep0 = *a.raster_step0;
    const int64_t s_end = s0 + nsteps;
    auto hs_of = [&](int64_t x) { return (int32_t)((h0 + (x - s0)) % a.H); };
    // pull steps: the bitmaps written since `bits_from`, if the previous
    // steps were this group's too, else from s0 on
    int64_t bits_from = s0;
    if (PULL && *(volatile int64_t*)(a.bits_span + 1) == s0) bits_from = *(volatile int64_t*)a.bits_span;
    if (threadIdx.x == 0) {
        abort_flag = 0;
        blk_ev = 0;
    }
    // prologue: the arrivals of the first window's later steps (its first
    // step's are delivered), their history slots cleared
    {
        const int n = (int)(nsteps < W ? nsteps - 1 : W - 1);
        if (lead)
            for (int k = 1; k <= n; ++k) a.hist_cnt[hs_of(s0 + k)] = 0;
        __syncthreads();
        if (n > 0) deliver_window<FX, WMAX, PULL>(a, s0 + 1, n, s0, h0, wpre, warp, nwarps, &blk_ev, bits_from);
        if (!grid_barrier(a, &abort_flag)) return;
    }
    for (int64_t w0 = s0; w0 < s_end;) {
        const int wl = (int)(s_end - w0 < W ? s_end - w0 : W);
        neuron_window<CUR, FX, WMAX, PULL>(a, w0, wl, hs_of(w0), warp, nwarps);
        if (!grid_barrier(a, &abort_flag)) return;
        // the window's spikes are complete: its raster, then the next
        // window's arrivals (only those of s_end after the last window)
        if (rec && blockIdx.x == 0)
            for (int k = 0; k < wl; ++k) raster_copy(a, w0 + k, hs_of(w0 + k), rstep0, rbase);
        const int64_t next = w0 + wl;
        const int nn = (int)(next < s_end ? (s_end - next < W ? s_end - next : W) : 1);
        if (lead)
            for (int k = 0; k < nn; ++k) a.hist_cnt[hs_of(next + k)] = 0;
        deliver_window<FX, WMAX, PULL>(a, next, nn, w0, hs_of(w0), wpre, warp, nwarps, &blk_ev, bits_from);
        if (next >= s_end) {  // the block's events, before the last barrier
            __syncthreads();
            if (threadIdx.x == 0 && blk_ev) atomicAdd(a.events, blk_ev);
        }
        if (!grid_barrier(a, &abort_flag)) return;
        w0 = next;
    }
    if (lead) {
        if (rec) *a.raster_pos = rbase;
        *a.ev_mark = *(volatile unsigned long long*)a.events;
        a.slots[0] = (int32_t)((slot0 + nsteps) % a.M);
        a.slots[1] = hs_of(s_end);
        if (PULL) {
            a.bits_span[0] = bits_from;
            a.bits_span[1] = s_end;
        }
        __threadfence();
        *a.step = s_end;
    }
}

// ---------------------------------------------------------------------------
// Step group for a minimum delay of one step, where the arrivals of step s
// include the spikes of step s-1: per step the delivery of its arrivals, a
// grid barrier, the neuron update, a grid barrier.  The group starts and
// ends in the state the single-step kernels (k_deliver, then k_neuron)
// start from, so the two forms mix.  Its grid is sized to the neurons, so a
// small network takes few blocks and cheap barriers.  Waits are bounded
// (kStatusBarrier).
// ---------------------------------------------------------------------------
template <bool CUR, bool FX>
__global__ void __launch_bounds__(kPushBlock, 2) k_steps1(StepArgs a, int32_t nsteps)
{
    __shared__ int64_t pre[kMaxBuckets + 1];
    __shared__ int abort_flag;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    int64_t s = *a.step;
    int32_t slot = a.slots[0], hslot = a.slots[1];
    int64_t rbase = a.record ? *a.raster_pos : 0;
    const int64_t rstep0 = *a.raster_step0;
    if (threadIdx.x == 0) abort_flag = 0;
    for (int32_t i = 0; i < nsteps; ++i) {
        const int32_t next_h = hslot + 1 == a.H ? 0 : hslot + 1;
        // the arrivals of step s: spikes of steps <= s-1, complete at the last barrier
        if (threadIdx.x < 32) deliver_prefix(a, s, s, hslot, pre);
        __syncthreads();
        deliver_tasks<FX>(a, s, s, hslot, pre, warp, nwarps);
        if (!grid_barrier(a, &abort_flag)) return;
        // step s+1's slot held step s+1-H, which no delivery reads any more
        if (lead) a.hist_cnt[next_h] = 0;
        neuron_groups<2, CUR, FX>(a, s, hslot, acc_buf<FX>(a, a.acc_e, s), acc_buf<FX>(a, a.acc_i, s), warp, nwarps,
                              a.record ? rbase : 0);
        if (!grid_barrier(a, &abort_flag)) return;
        // step s is complete on every block
        const int32_t nspk = *(volatile int32_t*)(a.hist_cnt + hslot);
        if (lead && a.record) {
            const int64_t idx = s - rstep0;
            if (idx < a.raster_steps_cap)
                a.raster_counts[idx] = nspk;
            else
                atomicOr(a.status, kStatusRasterSteps);
            if (rbase + nspk > a.raster_ids_cap) atomicOr(a.status, kStatusRasterIds);
        }
        if (a.record) rbase += nspk;
        s += 1;
        hslot = next_h;
        slot = slot + 1 == a.M ? 0 : slot + 1;
    }
    if (lead) {
        if (a.record) *a.raster_pos = rbase;
        a.slots[0] = slot;
        a.slots[1] = hslot;
        __threadfence();
        *a.step = s;
    }
}

// ---------------------------------------------------------------------------
// Pipelined step group (minimum delay >= 4): during step s every block
// updates its neurons of step s and delivers the arrivals of step s+2 (they
// depend only on spikes of steps <= s-2), so a block waits only until every
// block has finished step s-2 — an arrive/wait barrier split across two
// steps instead of a full barrier per step.  The accumulators rotate over
// four buffers: step s+2's is the one step s-2 read and cleared.  The
// history holds H >= max delay + 3 steps so the slot cleared for step s+2
// is read by no delivery still running.  Block 0 copies finished steps'
// spike ids from the history into the raster two steps behind.  The
// prologue delivers the arrivals of step s0+1; the last deliveries are those
// of the group's last step + 1 - 1, so the group ends in the state the
// single-step kernels start from.  Waits are bounded (kStatusBarrier).
//
// Phases: 0 is the prologue, k >= 1 is iteration k-1.  Blocks are never
// more than two phases apart (a block in iteration i waited for phase i-1),
// so four arrival counters used round-robin keep phases apart: counter
// p % 4 has counted nb per earlier use when phase p completes, and the next
// phase that uses it (p + 4) starts only after phase p + 2 completed.
// ---------------------------------------------------------------------------
constexpr int kPhaseCounters = 4;

__device__ __forceinline__ bool wait_phase(const StepArgs& a, int32_t phase, int* abort_flag)
{
    if (threadIdx.x == 0) {
        volatile unsigned int* arrived = a.bar + (phase % kPhaseCounters);
        const unsigned int target = gridDim.x * (unsigned int)(phase / kPhaseCounters + 1);
        unsigned int it = 0;
        while (*arrived < target) {
            if (++it > kBarrierSpins) {
                atomicOr(a.status, kStatusBarrier);
                *abort_flag = 1;
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
    }
    __syncthreads();
    return *abort_flag == 0;
}

// The block's step is done, then it arrives on the phase counter.  With the
// schedule trace on, its spike counts per trace population and its delivered
// events go into step s's trace row and the events counter every step (and
// the block counters are cleared for reuse); without it the block's events
// accumulate in `ev` and go out once, with the group's last step (flush), so
// that the blocks do not queue on one counter every step.
__device__ __forceinline__ void arrive(const StepArgs& a, int32_t phase, int64_t s, int* pop, unsigned long long* ev,
                                       bool flush)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        if (pop) {
            if (a.trace) {
                float* row = a.trace + (s & (kTraceSteps - 1)) * kTraceCols;
                for (int c = 0; c < kTracePops; ++c) {
                    if (pop[c]) atomicAdd(row + c, (float)pop[c]);
                    pop[c] = 0;
                }
                if (*ev) {
                    atomicAdd(a.events, *ev);
                    atomicAdd(row + kTracePops, (float)*ev);
                }
                *ev = 0;
            } else if (flush) {
                if (*ev) atomicAdd(a.events, *ev);
                *ev = 0;
            }
        }
        __threadfence();
        atomicAdd(a.bar + (phase % kPhaseCounters), 1u);
    }
}

// Block 0 copies the spike ids of finished step sc into the raster.
__device__ __forceinline__ void raster_copy(const StepArgs& a, int64_t sc, int32_t hs, int64_t rstep0, int64_t& rbase)
{
    const int32_t cnt = *(volatile int32_t*)(a.hist_cnt + hs);
    const int32_t* ids = a.hist_ids + (size_t)hs * (size_t)a.n_src;
    for (int32_t j = threadIdx.x; j < cnt; j += blockDim.x)
        if (rbase + j < a.raster_ids_cap) a.raster_ids[rbase + j] = ids[j];
    if (threadIdx.x == 0) {
        const int64_t idx = sc - rstep0;
        if (idx < a.raster_steps_cap)
            a.raster_counts[idx] = cnt;
        else
            atomicOr(a.status, kStatusRasterSteps);
        if (rbase + cnt > a.raster_ids_cap) atomicOr(a.status, kStatusRasterIds);
    }
    rbase += cnt;
}

template <bool CUR, int MINB, bool FX>
__global__ void __launch_bounds__(kPushBlock, MINB) k_pipe(StepArgs a, int32_t nsteps)
{
    __shared__ int64_t pre[kMaxBuckets + 1];
    __shared__ int abort_flag;
    __shared__ int pop_cnt[2][kTracePops];        // by step parity
    __shared__ unsigned long long blk_ev[2];
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    const int64_t s0 = *a.step;
    const int32_t slot0 = a.slots[0], h0 = a.slots[1];
    const bool rec = a.record != 0;
    int64_t rbase = rec ? *a.raster_pos : 0;
    const int64_t rstep0 = *a.raster_step0;
    const int64_t s_end = s0 + nsteps;
    auto hs_of = [&](int64_t x) { return (int32_t)((h0 + (x - s0)) % a.H); };
    if (threadIdx.x == 0) abort_flag = 0;
    if (threadIdx.x < 2 * kTracePops) pop_cnt[threadIdx.x / kTracePops][threadIdx.x % kTracePops] = 0;
    if (threadIdx.x < 2) blk_ev[threadIdx.x] = 0;
    // prologue: arrivals of step s0+1; the slot of step s0+1 cleared, and the
    // trace rows of steps s0+1, s0+2 (row s0 was cleared by the step before)
    if (lead) {
        a.hist_cnt[hs_of(s0 + 1)] = 0;
        if (a.trace)
            for (int64_t x = s0 + 1; x <= s0 + 2; ++x)
                for (int c = 0; c < kTraceCols; ++c) a.trace[(x & (kTraceSteps - 1)) * kTraceCols + c] = 0.f;
    }
    __syncthreads();
    if (nsteps > 0) {
        if (threadIdx.x < 32) deliver_prefix(a, s0 + 1, s0, h0, pre);
        __syncthreads();
        deliver_tasks<FX>(a, s0 + 1, s0, h0, pre, warp, nwarps);
    }
    arrive(a, 0, 0, nullptr, nullptr, false);
    for (int32_t i = 0; i < nsteps; ++i) {
        const int64_t s = s0 + i;
        const int32_t hs = hs_of(s);
        const bool deliver = s + 2 <= s_end;
        // every block has finished step s-2 (phase i-1; for i = 1 the prologue)
        if (i >= 1 && !wait_phase(a, i - 1, &abort_flag)) return;
        if (lead && s + 2 <= s_end) a.hist_cnt[hs_of(s + 2)] = 0;
        if (lead && a.trace) {  // no block writes step s+3's row before lead finishes step s+1
            float* row = a.trace + ((s + 3) & (kTraceSteps - 1)) * kTraceCols;
            for (int c = 0; c < kTraceCols; ++c) row[c] = 0.f;
        }
        if (rec && blockIdx.x == 0 && i >= 2) raster_copy(a, s - 2, hs_of(s - 2), rstep0, rbase);
        const int b = i & 1;
        unsigned long long* evb = a.trace ? &blk_ev[b] : &blk_ev[0];  // per step, or for the group
        if (deliver && threadIdx.x < 32) deliver_prefix(a, s + 2, s, hs, pre);
        neuron_groups<2, CUR, FX>(a, s, hs, acc_buf<FX>(a, a.acc_e, s), acc_buf<FX>(a, a.acc_i, s), warp, nwarps, 0,
                              a.trace ? pop_cnt[b] : nullptr, false);
        __syncthreads();
        if (deliver) deliver_tasks<FX>(a, s + 2, s, hs, pre, warp, nwarps, evb);
        arrive(a, i + 1, s, pop_cnt[b], evb, i == nsteps - 1);
    }
    // the group's last steps: all blocks done (phases n-1 and n), remaining raster, the clock
    if (nsteps >= 1 && !wait_phase(a, nsteps - 1, &abort_flag)) return;
    if (!wait_phase(a, nsteps, &abort_flag)) return;
    if (rec && blockIdx.x == 0)
        for (int64_t x = (nsteps >= 2 ? s_end - 2 : s0); x < s_end; ++x) raster_copy(a, x, hs_of(x), rstep0, rbase);
    if (lead) {
        if (rec) *a.raster_pos = rbase;
        *a.ev_mark = *(volatile unsigned long long*)a.events;  // every block's events are in
        a.slots[0] = (int32_t)((slot0 + nsteps) % a.M);
        a.slots[1] = hs_of(s_end);
        __threadfence();
        *a.step = s_end;
    }
}

// ---------------------------------------------------------------------------
// Event push, mgsim_syn_fast_core + pushInnerSpike (mgcore.cu:271-305,
// :112-115): every synapse of a spiking neuron adds its weight to
// ring[(s + delay) % M][target], the exc ring when weight > 0, else inh.
// Work unit: one warp per (spike, 128-synapse chunk of its row).
// ---------------------------------------------------------------------------
template <bool FX>
__global__ void __launch_bounds__(kPushBlock) k_push(StepArgs a)
{
    const int32_t cnt = *(volatile int32_t*)a.spk_count;
    const int32_t slot0 = a.slots[0];
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
        if (!MGC_OK_INDEX(nid >= 0 && nid < a.n)) continue;
        if (c == 0 && lane == 0 && a.record && rpos + j < a.raster_ids_cap) a.raster_ids[rpos + j] = nid;
        const int64_t rb = a.row_ptr[nid], re = a.row_ptr[nid + 1];
        if (!MGC_OK_INDEX(rb >= 0 && rb <= re && re <= a.n_syn)) continue;
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
            if (!MGC_OK_INDEX(tgt < (uint32_t)a.ns && slot >= 0 && slot < a.M)) continue;
            const float wt = as_f(w[u].y);
            float* ring = wt > 0.0f ? a.ring_e : a.ring_i;
            const size_t at = (size_t)slot * (size_t)a.ns + tgt;
            if (FX)
                red_add_fx(reinterpret_cast<unsigned long long*>(ring) + at, to_fx(wt, a.fx_scale));
            else
                red_add(ring + at, wt);
        }
    }
    if (lane == 0 && ev) atomicAdd(a.events, ev);
    if (last_block(a.done)) step_epilogue(a);
}


}  // namespace mgc
