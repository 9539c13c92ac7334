// Network construction on the device: neuron arrays and constants, the
// delivery method, the CSR (stable radix sort of an explicit synapse list,
// or the fixed in-degree generator), the method's buffers and launch shapes.
// Replaces build_multinet / copy_subnet_gpu / init_state / copy_consts_gpu
// (src/simulator/mgsim/adj/mgsim.cpp:8-144, mgnet.cpp:92-146,
// mgcore.cu:665-669, 685-748).
#include <cub/cub.cuh>

#include <cmath>
#include <memory>

#include "sim.h"

using namespace mgc;

namespace {

__global__ void k_count_rows(const uint32_t* key, int64_t S, int kshift, int64_t* deg)
{
    GRID_STRIDE(k, S) atomicAdd(reinterpret_cast<unsigned long long*>(deg + (key[k] >> kshift)), 1ull);
}

// Synapse count of every (source, delay bucket) from the sorted keys.
__global__ void k_count_buckets(const uint32_t* key, int64_t S, int dbits, int D, int64_t* cnt)
{
    GRID_STRIDE(k, S)
    {
        const uint32_t src = key[k] >> dbits, b = key[k] & ((1u << dbits) - 1u);
        atomicAdd(reinterpret_cast<unsigned long long*>(cnt + (size_t)src * D + b), 1ull);
    }
}


__global__ void k_max_gap(const int64_t* off, int64_t count, unsigned long long* out)
{
    GRID_STRIDE(i, count) atomicMax(out, (unsigned long long)(off[i + 1] - off[i]));
}

__global__ void k_validate(const int32_t* src, const int32_t* tar, const int32_t* delay, int64_t S, int32_t n_src,
                           int32_t n, int32_t dlim, int32_t* bad)
{
    GRID_STRIDE(k, S)
    {
        if (src[k] < 0 || src[k] >= n_src || tar[k] < 0 || tar[k] >= n || delay[k] < 1 || delay[k] >= dlim)
            atomicOr(bad, 1);
    }
}

// Sort key of a synapse: source, then (deferred) delay bucket.
__global__ void k_explicit_keys(const int32_t* src, const int32_t* delay, int64_t S, int dbits, int dmin,
                                uint32_t* keys, uint32_t* vals)
{
    GRID_STRIDE(k, S)
    {
        keys[k] = ((uint32_t)src[k] << dbits) | (uint32_t)(dbits ? delay[k] - dmin : 0);
        vals[k] = (uint32_t)k;
    }
}

// CSR words from an explicit synapse list gathered in sorted order.
__global__ void k_gather_explicit(const uint32_t* order, const uint32_t* keys, int kshift, const int32_t* tar,
                                  const float* w, const int32_t* delay, const uint8_t* plastic_in, int64_t S,
                                  int tbits, uint2* syn, int64_t* csr_syn, int32_t* csr_src, uint8_t* plastic_out)
{
    GRID_STRIDE(p, S)
    {
        const uint32_t k = order[p];
        syn[p] = make_uint2((uint32_t)tar[k] | ((uint32_t)delay[k] << tbits), __float_as_uint(w[k]));
        csr_syn[p] = k;
        if (csr_src) csr_src[p] = (int32_t)(keys[p] >> kshift);
        if (plastic_out) plastic_out[p] = plastic_in ? (plastic_in[k] != 0) : 1;
    }
}

__global__ void k_inverse(const int64_t* csr_syn, int64_t S, uint32_t* pos_of)
{
    GRID_STRIDE(p, S) pos_of[csr_syn[p]] = (uint32_t)p;
}

__global__ void k_widen(const uint32_t* in, int64_t S, int64_t* out)
{
    GRID_STRIDE(p, S) out[p] = in[p];
}

__global__ void k_cast_keys(const int32_t* in, int64_t S, uint32_t* out)
{
    GRID_STRIDE(p, S) out[p] = (uint32_t)in[p];
}

// Incoming rows for the pull method: target, then delay, then source, then
// synapse-list order (the sort is stable).
__global__ void k_pull_keys(const int32_t* src, const int32_t* tar, const int32_t* delay, int64_t S, int tb, int db,
                            int dmin, uint64_t* keys, uint32_t* vals)
{
    GRID_STRIDE(k, S)
    {
        keys[k] = ((uint64_t)tar[k] << (db + tb)) | ((uint64_t)(delay[k] - dmin) << tb) | (uint64_t)src[k];
        vals[k] = (uint32_t)k;
    }
}

// Pull steps of the deferred method: for every CSR position its target (the
// sort key) and its source (one warp per source row of the bucketed CSR).
__global__ void k_row_sources(const int64_t* bucket, int32_t n_src, int D, const uint2* syn, uint32_t tmask,
                              uint32_t* tkey, uint32_t* pos, int32_t* src_of)
{
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n_src; r += nw) {
        const int64_t b = bucket[(size_t)r * D], e = bucket[(size_t)r * D + D];
        for (int64_t p = b + lane; p < e; p += 32) {
            tkey[p] = syn[p].x & tmask;
            pos[p] = (uint32_t)p;
            src_of[p] = (int32_t)r;
        }
    }
}

// Incoming entries {source | delay << tbits, weight} in target order.
__global__ void k_gather_in(const uint32_t* order, const uint2* syn, const int32_t* src_of, int64_t S, uint32_t tmask,
                            uint2* in_ent)
{
    GRID_STRIDE(i, S)
    {
        const uint32_t p = order[i];
        const uint2 w = syn[p];
        in_ent[i] = make_uint2((w.x & ~tmask) | (uint32_t)src_of[p], w.y);
    }
}

__global__ void k_gather_pull(const uint32_t* order, const int32_t* src, const float* w, const int32_t* delay,
                              const uint8_t* plastic_in, int64_t S, int tbits, uint2* ent, int64_t* ent_syn,
                              uint8_t* plastic_out)
{
    GRID_STRIDE(p, S)
    {
        const uint32_t k = order[p];
        ent[p] = make_uint2((uint32_t)src[k] | ((uint32_t)delay[k] << tbits), __float_as_uint(w[k]));
        ent_syn[p] = k;
        if (plastic_out) plastic_out[p] = plastic_in ? (plastic_in[k] != 0) : 1;
    }
}

// Fixed in-degree generator (see mgc_fixed_indegree_desc): synapse index
// i -> projection r (binary search over the block's table), target t, draw k.
struct ProjEntry {
    int64_t base;  // first synapse index of the projection
    uint64_t seed; // conn_seed of its block
    int32_t src_start, src_num, tar_start, k, dmin, dspan;
    float w;
    int32_t rid;     // projection index in the draws
    int32_t id_off;  // added to target ids in the draws
    int32_t tar_sub; // subtracted from target ids in the CSR words (a partition's first neuron)
};

__device__ __forceinline__ void fid_decode(const ProjEntry* pt, int32_t npr, int64_t i, int32_t& src, int32_t& tar,
                                           int32_t& delay, float& w)
{
    int lo = 0, hi = npr - 1;  // last r with base <= i
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pt[mid].base <= i) lo = mid; else hi = mid - 1;
    }
    const ProjEntry& e = pt[lo];
    const int64_t loc = i - e.base;
    const int32_t tl = (int32_t)(loc / e.k);
    const int32_t k = (int32_t)(loc - (int64_t)tl * e.k);
    tar = e.tar_start + tl;
    const U32x4 x = conn_draw(e.seed, (uint32_t)(tar + e.id_off), (uint32_t)k, (uint32_t)e.rid);
    src = e.src_start + (int32_t)scale_u32(x.x, (uint32_t)e.src_num);
    delay = e.dmin + (int32_t)scale_u32(x.y, (uint32_t)e.dspan);
    w = e.w;
    tar -= e.tar_sub;
}

// Keys of synapses [base, base + count) of one block; values are offsets
// from base.
__global__ void k_fid_keys(const ProjEntry* pt, int32_t npr, int64_t base, int64_t count, int dbits, int dmin,
                           uint32_t* keys, uint32_t* vals)
{
    GRID_STRIDE(j, count)
    {
        int32_t src, tar, d;
        float w;
        fid_decode(pt, npr, base + j, src, tar, d, w);
        keys[j] = ((uint32_t)src << dbits) | (uint32_t)(dbits ? d - dmin : 0);
        vals[j] = (uint32_t)j;
    }
}

__global__ void k_fid_gather(const ProjEntry* pt, int32_t npr, int64_t base, const uint32_t* order, int64_t count,
                             int tbits, uint2* syn)
{
    GRID_STRIDE(p, count)
    {
        int32_t src, tar, d;
        float w;
        fid_decode(pt, npr, base + order[p], src, tar, d, w);
        syn[p] = make_uint2((uint32_t)tar | ((uint32_t)d << tbits), __float_as_uint(w));
    }
}


// Stable radix sort of (key, value) pairs by key; keys < 2^key_bits.
template <class K>
mgc_status sort_pairs(const K* keys_in, K* keys_out, const uint32_t* vals_in, uint32_t* vals_out, int64_t S,
                      int key_bits, cudaStream_t st)
{
    if (S > (int64_t)0x7fffffff) return fail(MGC_ERR_INVALID, "more than 2^31-1 synapses in one sort");
    size_t tb = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys_in, keys_out, vals_in, vals_out, (int)S, 0, key_bits, st));
    DevTmp t;
    CK(dev_malloc(&t.p, std::max<size_t>(tb, 1)));
    CK(cub::DeviceRadixSort::SortPairs(t.p, tb, keys_in, keys_out, vals_in, vals_out, (int)S, 0, key_bits, st));
    CK(cudaStreamSynchronize(st));
    return MGC_OK;
}

// In-place exclusive scan of count+1 entries (the last entry becomes the total).
template <class T>
mgc_status exclusive_scan(T* v, int64_t count, cudaStream_t st)
{
    if (count + 1 > (int64_t)0x7fffffff) return fail(MGC_ERR_INVALID, "scan too long");
    size_t tb = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, v, v, (int)(count + 1), st));
    DevTmp t;
    CK(dev_malloc(&t.p, std::max<size_t>(tb, 1)));
    CK(cub::DeviceScan::ExclusiveSum(t.p, tb, v, v, (int)(count + 1), st));
    return MGC_OK;
}

mgc_status max_row(const int64_t* row_ptr, int32_t n, int64_t* out)
{
    std::vector<int64_t> h(n + 1);
    CK(cudaMemcpy(h.data(), row_ptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost));
    int64_t m = 0;
    for (int32_t i = 0; i < n; ++i) m = std::max(m, h[i + 1] - h[i]);
    *out = m;
    return MGC_OK;
}


// Neuron arrays, constants, step bookkeeping and raster buffers.
mgc_status init_common(mgc_sim* s, int32_t n, const int8_t* type, const float* rate, const float* v_init,
                       const float* lifc, const float* stdpc, uint64_t seed, int64_t raster_steps,
                       int64_t raster_ids)
{
    StepArgs& a = s->a;
    a.n = n;
    a.ns = (n + 3) & ~3;  // neuron arrays padded with RAW neurons for 16-byte access
    a.n_src = n;
    a.src_base = 0;
    s->n_src = n;
    const size_t ns = a.ns;
    a.seed = seed;
    memcpy(a.C, lifc, sizeof(a.C));
    if (stdpc) memcpy(a.P, stdpc, sizeof(a.P));
    if (!(lifc[0] > 0.0f)) return fail(MGC_ERR_INVALID, "lifconst[0] (DT) must be > 0");
    a.refrac_steps = (int32_t)roundf(lifc[8] / lifc[0]) - 1;  // mgcore.cu:184
    a.lifb_leak = lifc[9] != 0.0f ? lifc[9] : 0.005f;          // mgcore.cu:190
    int8_t* d_type;
    CKS(s->alloc(&d_type, ns));
    CK(cudaMemcpyAsync(d_type, type, n, cudaMemcpyHostToDevice, s->stream));
    a.type = d_type;
    a.has_cur = 0;
    for (int32_t i = 0; i < n; ++i) a.has_cur |= type[i] == kLIF || type[i] == kLIFE;
    float* d_rate;
    CKS(s->alloc(&d_rate, ns));
    if (rate) CK(cudaMemcpyAsync(d_rate, rate, 4 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
    a.rate = d_rate;
    std::vector<float> v0(ns, 0.0f);
    for (int32_t i = 0; i < n; ++i) v0[i] = v_init ? v_init[i] : lifc[1];  // mgsim.cpp:97
    // a POISSON neuron's V slot holds its probability (the update reads it
    // there); the V it reports is the initial one, which never changes
    s->pois_idx.clear();
    s->pois_v.clear();
    for (int32_t i = 0; i < n; ++i)
        if (type[i] == kPOISSON) {
            s->pois_idx.push_back(i);
            s->pois_v.push_back(v0[i]);
            v0[i] = rate ? rate[i] : 0.0f;
        }
    CKS(s->upload(&a.V, v0.data(), ns));
    CKS(s->alloc(&a.Iexc, ns));
    CKS(s->alloc(&a.Iinh, ns));
    CKS(s->alloc(&a.refrac, ns));
    CKS(s->alloc(&a.last_fired, ns));
    CKS(s->alloc(&a.fire_cnt, ns));
    CKS(s->alloc(&a.spk_count, 1));
    CKS(s->alloc(&a.step, 2));  // step, then the two slot counters
    a.slots = reinterpret_cast<int32_t*>(a.step + 1);
    CKS(s->alloc(&a.done, 1));
    CKS(s->alloc(&a.events, 1));
    CKS(s->alloc(&a.status, 1));
    CKS(s->alloc(&a.raster_pos, 1));
    CKS(s->alloc(&a.raster_step0, 1));
    s->raster_steps_cap = raster_steps > 0 ? raster_steps : kDefaultRasterSteps;
    if (raster_ids < 0) {
        a.record = 0;
        s->raster_ids_cap = 0;
    } else {
        a.record = 1;
        s->raster_ids_cap = raster_ids > 0 ? raster_ids : std::max<int64_t>(1 << 20, (int64_t)n * 64);
    }
    a.raster_steps_cap = a.record ? s->raster_steps_cap : 0;
    a.raster_ids_cap = s->raster_ids_cap;
    CKS(s->alloc(&a.raster_counts, a.record ? s->raster_steps_cap : 1, false));
    CKS(s->alloc(&a.raster_ids, a.record ? s->raster_ids_cap : 1, false));
    return MGC_OK;
}

// Delivery method for this network; fills the layout fields of s->a.
mgc_status choose_mode(mgc_sim* s, int requested)
{
    StepArgs& a = s->a;
    const int D = s->dmax - s->dmin + 1;
    const int dbits = D > 1 ? bits_for(D) : 0;
    // (a partition takes the deferred method even without synapses of its own)
    const bool deferred_ok = !s->stdp && (s->S > 0 || s->partition) && D <= kMaxBuckets &&
                             std::max(a.tbits, s->sbits) + dbits <= 32 &&
                             ((size_t)s->n_src * (size_t)D + 1) * sizeof(int64_t) <= kMaxBucketBytes;
    if (requested == MGC_MODE_DEFERRED && !deferred_ok)
        return fail(MGC_ERR_INVALID, "deferred delivery needs static weights and <= %d delays", kMaxBuckets);
    // pull: explicit networks, on request.  AUTO takes the ring push for
    // plastic networks: with STDP fused into it (k_push_stdp) and fixed-point
    // sums it is deterministic too, and it ran 11.7 us per step against 42.3
    // for the pull on the 3.8e6-synapse STDP network of 784 -> 1,600 neurons
    const bool pull_ok = s->explicit_net && s->S < (int64_t(1) << 32) && a.tbits + dbits <= 32;
    if (requested == MGC_MODE_PULL && !pull_ok)
        return fail(MGC_ERR_INVALID, "the pull method needs an explicit synapse list of < 2^32 synapses");
    if (requested == MGC_MODE_PULL) {
        s->mode = MGC_MODE_PULL;
        a.pull = 1;
        a.deferred = 0;
        a.D = D;
        a.dmin = s->dmin;
        a.H = 1;
        return MGC_OK;
    }
    if (requested == MGC_MODE_PUSH || !deferred_ok) {
        s->mode = MGC_MODE_PUSH;
        a.deferred = 0;
        a.D = 1;
        a.H = 1;
    } else {
        s->mode = MGC_MODE_DEFERRED;
        a.deferred = 1;
        a.D = D;
        a.dmin = s->dmin;
        // the step groups clear the history slots of the steps up to a
        // window (the pipelined group: 3 steps) ahead
        a.H = s->dmax + std::max(4, std::min(kMaxWindow, s->dmin));
    }
    return MGC_OK;
}

int sort_dbits(const mgc_sim* s) { return s->a.deferred && s->a.D > 1 ? bits_for(s->a.D) : 0; }

// Row and bucket counts are accumulated from sorted keys (one call per
// sorted block), then turned into offsets by finish_build.
mgc_status begin_layout(mgc_sim* s)
{
    StepArgs& a = s->a;
    int64_t* row_ptr;
    CKS(s->alloc(&row_ptr, (size_t)s->n_src + 1));
    a.row_ptr = row_ptr;
    if (a.deferred) {
        int64_t* bucket;
        CKS(s->alloc(&bucket, (size_t)s->n_src * a.D + 1));
        a.bucket = bucket;
    }
    return MGC_OK;
}

void count_keys(mgc_sim* s, const uint32_t* keys, int64_t count)
{
    if (count <= 0) return;
    const int dbits = sort_dbits(s);
    k_count_rows<<<grid_for(count), 256, 0, s->stream>>>(keys, count, dbits, const_cast<int64_t*>(s->a.row_ptr));
    if (s->a.deferred)
        k_count_buckets<<<grid_for(count), 256, 0, s->stream>>>(keys, count, dbits, s->a.D,
                                                                 const_cast<int64_t*>(s->a.bucket));
}


// Trace buffers and scheduler state of the fused method.  Trace population
// of a neuron: as the builder set it (population index, or neuron type class
// for synapse-list networks), clamped to kTracePops - 1.
mgc_status init_sched(mgc_sim* s)
{
    StepArgs& a = s->a;
    std::vector<uint8_t> tp(a.ns, 0);
    for (size_t i = 0; i < s->tpop_host.size() && i < tp.size(); ++i)
        tp[i] = (uint8_t)std::min<int>(s->tpop_host[i], kTracePops - 1);
    uint8_t* d_tp;
    CKS(s->upload(&d_tp, tp.data(), tp.size()));
    a.tpop = d_tp;
    CKS(s->alloc(&a.trace, (size_t)kTraceSteps * kTraceCols));
    CKS(s->alloc(&a.ev_mark, 1));
    CKS(s->alloc(&a.bar, 4));
    CKS(s->alloc(&s->sched, 1));
    CKS(s->alloc(&s->sched_data, (size_t)kMaxDataset * kTraceCols));
    SchedState h;
    memset(&h, 0, sizeof(h));
    h.mode = kSchedStatic;
    h.static_variant = s->fused_variant;
    h.forced_variant = -1;
    h.threshold = 1e30f;
    h.hi_variant = 1;
    for (int i = 0; i < kMlpIn; ++i) h.xs[i] = 1.f;
    for (int o = 0; o < kMlpOut; ++o) h.ys[o] = 1.f;
    CK(cudaMemcpyAsync(s->sched, &h, sizeof(h), cudaMemcpyHostToDevice, s->stream));
    return MGC_OK;
}


// Shared tail of the builders: offsets, method buffers and launch shapes.
mgc_status finish_build(mgc_sim* s)
{
    StepArgs& a = s->a;
    int64_t* row_ptr = const_cast<int64_t*>(a.row_ptr);
    int64_t max_len = 0;
    CKS(exclusive_scan(row_ptr, s->n_src, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (s->S > 0) CKS(max_row(row_ptr, s->n_src, &max_len));
    a.chunks_per_spike = (int32_t)std::max<int64_t>(1, (max_len + kChunk - 1) / kChunk);
    const size_t words = a.fx ? 2 : 1;  // accumulator entries: fp32, or 64-bit fixed point
    if (a.deferred) {
        const int64_t nb = (int64_t)s->n_src * a.D;
        int64_t* bucket = const_cast<int64_t*>(a.bucket);
        CKS(exclusive_scan(bucket, nb, s->stream));
        DevTmp t;
        unsigned long long* dmax_gap;
        CKS(tmp_alloc(t, &dmax_gap, 1));
        CK(cudaMemsetAsync(dmax_gap, 0, 8, s->stream));
        k_max_gap<<<grid_for(nb), 256, 0, s->stream>>>(bucket, nb, dmax_gap);
        unsigned long long gap = 0;
        CK(cudaMemcpyAsync(&gap, dmax_gap, 8, cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        // long segments (few delays, large out-degree) are cut into chunks so
        // one step's synapses spread over all warps
        set_chunking(a, (int64_t)gap, kDefaultChunk);
        s->max_gap = (int64_t)gap;
        CKS(s->alloc(&a.hist_ids, (size_t)a.H * s->n_src, false));
        CKS(s->alloc(&a.hist_cnt, a.H));
        // step buffers, s & acc_mask; eight when windows of 5 steps or more fit
        s->acc_buffers = s->dmin > kAccBuffers ? kAccBuffersWide : kAccBuffers;
        a.acc_mask = kAccBuffers - 1;
        CKS(s->alloc(&a.acc_e, s->acc_buffers * (size_t)a.ns * words));
        CKS(s->alloc(&a.acc_i, s->acc_buffers * (size_t)a.ns * words));
        // fused step kernel: one resident wave, every warp updates then delivers
        s->fused = s->dmin >= 2;
        s->fused_variant = 1;
        // step groups by default (faster than one launch per step on every
        // measured load); the pipelined form needs a minimum delay >= 4.
        // The windowed form is faster on the measured loads; the autotuner
        // or the caller selects it
        s->persistent = s->fused ? (s->dmin >= 4 ? 2 : 1) : 1;
        if (!s->fused) CKS(s->alloc(&a.bar, 4));  // the grid barrier's arrivals and generation
        if (s->fused) {
            // windowed group: the delivery prefixes of a window's steps in
            // dynamic shared memory (up to 4, or 8 for the wide instantiation)
            s->window = std::min(kMaxWindow, s->dmin);
            for (int wide = 0; wide < 2; ++wide) {
                const size_t steps = wide ? kMaxWindow : kAccBuffers;
                s->window_smem[wide] = steps * (size_t)(a.D + 1) * sizeof(int64_t);
            }
            CKS(init_sched(s));
        }
    } else {
        a.M = s->M;
        CKS(s->alloc(&a.ring_e, (size_t)s->M * a.ns * words));
        CKS(s->alloc(&a.ring_i, (size_t)s->M * a.ns * words));
        CKS(s->alloc(&a.spk, s->n));
        if (a.pull || s->stdp) {  // this step's spikes as a bitmap (the pull, the ring STDP's incoming side)
            const int64_t groups = a.ns / 4;
            CKS(s->alloc(&a.fired_bits, (size_t)((groups + 31) / 32) * 4));
        }
    }
    a.M = s->M;
    CKS(launch_shapes(s));
    CK(cudaStreamSynchronize(s->stream));
    return MGC_OK;
}


mgc_status check_tbits(mgc_sim* s)
{
    StepArgs& a = s->a;
    a.tbits = bits_for(s->n);
    a.tmask = a.tbits >= 32 ? 0xffffffffu : ((1u << a.tbits) - 1u);
    s->sbits = bits_for(s->n_src);
    if (a.tbits + bits_for((int64_t)s->dmax + 1) > 32)
        return fail(MGC_ERR_INVALID, "max delay %d with %d neurons does not fit a 32-bit CSR word", s->dmax, s->n);
    return MGC_OK;
}

// One partition of a larger network: the handle simulates neurons
// [first, first + count) of n_src, holds the synapses that target them
// (targets renumbered from 0, sources kept) and takes the whole network's
// delay range, so that every partition has the same history length and
// exchange window.
struct PartSpec {
    int32_t n_src, first, count, dmin, dmax;
    bool fx_given;   // the accumulation plan of the whole network (fx), not of the partition's synapses
    struct FxPlan {
        bool hetero;     // some neuron receives unequal weights of one sign
        int32_t shift;   // fixed-point shift for the network's weights
    } fx;
};
using FxPlan = PartSpec::FxPlan;

// Shift of the fixed-point accumulation: the largest for which any neuron's
// sum of one step fits 61 bits (bound = the largest sum of |w| over one
// neuron's incoming synapses; a synapse delivers at most once per arrival
// step), and no larger than needed to make every weight an exact multiple
// of 2^-shift (min_exp: the smallest frexp exponent of a nonzero |w|; the
// 24-bit mantissa's last bit is 2^(e-24)).  Kept within the range where
// 2^shift and 2^-shift are normal floats.
int32_t fx_shift_for(double bound, int min_exp, bool exact)
{
    int k = 0;
    if (bound > 0.0) {
        int e = 0;
        std::frexp(bound, &e);  // bound < 2^e
        k = 61 - e;
        if (exact) k = std::min(k, 24 - min_exp);
    }
    return std::max(-100, std::min(120, k));
}

// The plan of a synapse list (targets, weights); plastic synapses may take
// any weight up to wlim in magnitude.
FxPlan fx_plan_list(int32_t n, int64_t S, const int32_t* tar, const float* w, const uint8_t* plastic, bool stdp,
                    float wlim)
{
    std::vector<float> first_e(n, 0.0f), first_i(n, 1.0f);  // 1.0: no inhibitory weight seen yet
    std::vector<double> sum(n, 0.0);
    bool hetero = false, any_plastic = false;
    int min_exp = 1 << 20;
    for (int64_t k = 0; k < S; ++k) {
        const int32_t t = tar[k];
        if (t < 0 || t >= n) continue;  // refused later by validation
        const float x = w[k];
        const bool pl = stdp && (!plastic || plastic[k]);
        any_plastic |= pl;
        sum[t] += pl ? std::max((double)std::fabs(x), (double)wlim) : (double)std::fabs(x);
        if (x != 0.0f) {
            int e = 0;
            std::frexp(x, &e);
            min_exp = std::min(min_exp, e);
        }
        if (x > 0.0f) {
            if (first_e[t] == 0.0f) first_e[t] = x;
            else hetero |= first_e[t] != x;
        } else {
            if (first_i[t] == 1.0f) first_i[t] = x;
            else hetero |= first_i[t] != x;
        }
    }
    double bound = 0.0;
    for (int32_t t = 0; t < n; ++t) bound = std::max(bound, sum[t]);
    return FxPlan{hetero || any_plastic, fx_shift_for(bound, min_exp, !any_plastic)};
}

// The plan of fixed in-degree blocks: projection r gives each neuron of its
// target population pr_k[r] synapses of weight pr_w[r].
FxPlan fx_plan_blocks(const mgc_fixed_indegree_desc* blocks, int32_t n_blocks)
{
    bool hetero = false;
    double bound = 0.0;
    int min_exp = 1 << 20;
    for (int b = 0; b < n_blocks; ++b) {
        const mgc_fixed_indegree_desc& d = blocks[b];
        for (int tp = 0; tp < d.n_pops; ++tp) {
            double sum = 0.0;
            float we = 0.0f, wi = 1.0f;
            for (int r = 0; r < d.n_proj; ++r) {
                if (d.pr_tar[r] != tp || d.pr_k[r] <= 0) continue;
                const float x = d.pr_w[r];
                sum += (double)d.pr_k[r] * std::fabs((double)x);
                if (x != 0.0f) {
                    int e = 0;
                    std::frexp(x, &e);
                    min_exp = std::min(min_exp, e);
                }
                if (x > 0.0f) {
                    hetero |= we != 0.0f && we != x;
                    we = x;
                } else {
                    hetero |= wi != 1.0f && wi != x;
                    wi = x;
                }
            }
            bound = std::max(bound, sum);
        }
    }
    return FxPlan{hetero, fx_shift_for(bound, min_exp, true)};
}

// Turns fixed-point accumulation on when some neuron receives unequal
// weights of one sign (their fp32 sum would depend on the arrival order),
// except for the pull method, whose per-target pass adds in a fixed order.
void apply_fx(mgc_sim* s, const FxPlan& p)
{
    s->hetero = p.hetero;
    s->fx_shift = p.shift;
    s->a.fx = p.hetero && !s->a.pull ? 1 : 0;
    s->a.fx_scale = std::ldexp(1.0f, p.shift);
    s->a.fx_unscale = std::ldexp(1.0f, -p.shift);
}

// Applies a partition spec to a handle whose neuron arrays are built.
void apply_part(mgc_sim* s, const PartSpec& p)
{
    s->partition = true;
    s->n_src = p.n_src;
    s->a.n_src = p.n_src;
    s->a.src_base = p.first;
}

mgc_status create_explicit(const mgc_net_desc* d, const PartSpec* part, mgc_sim** out);
mgc_status create_fixed_indegree(const mgc_fixed_indegree_desc* blocks, int32_t n_blocks, const PartSpec* part,
                                 mgc_sim** out);

}  // namespace

namespace mgc {

// Grids of the kernels this handle launches, from their occupancy (which
// depends on the instantiation: current arrays, register budget, fp32 or
// fixed-point accumulation).  Step groups are cooperative launches whose
// blocks must all be resident.
mgc_status launch_shapes(mgc_sim* s)
{
    StepArgs& a = s->a;
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, s->device));
    const int sms = prop.multiProcessorCount;
    int occ = 0;
    if (a.deferred) {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, deliver_kernel(s), kPushBlock, 0));
        s->deliver_grid = sms * std::max(1, occ);
        if (s->fused) {
            for (int v = 0; v < 2; ++v) {
                CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fused_kernel(s, v), kPushBlock, 0));
                s->fused_grid_v[v] = sms * std::min(std::max(1, occ), v == 0 ? 2 : 3);
            }
            s->fused_grid = s->fused_grid_v[s->fused_variant];
            for (int p = 1; p <= 2; ++p)
                for (int v = 0; v < 2; ++v) {
                    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, steps_kernel(s, p, v), kPushBlock, 0));
                    s->group_grid_v[p - 1][v] = sms * std::min(std::max(1, occ), v == 0 ? 2 : 3);
                }
            for (int wide = 0; wide < 2; ++wide)
                for (int v = 0; v < 2; ++v) {
                    for (int pl = 0; pl < 2; ++pl)
                        CK(cudaFuncSetAttribute((const void*)window_kernel(s, v, wide, pl),
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->window_smem[wide]));
                    // both forms of a variant are compiled for the same blocks per SM
                    const WindowKernel k = window_kernel(s, v, wide, false);
                    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, kPushBlock, s->window_smem[wide]));
                    s->window_grid_v[wide][v] = sms * std::min(std::max(1, occ), v == 0 ? 2 : 3);
                }
        } else {
            // minimum delay 1: a barrier-per-phase step group sized to the
            // neurons (8 warps x 64 neuron groups a block per pass)
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, steps_kernel(s, 1, 0), kPushBlock, 0));
            const int64_t wave = (int64_t)sms * std::max(1, occ);
            const int64_t want = ((int64_t)a.ns / 4 + 511) / 512;
            s->group_grid1 = (int)std::max<int64_t>(1, std::min(wave, want));
        }
    } else {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, push_kernel(s), kPushBlock, 0));
        s->push_grid = sms * std::max(1, occ);
        if (a.pull) {
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pull_kernel(s), kPushBlock, 0));
            s->pull_grid = sms * std::max(1, occ);
        }
    }
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, neuron_kernel(s), kNeuronBlock, 0));
    s->neuron_grid = (int)std::max<int64_t>(
        1, std::min<int64_t>((int64_t)sms * std::max(1, occ), (a.ns / 4 + kNeuronBlock - 1) / kNeuronBlock));
    return MGC_OK;
}

// Segments of up to `gap` synapses cut into chunks of about `target`
// (a multiple of 32), at most kMaxChunks per segment.
void set_chunking(StepArgs& a, int64_t gap, int64_t target)
{
    int64_t ch = std::max<int64_t>(1, (gap + target - 1) / target);
    ch = std::min<int64_t>(ch, kMaxChunks);
    int64_t len = (std::max<int64_t>(gap, 1) + ch - 1) / ch;
    len = (len + 31) / 32 * 32;
    a.bucket_chunks = (int32_t)ch;
    a.chunk_len = (int32_t)len;
}

// Construction steps for the other builders (netgen.cu): the neuron arrays,
// the method (with the fixed-point plan), and the shared tail.
mgc_status build_neurons(mgc_sim* s, int32_t n, const int8_t* type, const float* rate, const float* v_init,
                         const float* lifc, const float* stdpc, uint64_t seed, int64_t raster_steps,
                         int64_t raster_ids)
{
    return init_common(s, n, type, rate, v_init, lifc, stdpc, seed, raster_steps, raster_ids);
}

mgc_status build_method(mgc_sim* s, int requested, bool hetero, int32_t fx_shift)
{
    CKS(check_tbits(s));
    CKS(choose_mode(s, requested));
    apply_fx(s, FxPlan{hetero, fx_shift});
    return MGC_OK;
}

int32_t fx_shift_rule(double bound, int min_exp, bool exact) { return fx_shift_for(bound, min_exp, exact); }

mgc_status build_set_fx(mgc_sim* s, bool hetero, int32_t fx_shift)
{
    apply_fx(s, FxPlan{hetero, fx_shift});
    return MGC_OK;
}

mgc_status build_finish(mgc_sim* s) { return finish_build(s); }

// The CSR (and the method's extra layouts) of a network handed over as a
// device-resident synapse list in synapse-list order: sources, targets,
// weights, delays in steps and (STDP) plasticity flags (or null).  The
// builders call begin_list_layout once the method is chosen, then this.
mgc_status begin_list_layout(mgc_sim* s)
{
    StepArgs& a = s->a;
    CKS(begin_layout(s));
    uint2* syn;
    CKS(s->alloc(&syn, s->S, false));
    a.syn = syn;
    a.n_syn = s->S;
    CKS(s->alloc(&s->csr_syn64, s->S, false));
    return MGC_OK;
}

mgc_status csr_from_list(mgc_sim* s, int32_t* src, int32_t* tar, float* w, int32_t* dl, uint8_t* pl)
{
    StepArgs& a = s->a;
    const int64_t S = s->S;
    const int dbits = sort_dbits(s);
    uint2* syn = a.syn;
    DevTmp t_keys2;
    uint32_t* keys2 = nullptr;
    {
        DevTmp t_keys, t_vals, t_order, t_bad;
        int32_t* bad;
        uint32_t *keys, *vals, *order;
        CKS(tmp_alloc(t_bad, &bad, 1));
        CK(cudaMemsetAsync(bad, 0, 4, s->stream));
        k_validate<<<grid_for(S), 256, 0, s->stream>>>(src, tar, dl, S, s->n_src, s->n, 1 << (32 - a.tbits), bad);
        int32_t hbad = 0;
        CK(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        if (hbad) return fail(MGC_ERR_INVALID, "synapse with out-of-range source, target or delay");
        if (a.pull) {
            const int db = s->dmax > s->dmin ? bits_for(s->dmax - s->dmin + 1) : 0;
            DevTmp t_k64a, t_k64b, t_v, t_o;
            uint64_t *k64a, *k64b;
            uint32_t *pv, *po;
            CKS(tmp_alloc(t_k64a, &k64a, S));
            CKS(tmp_alloc(t_k64b, &k64b, S));
            CKS(tmp_alloc(t_v, &pv, S));
            CKS(tmp_alloc(t_o, &po, S));
            k_pull_keys<<<grid_for(S), 256, 0, s->stream>>>(src, tar, dl, S, a.tbits, db, s->dmin, k64a, pv);
            CKS(sort_pairs(k64a, k64b, pv, po, S, 2 * a.tbits + db, s->stream));
            int64_t* in_ptr;
            uint2* in_ent;
            uint8_t* in_pl = nullptr;
            CKS(s->alloc(&in_ptr, (size_t)s->n + 1));
            CKS(s->alloc(&in_ent, S, false));
            CKS(s->alloc(&s->in_syn64, S, false));
            if (s->stdp && pl) CKS(s->alloc(&in_pl, S, false));
            k_gather_pull<<<grid_for(S), 256, 0, s->stream>>>(po, src, w, dl, pl, S, a.tbits, in_ent, s->in_syn64,
                                                               in_pl);
            uint32_t* tkeys = reinterpret_cast<uint32_t*>(pv);
            k_cast_keys<<<grid_for(S), 256, 0, s->stream>>>(tar, S, tkeys);
            k_count_rows<<<grid_for(S), 256, 0, s->stream>>>(tkeys, S, 0, in_ptr);
            CKS(exclusive_scan(in_ptr, s->n, s->stream));
            CK(cudaStreamSynchronize(s->stream));
            a.in_ptr = in_ptr;
            a.in_ent = in_ent;
            a.in_plastic = in_pl;
        }
        // CSR by source (and delay bucket), synapse-list order inside (stable)
        CKS(tmp_alloc(t_keys, &keys, S));
        CKS(tmp_alloc(t_vals, &vals, S));
        CKS(tmp_alloc(t_order, &order, S));
        CKS(tmp_alloc(t_keys2, &keys2, S));
        k_explicit_keys<<<grid_for(S), 256, 0, s->stream>>>(src, dl, S, dbits, s->dmin, keys, vals);
        CKS(sort_pairs(keys, keys2, vals, order, S, s->sbits + dbits, s->stream));
        int32_t* csr_src = nullptr;
        uint8_t* plastic = nullptr;
        if (s->stdp && !a.pull) {
            CKS(s->alloc(&csr_src, S, false));
            if (pl) CKS(s->alloc(&plastic, S, false));
        }
        k_gather_explicit<<<grid_for(S), 256, 0, s->stream>>>(order, keys2, dbits, tar, w, dl, pl, S, a.tbits, syn,
                                                               s->csr_syn64, csr_src, plastic);
        a.csr_src = csr_src;
        a.plastic = plastic;
        if (s->stdp && !a.pull) {
            // incoming lists: CSR positions sorted by target, synapse-list order
            int64_t* dend_off;
            int64_t* dend_pos;
            CKS(s->alloc(&dend_off, (size_t)s->n + 1));
            CKS(s->alloc(&dend_pos, S, false));
            k_cast_keys<<<grid_for(S), 256, 0, s->stream>>>(tar, S, keys);
            k_count_rows<<<grid_for(S), 256, 0, s->stream>>>(keys, S, 0, dend_off);
            CKS(exclusive_scan(dend_off, s->n, s->stream));
            k_inverse<<<grid_for(S), 256, 0, s->stream>>>(s->csr_syn64, S, vals);  // vals := pos_of
            uint32_t* keys_out = reinterpret_cast<uint32_t*>(src);  // src is no longer needed
            CKS(sort_pairs(keys, keys_out, vals, order, S, a.tbits, s->stream));
            k_widen<<<grid_for(S), 256, 0, s->stream>>>(order, S, dend_pos);
            a.dend_off = dend_off;
            a.dend_pos = dend_pos;
            int64_t max_in = 0;
            CK(cudaStreamSynchronize(s->stream));
            CKS(max_row(dend_off, s->n, &max_in));
            a.chunks_in_per_spike = (int32_t)std::max<int64_t>(1, (max_in + kChunk - 1) / kChunk);
        }
        count_keys(s, keys2, S);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s->stream));
    }
    return MGC_OK;
}


// The deferred method's incoming rows and history bitmaps for pull steps
// (mgc_set_pull), built once from the handle's CSR: rows by target, in CSR
// order inside (a stable sort), entries {source | delay << tbits, weight}.
mgc_status build_in_rows(mgc_sim* s)
{
    StepArgs& a = s->a;
    if (a.in_ent) return MGC_OK;
    const int64_t S = s->S;
    if (S >= (int64_t(1) << 32)) return fail(MGC_ERR_INVALID, "pull steps need fewer than 2^32 synapses");
    int64_t* in_ptr = nullptr;
    uint2* in_ent = nullptr;
    uint32_t* bits = nullptr;
    const int64_t groups = a.ns / 4;
    const int32_t words = (int32_t)((groups + 31) / 32 * 4);
    CKS(s->alloc(&in_ptr, (size_t)s->n + 1));
    CKS(s->alloc(&in_ent, (size_t)std::max<int64_t>(S, 1), false));
    CKS(s->alloc(&bits, (size_t)a.H * (size_t)words));
    int64_t* span = nullptr;
    CKS(s->alloc(&span, 2));
    {
        DevTmp t_k, t_k2, t_p, t_o, t_s;
        uint32_t *k, *k2, *pos, *order;
        int32_t* src_of;
        CKS(tmp_alloc(t_k, &k, S));
        CKS(tmp_alloc(t_k2, &k2, S));
        CKS(tmp_alloc(t_p, &pos, S));
        CKS(tmp_alloc(t_o, &order, S));
        CKS(tmp_alloc(t_s, &src_of, S));
        if (S > 0) {
            k_row_sources<<<grid_for((int64_t)s->n_src * 32), 256, 0, s->stream>>>(a.bucket, s->n_src, a.D, a.syn,
                                                                                    a.tmask, k, pos, src_of);
            CKS(sort_pairs(k, k2, pos, order, S, a.tbits, s->stream));
            k_gather_in<<<grid_for(S), 256, 0, s->stream>>>(order, a.syn, src_of, S, a.tmask, in_ent);
            k_count_rows<<<grid_for(S), 256, 0, s->stream>>>(k2, S, 0, in_ptr);
        }
        CKS(exclusive_scan(in_ptr, s->n, s->stream));
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s->stream));
    }
    a.in_ptr = in_ptr;
    a.in_ent = in_ent;
    a.hist_bits = bits;
    a.bits_words = words;
    a.bits_span = span;
    const int64_t none[2] = {0, -1};  // no step has its bitmap yet
    CK(cudaMemcpy(span, none, sizeof(none), cudaMemcpyHostToDevice));
    return MGC_OK;
}

void release_in_rows(mgc_sim* s)
{
    StepArgs& a = s->a;
    if (a.pull || !a.in_ent) return;  // the pull method's rows are its synapses
    cudaStreamSynchronize(s->stream);
    for (void* p : {(void*)a.in_ptr, (void*)a.in_ent, (void*)a.hist_bits, (void*)a.bits_span}) s->release(p);
    a.in_ptr = nullptr;
    a.in_ent = nullptr;
    a.hist_bits = nullptr;
    a.bits_span = nullptr;
    a.bits_words = 0;
    a.pull_min = 0;
}

}  // namespace mgc

extern "C" {

mgc_status mgc_create(const mgc_net_desc* d, mgc_sim** out) { return create_explicit(d, nullptr, out); }

mgc_status mgc_create_partition(const mgc_net_desc* d, int32_t first, int32_t count, mgc_sim** out)
{
    if (!d || !out) return fail(MGC_ERR_INVALID, "null argument");
    *out = nullptr;
    if (d->n_neurons <= 0 || !d->type) return fail(MGC_ERR_INVALID, "network needs neurons and types");
    if (first < 0 || count <= 0 || (int64_t)first + count > d->n_neurons)
        return fail(MGC_ERR_INVALID, "partition [%d, %lld) outside the network's %d neurons", first,
                    (long long)first + count, d->n_neurons);
    if (d->stdp) return fail(MGC_ERR_INVALID, "a partition needs static weights (the deferred method)");
    if (d->mode != MGC_MODE_AUTO && d->mode != MGC_MODE_DEFERRED)
        return fail(MGC_ERR_INVALID, "a partition runs the deferred method");
    if (d->n_synapses < 0 || (d->n_synapses > 0 && (!d->syn_src || !d->syn_tar || !d->syn_weight || !d->syn_delay)))
        return fail(MGC_ERR_INVALID, "synapse arrays missing");
    // the whole network's delay range; the synapses of this partition's targets
    PartSpec p{d->n_neurons, first, count, 0x7fffffff, 0, true,
               fx_plan_list(d->n_neurons, d->n_synapses, d->syn_tar, d->syn_weight, nullptr, false, 0.0f)};
    std::vector<int32_t> src, tar, dl;
    std::vector<float> w;
    const int32_t last = first + count;
    for (int64_t k = 0; k < d->n_synapses; ++k) {
        p.dmin = std::min(p.dmin, d->syn_delay[k]);
        p.dmax = std::max(p.dmax, d->syn_delay[k]);
        const int32_t t = d->syn_tar[k];
        if (t < first || t >= last) continue;
        src.push_back(d->syn_src[k]);
        tar.push_back(t - first);
        dl.push_back(d->syn_delay[k]);
        w.push_back(d->syn_weight[k]);
    }
    if (d->n_synapses == 0) p.dmin = p.dmax = 1;
    if (p.dmin < 2)
        return fail(MGC_ERR_INVALID, "partitions exchange spikes every min_delay - 1 steps: min_delay %d < 2", p.dmin);
    mgc_net_desc loc = *d;
    loc.n_neurons = count;
    loc.type = d->type + first;
    loc.rate = d->rate ? d->rate + first : nullptr;
    loc.v_init = d->v_init ? d->v_init + first : nullptr;
    loc.n_synapses = (int64_t)src.size();
    loc.syn_src = src.data();
    loc.syn_tar = tar.data();
    loc.syn_weight = w.data();
    loc.syn_delay = dl.data();
    loc.syn_plastic = nullptr;
    loc.mode = MGC_MODE_DEFERRED;
    loc.id_offset = d->id_offset + first;  // POISSON draws keyed by the global id
    return create_explicit(&loc, &p, out);
}

}  // extern "C"

namespace {

mgc_status create_explicit(const mgc_net_desc* d, const PartSpec* part, mgc_sim** out)
{
    if (!d || !out) return fail(MGC_ERR_INVALID, "null argument");
    *out = nullptr;
    if (d->n_neurons <= 0 || !d->type) return fail(MGC_ERR_INVALID, "network needs neurons and types");
    if (d->n_synapses < 0 || (d->n_synapses > 0 && (!d->syn_src || !d->syn_tar || !d->syn_weight || !d->syn_delay)))
        return fail(MGC_ERR_INVALID, "synapse arrays missing");
    if (d->mode < MGC_MODE_AUTO || d->mode > MGC_MODE_PULL) return fail(MGC_ERR_INVALID, "unknown mode %d", d->mode);
    CKS(pick_device(d->device));
    std::unique_ptr<mgc_sim> s(new mgc_sim);
    s->device = d->device;
    CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->n = d->n_neurons;
    s->S = d->n_synapses;
    s->stdp = d->stdp != 0;
    s->explicit_net = true;
    CKS(init_common(s.get(), s->n, d->type, d->rate, d->v_init, d->lifconst, d->stdpconst, d->seed,
                    d->raster_steps, d->raster_ids));
    if (part) apply_part(s.get(), *part);
    StepArgs& a = s->a;
    a.stdp = s->stdp;
    a.id_offset = d->id_offset;
    // trace populations by neuron type: POISSON, LIF family, the rest
    s->tpop_host.resize(s->n);
    for (int32_t i = 0; i < s->n; ++i) {
        const int t = d->type[i];
        s->tpop_host[i] = t == MGC_POISSON ? 0 : (t == MGC_LIF || t == MGC_LIFE || t == MGC_LIFB ? 1 : 2);
    }
    const int64_t S = s->S;
    // delay range (mgsim.cpp:42-51); M = max_delay + 1 (:71)
    int32_t dmin = 0x7fffffff, dmax = 0;
    for (int64_t k = 0; k < S; ++k) {
        dmin = std::min(dmin, d->syn_delay[k]);
        dmax = std::max(dmax, d->syn_delay[k]);
    }
    if (S == 0) dmin = dmax = 1;
    if (dmin < 1) return fail(MGC_ERR_INVALID, "synaptic delay below one step (%d)", dmin);
    if (part) {
        dmin = part->dmin;
        dmax = part->dmax;
    }
    s->dmin = dmin;
    s->dmax = dmax;
    s->M = dmax + 1;
    CKS(check_tbits(s.get()));
    CKS(choose_mode(s.get(), d->mode));
    apply_fx(s.get(), part && part->fx_given
                          ? part->fx
                          : fx_plan_list(s->n, S, d->syn_tar, d->syn_weight, d->syn_plastic, s->stdp,
                                         std::max(std::fabs(d->stdpconst[4]), std::fabs(d->stdpconst[5]))));
    CKS(begin_list_layout(s.get()));
    if (S > 0) {
        DevTmp t_src, t_tar, t_w, t_d, t_pl;
        int32_t *src, *tar, *dl;
        float* w;
        uint8_t* pl = nullptr;
        CKS(tmp_alloc(t_src, &src, S));
        CKS(tmp_alloc(t_tar, &tar, S));
        CKS(tmp_alloc(t_w, &w, S));
        CKS(tmp_alloc(t_d, &dl, S));
        CK(cudaMemcpyAsync(src, d->syn_src, 4 * S, cudaMemcpyHostToDevice, s->stream));
        CK(cudaMemcpyAsync(tar, d->syn_tar, 4 * S, cudaMemcpyHostToDevice, s->stream));
        CK(cudaMemcpyAsync(w, d->syn_weight, 4 * S, cudaMemcpyHostToDevice, s->stream));
        CK(cudaMemcpyAsync(dl, d->syn_delay, 4 * S, cudaMemcpyHostToDevice, s->stream));
        if (s->stdp && d->syn_plastic) {
            CKS(tmp_alloc(t_pl, &pl, S));
            CK(cudaMemcpyAsync(pl, d->syn_plastic, S, cudaMemcpyHostToDevice, s->stream));
        }
        CKS(csr_from_list(s.get(), src, tar, w, dl, pl));
    }
    CKS(finish_build(s.get()));
    *out = s.release();
    return MGC_OK;
}

// Independent fixed in-degree networks ("blocks") laid side by side in one
// handle: block b's neurons get ids [start_b, start_b + n_b) with start_b
// the sum of the earlier blocks' sizes, its populations are relative to
// start_b, and its synapses and draws are those it would generate alone with
// id_offset = start_b and proj_offset = the number of earlier projections.
// Each block is generated and sorted separately (a block's synapses occupy
// one contiguous CSR range), so the total may exceed what one sort takes.
// With a partition spec (one block): only the neurons [first, first + count)
// and the synapses that target them, drawn as in the whole network.
mgc_status create_fixed_indegree(const mgc_fixed_indegree_desc* blocks, int32_t n_blocks, const PartSpec* part,
                                 mgc_sim** out)
{
    if (!blocks || !out || n_blocks <= 0) return fail(MGC_ERR_INVALID, "null argument or no blocks");
    *out = nullptr;
    if (part && n_blocks != 1) return fail(MGC_ERR_INVALID, "a partition is cut from one network");
    const mgc_fixed_indegree_desc& d0 = blocks[0];
    if (d0.mode < MGC_MODE_AUTO || d0.mode > MGC_MODE_DEFERRED)
        return fail(MGC_ERR_INVALID, "unknown mode %d", d0.mode);
    CKS(pick_device(d0.device));
    std::vector<int64_t> start(n_blocks + 1, 0), pbase(n_blocks + 1, 0), sbase(n_blocks + 1, 0);
    std::vector<ProjEntry> pt;
    int32_t dmin = 0x7fffffff, dmax = 0;
    for (int b = 0; b < n_blocks; ++b) {
        const mgc_fixed_indegree_desc& d = blocks[b];
        if (d.n_pops <= 0 || d.n_proj < 0) return fail(MGC_ERR_INVALID, "block %d: need 1+ populations", b);
        if (memcmp(d.lifconst, d0.lifconst, sizeof(d0.lifconst)) != 0)
            return fail(MGC_ERR_INVALID, "block %d: blocks share one LIF constant set", b);
        int64_t nb = 0;
        for (int p = 0; p < d.n_pops; ++p) {
            if (d.pop_start[p] < 0 || d.pop_num[p] < 0) return fail(MGC_ERR_INVALID, "block %d: bad population %d", b, p);
            nb = std::max<int64_t>(nb, (int64_t)d.pop_start[p] + d.pop_num[p]);
        }
        start[b + 1] = start[b] + nb;
        int64_t S = sbase[b];
        for (int r = 0; r < d.n_proj; ++r) {
            const int sp = d.pr_src[r], tp = d.pr_tar[r];
            if (sp < 0 || sp >= d.n_pops || tp < 0 || tp >= d.n_pops || d.pr_k[r] < 0 || d.pr_dmin[r] < 1 ||
                d.pr_dmax[r] < d.pr_dmin[r] || (d.pr_k[r] > 0 && d.pop_num[sp] == 0))
                return fail(MGC_ERR_INVALID, "block %d: bad projection %d", b, r);
            ProjEntry e{};
            e.base = S;
            e.src_start = (int32_t)start[b] + d.pop_start[sp];
            e.src_num = d.pop_num[sp];
            e.tar_start = (int32_t)start[b] + d.pop_start[tp];
            int32_t tar_num = d.pop_num[tp];
            if (part) {  // the targets inside the partition, renumbered from its first neuron
                const int64_t lo = std::max<int64_t>(e.tar_start, part->first);
                const int64_t hi = std::min<int64_t>((int64_t)e.tar_start + tar_num, (int64_t)part->first + part->count);
                e.tar_start = (int32_t)lo;
                tar_num = (int32_t)std::max<int64_t>(0, hi - lo);
                e.tar_sub = part->first;
            }
            e.k = std::max(1, d.pr_k[r]);
            e.dmin = d.pr_dmin[r];
            e.dspan = d.pr_dmax[r] - d.pr_dmin[r] + 1;
            e.w = d.pr_w[r];
            e.seed = d.conn_seed;
            e.rid = (int32_t)(pbase[b] + r + d.proj_offset);
            e.id_off = d.id_offset;  // block-local ids are already shifted by start_b
            pt.push_back(e);
            const int64_t sr = (int64_t)tar_num * d.pr_k[r];
            S += sr;
            if ((int64_t)d.pop_num[tp] * d.pr_k[r] > 0) {  // the whole network's delay range
                dmin = std::min(dmin, d.pr_dmin[r]);
                dmax = std::max(dmax, d.pr_dmax[r]);
            }
        }
        sbase[b + 1] = S;
        pbase[b + 1] = pbase[b] + d.n_proj;
        if (S - sbase[b] > (int64_t)0x7fffffff)
            return fail(MGC_ERR_INVALID, "block %d has more than 2^31-1 synapses; split it", b);
    }
    if (start[n_blocks] > 0x7fffffff) return fail(MGC_ERR_INVALID, "more than 2^31-1 neurons");
    const int32_t n = (int32_t)start[n_blocks];
    const int64_t S = sbase[n_blocks];
    if (dmin > dmax) dmin = dmax = 1;  // no synapses in the whole network
    PartSpec ps{};
    if (part) {
        ps = *part;
        ps.n_src = n;
        ps.dmin = dmin;
        ps.dmax = dmax;
        if (ps.first < 0 || ps.count <= 0 || (int64_t)ps.first + ps.count > n)
            return fail(MGC_ERR_INVALID, "partition [%d, %lld) outside the network's %d neurons", ps.first,
                        (long long)ps.first + ps.count, n);
        if (dmin < 2)
            return fail(MGC_ERR_INVALID, "partitions exchange spikes every min_delay - 1 steps: min_delay %d < 2",
                        dmin);
        if (d0.mode != MGC_MODE_AUTO && d0.mode != MGC_MODE_DEFERRED)
            return fail(MGC_ERR_INVALID, "a partition runs the deferred method");
    }
    std::vector<int8_t> type(n, (int8_t)MGC_RAW);
    std::vector<uint8_t> tpop(n, 0);
    std::vector<float> rate(n, 0.0f), v0(n, d0.lifconst[1]);
    for (int b = 0; b < n_blocks; ++b) {
        const mgc_fixed_indegree_desc& d = blocks[b];
        const int64_t nb = start[b + 1] - start[b];
        for (int p = 0; p < d.n_pops; ++p)
            for (int32_t i = 0; i < d.pop_num[p]; ++i) {
                type[start[b] + d.pop_start[p] + i] = (int8_t)d.pop_type[p];
                tpop[start[b] + d.pop_start[p] + i] = (uint8_t)std::min(p, kTracePops - 1);
            }
        if (d.rate) memcpy(rate.data() + start[b], d.rate, 4 * nb);
        if (d.v_init) memcpy(v0.data() + start[b], d.v_init, 4 * nb);
    }
    const int32_t first = part ? ps.first : 0, nloc = part ? ps.count : n;
    std::unique_ptr<mgc_sim> s(new mgc_sim);
    s->device = d0.device;
    CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->n = nloc;
    s->S = S;
    s->stdp = false;
    float stdpc[6] = {0.1f, -0.01f, 17.0f, 34.0f, 40.0f, 0.0f};
    CKS(init_common(s.get(), nloc, type.data() + first, rate.data() + first, v0.data() + first, d0.lifconst, stdpc,
                    d0.seed, d0.raster_steps, d0.raster_ids));
    s->tpop_host.assign(tpop.begin() + first, tpop.begin() + first + nloc);
    if (part) apply_part(s.get(), ps);
    StepArgs& a = s->a;
    a.id_offset = d0.id_offset + first;  // POISSON draws keyed by the global id
    s->dmin = dmin;
    s->dmax = dmax;
    s->M = dmax + 1;
    CKS(check_tbits(s.get()));
    CKS(choose_mode(s.get(), d0.mode));
    apply_fx(s.get(), fx_plan_blocks(blocks, n_blocks));
    const int dbits = sort_dbits(s.get());
    CKS(begin_layout(s.get()));
    uint2* syn;
    CKS(s->alloc(&syn, S, false));
    a.syn = syn;
    a.n_syn = S;
    if (S > 0) {
        DevTmp t_pt;
        ProjEntry* dpt;
        CKS(tmp_alloc(t_pt, &dpt, pt.size()));
        CK(cudaMemcpyAsync(dpt, pt.data(), sizeof(ProjEntry) * pt.size(), cudaMemcpyHostToDevice, s->stream));
        int64_t maxS = 0;
        for (int b = 0; b < n_blocks; ++b) maxS = std::max(maxS, sbase[b + 1] - sbase[b]);
        DevTmp t_keys, t_vals, t_keys2, t_order;
        uint32_t *keys, *vals, *keys2, *order;
        CKS(tmp_alloc(t_keys, &keys, maxS));
        CKS(tmp_alloc(t_vals, &vals, maxS));
        CKS(tmp_alloc(t_keys2, &keys2, maxS));
        CKS(tmp_alloc(t_order, &order, maxS));
        for (int b = 0; b < n_blocks; ++b) {
            const int64_t Sb = sbase[b + 1] - sbase[b];
            if (Sb == 0) continue;
            const ProjEntry* bpt = dpt + pbase[b];
            const int npr = (int)(pbase[b + 1] - pbase[b]);
            k_fid_keys<<<grid_for(Sb), 256, 0, s->stream>>>(bpt, npr, sbase[b], Sb, dbits, s->dmin, keys, vals);
            CKS(sort_pairs(keys, keys2, vals, order, Sb, s->sbits + dbits, s->stream));
            k_fid_gather<<<grid_for(Sb), 256, 0, s->stream>>>(bpt, npr, sbase[b], order, Sb, a.tbits, syn + sbase[b]);
            count_keys(s.get(), keys2, Sb);
            CK(cudaGetLastError());
        }
        CK(cudaStreamSynchronize(s->stream));
    }
    CKS(finish_build(s.get()));
    *out = s.release();
    return MGC_OK;
}

}  // namespace

extern "C" {

mgc_status mgc_create_batch(const mgc_fixed_indegree_desc* blocks, int32_t n_blocks, mgc_sim** out)
{
    return create_fixed_indegree(blocks, n_blocks, nullptr, out);
}

mgc_status mgc_create_fixed_indegree(const mgc_fixed_indegree_desc* d, mgc_sim** out)
{
    return create_fixed_indegree(d, 1, nullptr, out);
}

mgc_status mgc_create_fixed_indegree_partition(const mgc_fixed_indegree_desc* d, int32_t first, int32_t count,
                                               mgc_sim** out)
{
    const PartSpec p{0, first, count, 0, 0, false, {}};  // sizes and delays filled in from the description
    return create_fixed_indegree(d, 1, &p, out);
}

}  // extern "C"

extern "C" mgc_status mgc_set_accumulation(mgc_sim* s, int32_t mode)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    if (mode != MGC_ACC_FLOAT && mode != MGC_ACC_FIXED) return fail(MGC_ERR_INVALID, "unknown accumulation %d", mode);
    const int fx = mode == MGC_ACC_FIXED;
    if (fx == s->a.fx) return MGC_OK;
    if (fx && s->a.pull)
        return fail(MGC_ERR_INVALID, "the pull method adds every input in a fixed order (no fixed-point accumulation)");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    int64_t step = 0;
    CK(cudaMemcpy(&step, s->a.step, 8, cudaMemcpyDeviceToHost));
    if (step != 0 || s->graph) return fail(MGC_ERR_INVALID, "the accumulation is chosen before the first step");
    StepArgs& a = s->a;
    float** bufs[2] = {a.deferred ? &a.acc_e : &a.ring_e, a.deferred ? &a.acc_i : &a.ring_i};
    const size_t entries = (a.deferred ? (size_t)s->acc_buffers : (size_t)s->M) * (size_t)a.ns;
    for (float** b : bufs) {
        float* nb = nullptr;
        CKS(s->alloc(&nb, entries * (fx ? 2 : 1)));  // zeroed: nothing has arrived before the first step
        s->release(*b);
        *b = nb;
    }
    a.fx = fx;
    CKS(launch_shapes(s));
    CK(cudaStreamSynchronize(s->stream));
    return MGC_OK;
}
