// C ABI of the simulation core (include/mgc.h): network upload and CSR
// construction on the device, the step driver (CUDA graphs of whole step
// groups), raster and state readout.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/mgc.h"
#include "kernels.cuh"
#include "sched.cuh"

using namespace mgc;

namespace {

thread_local std::string g_last_error;

mgc_status fail(mgc_status st, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

#define CK(expr)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            if (e_ == cudaErrorMemoryAllocation) {                                                \
                cudaGetLastError();                                                               \
                return fail(MGC_ERR_NOMEM, "%s: %s", #expr, cudaGetErrorString(e_));              \
            }                                                                                     \
            return fail(MGC_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                \
        }                                                                                         \
    } while (0)

#define CKS(expr)                    \
    do {                             \
        mgc_status s_ = (expr);      \
        if (s_ != MGC_OK) return s_; \
    } while (0)

// Host-side fault injection (mgc_fault_inject_alloc): when positive, the
// device allocation that brings the count to zero fails as if the device
// were out of memory.
std::atomic<int64_t> g_fail_alloc{0};

cudaError_t dev_malloc(void** p, size_t bytes)
{
    int64_t n = g_fail_alloc.load();
    while (n > 0) {
        if (g_fail_alloc.compare_exchange_weak(n, n - 1)) {
            if (n == 1) return cudaErrorMemoryAllocation;
            break;
        }
    }
    return cudaMalloc(p, bytes);
}

constexpr int64_t kDefaultRasterSteps = 1 << 16;
constexpr int kGraphSteps = 64;
constexpr size_t kMaxBucketBytes = size_t(16) << 30;  // deferred bucket table budget
constexpr int64_t kDefaultChunk = 128;                // synapses per delivery task
constexpr int64_t kMaxChunks = 64;                    // tasks per (spike, delay) segment

int bits_for(int64_t n)
{
    int b = 1;
    while ((int64_t(1) << b) < n) ++b;
    return b;
}

}  // namespace

struct mgc_sim {
    int device = 0;
    cudaStream_t stream = nullptr;
    StepArgs a{};
    int32_t n = 0, M = 0, dmin = 0, dmax = 0;
    int32_t n_src = 0;   // CSR rows: n, or the whole network's neurons (partition)
    int sbits = 1;       // bits of a source id in the sort keys
    bool partition = false;  // simulates neurons [a.src_base, a.src_base + n) of a larger network
    std::vector<int32_t> pois_idx;  // POISSON neurons, and the V they report (their V slot holds
    std::vector<float> pois_v;      // the per-step probability)
    struct RasterStage {     // a device copy of the raster, waiting for the host
        int32_t* ids = nullptr;
        int32_t* counts = nullptr;
        int64_t* meta = nullptr;  // first step, steps, ids, raster status bits
        cudaEvent_t ev = nullptr;
    };
    RasterStage stages[2];
    int stage_head = 0, staged = 0;  // oldest outstanding stage, and how many
    cudaStream_t copy_stream = nullptr;
    int32_t pending = 0;     // partition: steps run since the last spike import
    int32_t* xch = nullptr;  // partition: device scratch of the exchange (spike counts)
    int64_t xch_cap = 0;
    int64_t S = 0;
    int mode = MGC_MODE_PUSH;
    bool stdp = false;
    int neuron_grid = 1, push_grid = 1, stdp_grid = 1, deliver_grid = 1, fused_grid = 1;
    bool fused = false;  // one launch per step (deferred, min delay >= 2)
    bool explicit_net = false;  // built from a synapse list (mgc_create)
    int pull_grid = 1;
    int64_t* in_syn64 = nullptr;  // synapse-list index of each incoming-row position (pull)
    bool ahead = true;   // arrivals of the current device step are already delivered
    std::vector<void*> allocs;
    size_t bytes = 0;
    int64_t* csr_syn64 = nullptr;  // synapse-list index of each CSR position (explicit nets)
    int64_t launches = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    int64_t raster_steps_cap = 0, raster_ids_cap = 0;
    int64_t max_gap = 0;  // longest (source, delay) segment (deferred)
    // fused method: two instantiations of the step kernel (2 or 3 resident
    // blocks per SM); `fused_variant` runs outside the scheduler's graphs
    int fused_variant = 1;
    int fused_grid_v[2] = {1, 1};
    std::vector<uint8_t> tpop_host;   // trace population of each neuron (set by the builders)
    SchedState* sched = nullptr;      // device
    float* sched_data = nullptr;      // device [kMaxDataset][kTraceCols]
    bool sched_graph = false;         // the step-group graph branches on the scheduler's choice
    int persistent = 0;               // fused method as cooperative step groups: 1 barrier per
                                      // step, 2 pipelined (min delay >= 4), 3 windowed
    int group_grid_v[2][2] = {{1, 1}, {1, 1}};  // [persistent-1][variant] co-resident grids
    int window = 1;                   // steps per window of the windowed group (<= min delay, <= 4)
    int window_grid_v[2] = {1, 1};    // its co-resident grids by variant
    size_t window_smem = 0;           // its dynamic shared memory: the window's delivery prefixes
    int group_grid1 = 1;              // minimum delay 1: the step group's grid
    int32_t sched_mode_h = 0;         // host mirrors of what decides the graph's shape
    bool sched_collect_h = false, sched_forced_h = false;

    ~mgc_sim()
    {
        if (device >= 0) cudaSetDevice(device);
        if (graph) cudaGraphExecDestroy(graph);
        if (stream) cudaStreamSynchronize(stream);
        for (RasterStage& g : stages)
            if (g.ev) cudaEventDestroy(g.ev);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        for (void* p : allocs) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }

    template <class T>
    mgc_status alloc(T** p, size_t count, bool zero = true)
    {
        void* v = nullptr;
        size_t b = std::max<size_t>(count, 1) * sizeof(T);
        CK(dev_malloc(&v, b));
        allocs.push_back(v);
        bytes += b;
        if (zero) CK(cudaMemsetAsync(v, 0, b, stream));
        *p = static_cast<T*>(v);
        return MGC_OK;
    }

    template <class T>
    mgc_status upload(T** p, const T* host, size_t count)
    {
        CKS(alloc(p, count, host == nullptr));
        if (host && count) CK(cudaMemcpyAsync(*p, host, count * sizeof(T), cudaMemcpyHostToDevice, stream));
        return MGC_OK;
    }
};

namespace {

// Temporary device buffer freed on scope exit.
struct DevTmp {
    void* p = nullptr;
    ~DevTmp()
    {
        if (p) cudaFree(p);
    }
};

template <class T>
mgc_status tmp_alloc(DevTmp& t, T** p, size_t count)
{
    CK(dev_malloc(&t.p, std::max<size_t>(count, 1) * sizeof(T)));
    *p = static_cast<T*>(t.p);
    return MGC_OK;
}

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

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

// New POISSON probabilities into the neurons' V slots.
__global__ void k_rate_to_v(const int8_t* type, const float* rate, float* V, int32_t n)
{
    GRID_STRIDE(i, n)
    {
        if (type[i] == kPOISSON) V[i] = rate[i];
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

__global__ void k_iota(uint32_t* v, int64_t S)
{
    GRID_STRIDE(p, S) v[p] = (uint32_t)p;
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

int grid_for(int64_t n, int block = 256)
{
    int64_t g = (n + block - 1) / block;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
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

mgc_status pick_device(int device)
{
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(MGC_ERR_NODEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    }
    if (device < 0 || device >= count) return fail(MGC_ERR_INVALID, "device %d out of range", device);
    CK(cudaSetDevice(device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return fail(MGC_ERR_NODEVICE, "device %d is sm_%d%d; this library holds sm_100a code only", device,
                    prop.major, prop.minor);
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
    // pull: explicit networks whose per-step pass over all synapses is
    // cheap; AUTO takes it for plastic networks of up to 2^26 synapses
    const bool pull_ok = s->explicit_net && s->S < (int64_t(1) << 32) && a.tbits + dbits <= 32;
    if (requested == MGC_MODE_PULL && !pull_ok)
        return fail(MGC_ERR_INVALID, "the pull method needs an explicit synapse list of < 2^32 synapses");
    if (requested == MGC_MODE_PULL ||
        (requested == MGC_MODE_AUTO && s->stdp && pull_ok && s->S <= (int64_t(1) << 26))) {
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
        a.H = s->dmax + 4;  // + 3: the windowed step group clears the next window's slots
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

// The fused step kernel for this network (with or without LIF/LIFE
// currents), variant 0 compiled for 2 resident blocks per SM, 1 for 3.
using StepKernel = void (*)(StepArgs);
StepKernel fused_kernel(const mgc_sim* s, int v)
{
    if (s->a.has_cur) return v == 0 ? k_fused<true, 2> : k_fused<true, 3>;
    return v == 0 ? k_fused<false, 2> : k_fused<false, 3>;
}

// The step-group kernels of the same variant: p = 1 one barrier per step,
// p = 2 pipelined.
using GroupKernel = void (*)(StepArgs, int32_t);
GroupKernel steps_kernel(const mgc_sim* s, int p, int v)
{
    if (!s->fused) return s->a.has_cur ? k_steps1<true> : k_steps1<false>;  // minimum delay 1
    if (p == 2) {
        if (s->a.has_cur) return v == 0 ? k_pipe<true, 2> : k_pipe<true, 3>;
        return v == 0 ? k_pipe<false, 2> : k_pipe<false, 3>;
    }
    if (s->a.has_cur) return v == 0 ? k_steps<true, 2> : k_steps<true, 3>;
    return v == 0 ? k_steps<false, 2> : k_steps<false, 3>;
}

// The windowed step group of variant v (templates over the update's
// current arrays and the register budget, as the other step groups).
using WindowKernel = void (*)(StepArgs, int32_t, int32_t);
WindowKernel window_kernel(const mgc_sim* s, int v)
{
    if (s->a.has_cur) return v == 0 ? k_window<true, 2> : k_window<true, 3>;
    return v == 0 ? k_window<false, 2> : k_window<false, 3>;
}

// The step-group mode the scheduler's graph runs for mode p: the windowed
// group keeps no schedule trace, so the graph takes the pipelined group (or
// the barrier per step, for a minimum delay below 4) in its place.
int graph_group_mode(const mgc_sim* s, int p) { return p == 3 ? (s->dmin >= 4 ? 2 : 1) : p; }

constexpr int32_t kPersistentSteps = 1024;  // steps per cooperative launch

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

// Stream-ordered write of one field of the device scheduler state.
template <class T>
mgc_status sched_put(mgc_sim* s, T SchedState::*field, T value)
{
    static SchedState layout;  // host object, for the field's offset only
    const size_t off = (size_t)(reinterpret_cast<const char*>(&(layout.*field)) - reinterpret_cast<const char*>(&layout));
    T staged = value;
    CK(cudaMemcpyAsync(reinterpret_cast<char*>(s->sched) + off, &staged, sizeof(T), cudaMemcpyHostToDevice, s->stream));
    return cudaStreamSynchronize(s->stream) == cudaSuccess ? MGC_OK : fail(MGC_ERR_CUDA, "scheduler write failed");
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
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, s->device));
    int occ = 0;
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
        CKS(s->alloc(&a.acc_e, kAccBuffers * (size_t)a.ns));  // step buffers, s % kAccBuffers
        CKS(s->alloc(&a.acc_i, kAccBuffers * (size_t)a.ns));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_deliver, kPushBlock, 0));
        s->deliver_grid = prop.multiProcessorCount * std::max(1, occ);
        // fused step kernel: one resident wave, every warp updates then delivers
        s->fused = s->dmin >= 2;
        for (int v = 0; v < 2; ++v) {
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fused_kernel(s, v), kPushBlock, 0));
            s->fused_grid_v[v] = prop.multiProcessorCount * std::min(std::max(1, occ), v == 0 ? 2 : 3);
        }
        s->fused_variant = 1;
        s->fused_grid = s->fused_grid_v[1];
        // step groups by default (faster than one launch per step on every
        // measured load); the pipelined form needs a minimum delay >= 4.
        // The windowed form is faster on the measured loads, but it changes
        // the order of the fp32 additions into one neuron's input (with
        // unequal weights per sign the last bits of V differ from the
        // reference's), so only the autotuner or the caller selects it
        s->persistent = s->fused ? (s->dmin >= 4 ? 2 : 1) : 1;
        if (!s->fused) {
            // minimum delay 1: a barrier-per-phase step group sized to the
            // neurons (8 warps x 64 neuron groups a block per pass)
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, steps_kernel(s, 1, 0), kPushBlock, 0));
            const int64_t wave = (int64_t)prop.multiProcessorCount * std::max(1, occ);
            const int64_t want = ((int64_t)a.ns / 4 + 511) / 512;
            s->group_grid1 = (int)std::max<int64_t>(1, std::min(wave, want));
            CKS(s->alloc(&a.bar, 4));  // the grid barrier's arrivals and generation
        }
        if (s->fused) {
            for (int p = 1; p <= 2; ++p)
                for (int v = 0; v < 2; ++v) {
                    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, steps_kernel(s, p, v), kPushBlock, 0));
                    s->group_grid_v[p - 1][v] = prop.multiProcessorCount * std::min(std::max(1, occ), v == 0 ? 2 : 3);
                }
            // windowed group: prefixes of up to kMaxWindow steps in dynamic shared memory
            s->window = std::min(kMaxWindow, s->dmin);
            s->window_smem = (size_t)kMaxWindow * (size_t)(a.D + 1) * sizeof(int64_t);
            for (int v = 0; v < 2; ++v) {
                CK(cudaFuncSetAttribute((const void*)window_kernel(s, v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)s->window_smem));
                CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, window_kernel(s, v), kPushBlock,
                                                                 s->window_smem));
                s->window_grid_v[v] = prop.multiProcessorCount * std::min(std::max(1, occ), v == 0 ? 2 : 3);
            }
            CKS(init_sched(s));
        }
    } else {
        a.M = s->M;
        CKS(s->alloc(&a.ring_e, (size_t)s->M * a.ns));
        CKS(s->alloc(&a.ring_i, (size_t)s->M * a.ns));
        CKS(s->alloc(&a.spk, s->n));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_push, kPushBlock, 0));
        s->push_grid = prop.multiProcessorCount * std::max(1, occ);
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stdp, kPushBlock, 0));
        s->stdp_grid = prop.multiProcessorCount * std::max(1, occ);
        if (a.pull) {
            const int64_t groups = a.ns / 4;
            CKS(s->alloc(&a.fired_bits, (size_t)((groups + 31) / 32) * 4));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pull, kPushBlock, 0));
            s->pull_grid = prop.multiProcessorCount * std::max(1, occ);
        }
    }
    a.M = s->M;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_neuron, kNeuronBlock, 0));
    s->neuron_grid = (int)std::max<int64_t>(
        1, std::min<int64_t>((int64_t)prop.multiProcessorCount * std::max(1, occ),
                             (a.ns / 4 + kNeuronBlock - 1) / kNeuronBlock));
    CK(cudaStreamSynchronize(s->stream));
    return MGC_OK;
}

int kernels_per_step(const mgc_sim* s)
{
    if (s->a.deferred) return s->fused ? 1 : 2;
    if (s->a.pull) return 2;
    return s->stdp ? 3 : 2;
}

mgc_status enqueue_step(mgc_sim* s)
{
    if (s->a.deferred) {
        if (s->fused) {
            if (!s->ahead) {  // arrivals of this step not yet delivered
                k_deliver<<<s->deliver_grid, kPushBlock, 0, s->stream>>>(s->a);
                s->launches += 1;
            }
            fused_kernel(s, s->fused_variant)<<<s->fused_grid, kPushBlock, 0, s->stream>>>(s->a);
            s->ahead = true;
            s->launches += 1;
        } else {
            k_deliver<<<s->deliver_grid, kPushBlock, 0, s->stream>>>(s->a);
            k_neuron<<<s->neuron_grid, kNeuronBlock, 0, s->stream>>>(s->a);
            s->launches += 2;
        }
    } else {
        k_neuron<<<s->neuron_grid, kNeuronBlock, 0, s->stream>>>(s->a);
        if (s->a.pull) {
            k_pull<<<s->pull_grid, kPushBlock, 0, s->stream>>>(s->a);
        } else {
            k_push<<<s->push_grid, kPushBlock, 0, s->stream>>>(s->a);
            if (s->stdp) k_stdp<<<s->stdp_grid, kPushBlock, 0, s->stream>>>(s->a);
        }
        s->launches += kernels_per_step(s);
    }
    CK(cudaGetLastError());
    return MGC_OK;
}

mgc_status build_graph(mgc_sim* s)
{
    // every captured step must start in the same delivery state: for the
    // fused method that is "arrivals already delivered", which the step
    // before the graph establishes (mgc_run brings it about first)
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    const int64_t before = s->launches;
    for (int i = 0; i < kGraphSteps; ++i) {
        mgc_status st = enqueue_step(s);
        if (st != MGC_OK) {
            cudaStreamEndCapture(s->stream, &g);
            if (g) cudaGraphDestroy(g);
            return st;
        }
    }
    s->launches = before;  // captured, not launched
    CK(cudaStreamEndCapture(s->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&s->graph, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    s->graph_steps = kGraphSteps;
    return MGC_OK;
}

// Step-group graph of the fused method: the scheduler's decision kernel,
// then a conditional SWITCH node whose body v runs kGraphSteps steps of
// variant v; the decision kernel sets the branch on the device, so the host
// never waits for it.
mgc_status build_sched_graph(mgc_sim* s)
{
    struct GraphGuard {
        cudaGraph_t g = nullptr;
        ~GraphGuard()
        {
            if (g) cudaGraphDestroy(g);
        }
    } guard;
    CK(cudaGraphCreate(&guard.g, 0));
    cudaGraphConditionalHandle handle;
    CK(cudaGraphConditionalHandleCreate(&handle, guard.g, (unsigned)s->fused_variant, cudaGraphCondAssignDefault));
    int32_t set_handle = 1;
    void* dargs[] = {&s->a, &s->sched, &s->sched_data, &handle, &set_handle};
    cudaKernelNodeParams kp = {};
    kp.func = (void*)k_sched_decide;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = dargs;
    cudaGraphNode_t decide;
    CK(cudaGraphAddKernelNode(&decide, guard.g, nullptr, 0, &kp));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeSwitch;
    cp.conditional.size = 2;
    cudaGraphNode_t cond;
    CK(cudaGraphAddNode(&cond, guard.g, &decide, 1, &cp));
    void* sargs[] = {&s->a};
    int32_t group_steps = kGraphSteps;
    void* gargs[] = {&s->a, &group_steps};
    for (int v = 0; v < 2; ++v) {
        cudaGraph_t body = cp.conditional.phGraph_out[v];
        cudaGraphNode_t prev = nullptr;
        if (s->persistent) {
            // the group as one cooperative step-group kernel of variant v,
            // after a node that clears its barrier counters
            const int p = graph_group_mode(s, s->persistent);
            cudaMemsetParams mp = {};
            mp.dst = s->a.bar;
            mp.value = 0;
            mp.elementSize = 4;
            mp.width = 4;
            mp.height = 1;
            mp.pitch = 0;
            cudaGraphNode_t clear, node;
            CK(cudaGraphAddMemsetNode(&clear, body, nullptr, 0, &mp));
            cudaKernelNodeParams gp = {};
            gp.func = (void*)steps_kernel(s, p, v);
            gp.gridDim = dim3(s->group_grid_v[p - 1][v]);
            gp.blockDim = dim3(kPushBlock);
            gp.kernelParams = gargs;
            CK(cudaGraphAddKernelNode(&node, body, &clear, 1, &gp));
            cudaLaunchAttributeValue coop = {};
            coop.cooperative = 1;
            CK(cudaGraphKernelNodeSetAttribute(node, cudaLaunchAttributeCooperative, &coop));
            continue;
        }
        for (int i = 0; i < kGraphSteps; ++i) {
            cudaKernelNodeParams sp = {};
            sp.func = (void*)fused_kernel(s, v);
            sp.gridDim = dim3(s->fused_grid_v[v]);
            sp.blockDim = dim3(kPushBlock);
            sp.kernelParams = sargs;
            cudaGraphNode_t node;
            CK(cudaGraphAddKernelNode(&node, body, prev ? &prev : nullptr, prev ? 1 : 0, &sp));
            prev = node;
        }
    }
    CK(cudaGraphInstantiate(&s->graph, guard.g, 0));
    s->graph_steps = kGraphSteps;
    s->sched_graph = true;
    return MGC_OK;
}

// The decision kernel and the SWITCH node are in the step-group graph only
// while something needs them (an adaptive mode, recording, calibration);
// otherwise the graph is the plain chain of the static variant's kernels.
bool sched_wanted(const mgc_sim* s)
{
    return s->sched && (s->sched_mode_h != kSchedStatic || s->sched_collect_h || s->sched_forced_h);
}

mgc_status refresh_graph(mgc_sim* s)
{
    if (s->graph && s->sched_graph != sched_wanted(s)) {
        CK(cudaStreamSynchronize(s->stream));
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
        s->sched_graph = false;
    }
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
};

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
    PartSpec p{d->n_neurons, first, count, 0x7fffffff, 0};
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
    const int dbits = sort_dbits(s.get());
    CKS(begin_layout(s.get()));
    uint2* syn;
    CKS(s->alloc(&syn, S, false));
    a.syn = syn;
    a.n_syn = S;
    CKS(s->alloc(&s->csr_syn64, S, false));
    DevTmp t_keys2;
    uint32_t* keys2 = nullptr;
    if (S > 0) {
        DevTmp t_src, t_tar, t_w, t_d, t_pl, t_keys, t_vals, t_order, t_bad;
        int32_t *src, *tar, *dl, *bad;
        float* w;
        uint8_t* pl = nullptr;
        uint32_t *keys, *vals, *order;
        CKS(tmp_alloc(t_src, &src, S));
        CKS(tmp_alloc(t_tar, &tar, S));
        CKS(tmp_alloc(t_w, &w, S));
        CKS(tmp_alloc(t_d, &dl, S));
        CKS(tmp_alloc(t_bad, &bad, 1));
        CK(cudaMemcpyAsync(src, d->syn_src, 4 * S, cudaMemcpyHostToDevice, s->stream));
        CK(cudaMemcpyAsync(tar, d->syn_tar, 4 * S, cudaMemcpyHostToDevice, s->stream));
        CK(cudaMemcpyAsync(w, d->syn_weight, 4 * S, cudaMemcpyHostToDevice, s->stream));
        CK(cudaMemcpyAsync(dl, d->syn_delay, 4 * S, cudaMemcpyHostToDevice, s->stream));
        if (s->stdp && d->syn_plastic) {
            CKS(tmp_alloc(t_pl, &pl, S));
            CK(cudaMemcpyAsync(pl, d->syn_plastic, S, cudaMemcpyHostToDevice, s->stream));
        }
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
            if (s->stdp && d->syn_plastic) CKS(s->alloc(&in_pl, S, false));
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
            if (d->syn_plastic) CKS(s->alloc(&plastic, S, false));
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
        }
        count_keys(s.get(), keys2, S);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s->stream));
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
    const PartSpec p{0, first, count, 0, 0};  // sizes and delays filled in from the description
    return create_fixed_indegree(d, 1, &p, out);
}

mgc_status mgc_run(mgc_sim* s, int64_t steps)
{
    if (!s || steps < 0) return fail(MGC_ERR_INVALID, "bad run arguments");
    if (s->partition) {
        // a delivery of step x reads spikes of steps <= x - min_delay, so at
        // most min_delay - 1 steps may run between two imports
        if (s->pending + steps > s->dmin - 1)
            return fail(MGC_ERR_INVALID, "partition: %lld steps since the last exchange, at most %d (min_delay - 1)",
                        (long long)(s->pending + steps), s->dmin - 1);
        s->pending += (int32_t)steps;
    }
    CK(cudaSetDevice(s->device));
    int64_t left = steps;
    if (s->a.deferred && s->fused && !s->ahead && left > 0) {
        CKS(enqueue_step(s));  // catches up the delivery, leaves ahead = true
        --left;
    }
    if (s->persistent && s->a.deferred && !sched_wanted(s)) {
        // one cooperative launch per group: every block resident, a grid
        // barrier between steps (or the pipelined arrive/wait) instead of a launch
        const int p = s->persistent, v = s->fused_variant;
        while (left > 0) {
            int32_t n = (int32_t)std::min<int64_t>(left, kPersistentSteps);
            // the schedule trace only while the scheduler's graph runs
            StepArgs ga = s->a;
            ga.trace = nullptr;
            void* args[] = {&ga, &n};
            CK(cudaMemsetAsync(s->a.bar, 0, 4 * sizeof(unsigned int), s->stream));  // clean barriers
            cudaError_t e;
            if (p == 3) {
                int32_t w = s->window;
                void* wargs[] = {&ga, &n, &w};
                e = cudaLaunchCooperativeKernel((const void*)window_kernel(s, v), dim3(s->window_grid_v[v]),
                                                dim3(kPushBlock), wargs, s->window_smem, s->stream);
            } else {
                const int grid = s->fused ? s->group_grid_v[p - 1][v] : s->group_grid1;
                e = cudaLaunchCooperativeKernel((const void*)steps_kernel(s, p, v), dim3(grid), dim3(kPushBlock),
                                                args, 0, s->stream);
            }
            if (e == cudaErrorCooperativeLaunchTooLarge || e == cudaErrorNotSupported) {
                // the blocks cannot all be resident here (e.g. a shared
                // device): fall back to the graphs of single-step kernels
                cudaGetLastError();
                s->persistent = 0;
                break;
            }
            CK(e);
            s->launches += 1;
            left -= n;
        }
        if (left == 0) return MGC_OK;
    }
    if (left >= kGraphSteps) {
        if (!s->graph) CKS(sched_wanted(s) ? build_sched_graph(s) : build_graph(s));
        while (left >= s->graph_steps) {
            CK(cudaGraphLaunch(s->graph, s->stream));
            s->launches += s->sched_graph && s->persistent ? 2  // the decision kernel and the step group
                                                           : (int64_t)s->graph_steps * kernels_per_step(s) +
                                                                 (s->sched_graph ? 1 : 0);
            left -= s->graph_steps;
        }
    }
    for (; left > 0; --left) CKS(enqueue_step(s));
    return MGC_OK;
}

mgc_status mgc_sync(mgc_sim* s)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    int32_t st = 0;
    CK(cudaMemcpy(&st, s->a.status, 4, cudaMemcpyDeviceToHost));
    if (st & kStatusBarrier) return fail(MGC_ERR_CUDA, "a grid barrier of the persistent step group timed out");
    if (st & kStatusBounds)
        return fail(MGC_ERR_CUDA, "an index check of the checked build failed (an index outside its array)");
    if (st & kStatusExchange)
        return fail(MGC_ERR_INVALID, "a spike exchange was refused: an id outside the network, or a window with more "
                                     "spikes than the exchange buffer holds");
    if (st) return fail(MGC_ERR_OVERFLOW, "raster buffer overflow (status %d)", st);
    return MGC_OK;
}

mgc_status mgc_set_rates(mgc_sim* s, const float* rate, int32_t n)
{
    if (!s || !rate || n != s->n) return fail(MGC_ERR_INVALID, "rate array must hold n_neurons entries");
    CK(cudaSetDevice(s->device));
    CK(cudaMemcpyAsync(const_cast<float*>(s->a.rate), rate, sizeof(float) * n, cudaMemcpyHostToDevice, s->stream));
    k_rate_to_v<<<grid_for(n), 256, 0, s->stream>>>(s->a.type, s->a.rate, s->a.V, n);
    CK(cudaGetLastError());
    s->launches += 1;
    return MGC_OK;
}

}  // extern "C"

namespace {

constexpr int32_t kRasterBits = kStatusRasterIds | kStatusRasterSteps;

// ns steps' counts c32 and their ni ids hid (step after step) into the
// caller's arrays, each step's ids sorted, the steps split over host threads.
mgc_status finish_raster(int64_t step0, int64_t ns, int64_t ni, const int32_t* c32, int32_t* hid, bool truncated,
                         int32_t status, int64_t* first_step, int64_t* counts, int64_t counts_cap, int32_t* ids,
                         int64_t ids_cap, int64_t* n_steps, int64_t* n_ids)
{
    truncated = truncated || ns > counts_cap || ni > ids_cap;
    std::vector<int64_t> off(ns + 1, 0);
    for (int64_t i = 0; i < ns; ++i) {
        off[i + 1] = off[i] + c32[i];
        if (counts && i < counts_cap) counts[i] = c32[i];
    }
    auto sort_steps = [&](int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; ++i)
            if (off[i + 1] <= ni) std::sort(hid + off[i], hid + off[i + 1]);
    };
    const int64_t nt = std::min<int64_t>(std::max(1u, std::thread::hardware_concurrency()), 16);
    if (ni > (1 << 16) && ns > 1 && nt > 1) {
        std::vector<std::thread> pool;
        for (int64_t t = 0; t < nt; ++t) pool.emplace_back(sort_steps, ns * t / nt, ns * (t + 1) / nt);
        for (auto& th : pool) th.join();
    } else {
        sort_steps(0, ns);
    }
    if (ids && hid != ids) memcpy(ids, hid, 4 * std::min(ni, ids_cap));
    if (first_step) *first_step = step0;
    if (n_steps) *n_steps = std::min(ns, counts_cap);
    if (n_ids) *n_ids = std::min(ni, ids_cap);
    if (truncated) return fail(MGC_ERR_OVERFLOW, "raster truncated (device status %d)", status);
    return MGC_OK;
}

// The raster so far into a stage (block-strided copies), then the clock of
// the next raster (k_raster_restart, after every block has read).
__global__ void k_raster_stage(StepArgs a, int32_t* ids, int32_t* counts, int64_t steps_cap, int64_t ids_cap)
{
    const int64_t ns = min(*a.step - *a.raster_step0, steps_cap);
    const int64_t ni = min(*a.raster_pos, ids_cap);
    GRID_STRIDE(i, ns) counts[i] = a.raster_counts[i];
    GRID_STRIDE(i, ni) ids[i] = a.raster_ids[i];
}

__global__ void k_raster_restart(StepArgs a, int64_t* meta, int64_t steps_cap, int64_t ids_cap)
{
    const int64_t step = *a.step, step0 = *a.raster_step0;
    meta[0] = step0;
    meta[1] = min(step - step0, steps_cap);
    meta[2] = min(*a.raster_pos, ids_cap);
    meta[3] = *a.status & kRasterBits;
    *a.raster_step0 = step;
    *a.raster_pos = 0;
    atomicAnd(a.status, ~kRasterBits);
}

}  // namespace

extern "C" {

mgc_status mgc_read_raster(mgc_sim* s, int64_t* first_step, int64_t* counts, int64_t counts_cap, int32_t* ids,
                           int64_t ids_cap, int64_t* n_steps, int64_t* n_ids)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    if (!s->a.record) return fail(MGC_ERR_INVALID, "raster recording is off for this handle");
    if (s->staged) return fail(MGC_ERR_INVALID, "collect the staged rasters first (mgc_raster_collect)");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    int64_t step = 0, step0 = 0, pos = 0;
    int32_t status = 0;
    CK(cudaMemcpy(&step, s->a.step, 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&step0, s->a.raster_step0, 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&pos, s->a.raster_pos, 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&status, s->a.status, 4, cudaMemcpyDeviceToHost));
    const int64_t ns = std::min(step - step0, s->raster_steps_cap);
    const int64_t ni = std::min(pos, s->raster_ids_cap);
    std::vector<int32_t> c32(ns);
    if (ns) CK(cudaMemcpy(c32.data(), s->a.raster_counts, 4 * ns, cudaMemcpyDeviceToHost));
    // the ids land in the caller's buffer when it holds them all (else in a
    // staging buffer)
    std::unique_ptr<int32_t[]> staging;
    int32_t* hid = ids;
    if (!ids || ids_cap < ni) {
        staging.reset(new int32_t[std::max<int64_t>(ni, 1)]);
        hid = staging.get();
    }
    if (ni) CK(cudaMemcpy(hid, s->a.raster_ids, 4 * ni, cudaMemcpyDeviceToHost));
    // the next raster starts here; only the raster's status bits are cleared
    const int64_t zero = 0;
    const int32_t kept = status & ~kRasterBits;
    CK(cudaMemcpy(s->a.raster_step0, &step, 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->a.raster_pos, &zero, 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->a.status, &kept, 4, cudaMemcpyHostToDevice));
    return finish_raster(step0, ns, ni, c32.data(), hid, (status & kRasterBits) != 0, status, first_step, counts,
                         counts_cap, ids, ids_cap, n_steps, n_ids);
}

mgc_status mgc_raster_stage(mgc_sim* s)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    if (!s->a.record) return fail(MGC_ERR_INVALID, "raster recording is off for this handle");
    if (s->staged == 2) return fail(MGC_ERR_INVALID, "two rasters are staged already: collect one first");
    CK(cudaSetDevice(s->device));
    mgc_sim::RasterStage& g = s->stages[(s->stage_head + s->staged) & 1];
    if (!g.ids) {
        CKS(s->alloc(&g.ids, (size_t)s->raster_ids_cap, false));
        CKS(s->alloc(&g.counts, (size_t)s->raster_steps_cap, false));
        CKS(s->alloc(&g.meta, 4));
        CK(cudaEventCreateWithFlags(&g.ev, cudaEventDisableTiming));
    }
    if (!s->copy_stream) CK(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
    k_raster_stage<<<grid_for(s->raster_ids_cap), 256, 0, s->stream>>>(s->a, g.ids, g.counts, s->raster_steps_cap,
                                                                        s->raster_ids_cap);
    k_raster_restart<<<1, 1, 0, s->stream>>>(s->a, g.meta, s->raster_steps_cap, s->raster_ids_cap);
    CK(cudaGetLastError());
    CK(cudaEventRecord(g.ev, s->stream));
    s->launches += 2;
    s->staged += 1;
    return MGC_OK;
}

mgc_status mgc_raster_collect(mgc_sim* s, int64_t* first_step, int64_t* counts, int64_t counts_cap, int32_t* ids,
                              int64_t ids_cap, int64_t* n_steps, int64_t* n_ids)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    if (!s->staged) return fail(MGC_ERR_INVALID, "no raster is staged (mgc_raster_stage)");
    CK(cudaSetDevice(s->device));
    mgc_sim::RasterStage& g = s->stages[s->stage_head];
    // the stage's copies are done; the steps enqueued after it keep running
    CK(cudaStreamWaitEvent(s->copy_stream, g.ev, 0));
    int64_t meta[4];
    CK(cudaMemcpyAsync(meta, g.meta, sizeof(meta), cudaMemcpyDeviceToHost, s->copy_stream));
    CK(cudaStreamSynchronize(s->copy_stream));
    const int64_t step0 = meta[0], ns = meta[1], ni = meta[2];
    const int32_t status = (int32_t)meta[3];
    std::vector<int32_t> c32(ns);
    std::unique_ptr<int32_t[]> staging;
    int32_t* hid = ids;
    if (!ids || ids_cap < ni) {
        staging.reset(new int32_t[std::max<int64_t>(ni, 1)]);
        hid = staging.get();
    }
    if (ns) CK(cudaMemcpyAsync(c32.data(), g.counts, 4 * ns, cudaMemcpyDeviceToHost, s->copy_stream));
    if (ni) CK(cudaMemcpyAsync(hid, g.ids, 4 * ni, cudaMemcpyDeviceToHost, s->copy_stream));
    CK(cudaStreamSynchronize(s->copy_stream));
    s->stage_head ^= 1;
    s->staged -= 1;
    return finish_raster(step0, ns, ni, c32.data(), hid, status != 0, status, first_step, counts, counts_cap, ids,
                         ids_cap, n_steps, n_ids);
}

mgc_status mgc_read_state(mgc_sim* s, float* v, float* i_exc, float* i_inh, int32_t* refrac, int32_t* last_fired,
                          int32_t* fire_cnt)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    const size_t n = s->n;
    if (v) {
        CK(cudaMemcpy(v, s->a.V, 4 * n, cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < s->pois_idx.size(); ++k) v[s->pois_idx[k]] = s->pois_v[k];
    }
    if (i_exc) CK(cudaMemcpy(i_exc, s->a.Iexc, 4 * n, cudaMemcpyDeviceToHost));
    if (i_inh) CK(cudaMemcpy(i_inh, s->a.Iinh, 4 * n, cudaMemcpyDeviceToHost));
    if (refrac) CK(cudaMemcpy(refrac, s->a.refrac, 4 * n, cudaMemcpyDeviceToHost));
    if (last_fired) CK(cudaMemcpy(last_fired, s->a.last_fired, 4 * n, cudaMemcpyDeviceToHost));
    if (fire_cnt) CK(cudaMemcpy(fire_cnt, s->a.fire_cnt, 4 * n, cudaMemcpyDeviceToHost));
    return MGC_OK;
}

mgc_status mgc_read_weights(mgc_sim* s, float* weight)
{
    if (!s || !weight) return fail(MGC_ERR_INVALID, "null argument");
    if (!s->csr_syn64) return fail(MGC_ERR_INVALID, "procedural networks have no synapse-list order");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    std::vector<uint2> syn(s->S);
    std::vector<int64_t> idx(s->S);
    // the pull method keeps the live weights in its incoming rows
    const uint2* src_words = s->a.pull ? s->a.in_ent : s->a.syn;
    const int64_t* src_idx = s->a.pull ? s->in_syn64 : s->csr_syn64;
    if (s->S) {
        CK(cudaMemcpy(syn.data(), src_words, 8 * s->S, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(idx.data(), src_idx, 8 * s->S, cudaMemcpyDeviceToHost));
    }
    for (int64_t p = 0; p < s->S; ++p) memcpy(&weight[idx[p]], &syn[p].y, 4);
    return MGC_OK;
}

mgc_status mgc_export_csr(mgc_sim* s, int64_t* row_ptr, int32_t* tgt, float* weight, int32_t* delay)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    if (row_ptr) CK(cudaMemcpy(row_ptr, s->a.row_ptr, 8 * ((size_t)s->n_src + 1), cudaMemcpyDeviceToHost));
    if (tgt || weight || delay) {
        // in pieces, so a large CSR needs no second full-size host copy
        const int64_t piece = int64_t(1) << 24;
        std::vector<uint2> buf((size_t)std::min<int64_t>(piece, std::max<int64_t>(s->S, 1)));
        for (int64_t p0 = 0; p0 < s->S; p0 += piece) {
            const int64_t c = std::min(piece, s->S - p0);
            CK(cudaMemcpy(buf.data(), s->a.syn + p0, 8 * c, cudaMemcpyDeviceToHost));
            for (int64_t q = 0; q < c; ++q) {
                if (tgt) tgt[p0 + q] = (int32_t)(buf[q].x & s->a.tmask);
                if (delay) delay[p0 + q] = (int32_t)(buf[q].x >> s->a.tbits);
                if (weight) memcpy(&weight[p0 + q], &buf[q].y, 4);
            }
        }
    }
    return MGC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Partition statistics on the device: one warp per source row of the CSR,
// the zones' counters in shared memory, flushed once per block.
// ---------------------------------------------------------------------------
namespace {

constexpr int kMaxZones = 4096;

__global__ void k_partition_stats(const int64_t* row_ptr, const uint2* syn, int32_t n_src, uint32_t tmask,
                                  int32_t tar_base, const int32_t* part, int32_t nparts, unsigned long long* out)
{
    extern __shared__ unsigned int zc[];  // [3][nparts]: syn by source zone, out by source zone, in by target zone
    for (int z = threadIdx.x; z < 3 * nparts; z += blockDim.x) zc[z] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t src = warp; src < n_src; src += nwarps) {
        const int64_t b = row_ptr[src], e = row_ptr[src + 1];
        if (e == b) continue;
        const int32_t zs = part[src];
        unsigned int crossing = 0;
        for (int64_t q = b + lane; q < e; q += 32) {
            const int32_t zt = part[(int32_t)(syn[q].x & tmask) + tar_base];
            if (zt != zs) {
                ++crossing;
                atomicAdd(&zc[2 * nparts + zt], 1u);
            }
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) crossing += __shfl_xor_sync(0xffffffffu, crossing, o);
        if (lane == 0) {
            atomicAdd(&zc[zs], (unsigned int)(e - b));
            atomicAdd(&zc[nparts + zs], crossing);
        }
    }
    __syncthreads();
    for (int z = threadIdx.x; z < 3 * nparts; z += blockDim.x)
        if (zc[z]) atomicAdd(out + z, (unsigned long long)zc[z]);
}

}  // namespace

extern "C" {

mgc_status mgc_partition_stats(mgc_sim* s, const int32_t* part, int32_t nparts, int64_t* cut, int64_t* zone_neurons,
                               int64_t* zone_syn, int64_t* zone_out, int64_t* zone_in)
{
    if (!s || !part) return fail(MGC_ERR_INVALID, "null argument");
    if (nparts < 1 || nparts > kMaxZones) return fail(MGC_ERR_INVALID, "1..%d zones (got %d)", kMaxZones, nparts);
    const int32_t n = s->n_src;
    std::vector<int64_t> zn(nparts, 0);
    for (int32_t i = 0; i < n; ++i) {
        if (part[i] < 0 || part[i] >= nparts)
            return fail(MGC_ERR_INVALID, "neuron %d in zone %d, outside 0..%d", i, part[i], nparts - 1);
        zn[part[i]] += 1;
    }
    CK(cudaSetDevice(s->device));
    DevTmp tp, to;
    int32_t* dpart;
    unsigned long long* dout;
    CKS(tmp_alloc(tp, &dpart, (size_t)n));
    CKS(tmp_alloc(to, &dout, 3 * (size_t)nparts));
    CK(cudaMemcpyAsync(dpart, part, 4 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemsetAsync(dout, 0, 8 * 3 * (size_t)nparts, s->stream));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, s->device));
    const size_t smem = 4 * 3 * (size_t)nparts;
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(k_partition_stats, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // a partition handle's targets are local ids; their zones are those of
    // the whole-network ids from its first neuron on
    k_partition_stats<<<prop.multiProcessorCount * 4, 256, smem, s->stream>>>(s->a.row_ptr, s->a.syn, n, s->a.tmask,
                                                                              s->a.src_base, dpart, nparts, dout);
    CK(cudaGetLastError());
    s->launches += 1;
    std::vector<unsigned long long> h(3 * (size_t)nparts);
    CK(cudaMemcpyAsync(h.data(), dout, 8 * h.size(), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    int64_t total_cut = 0;
    for (int32_t z = 0; z < nparts; ++z) {
        if (zone_neurons) zone_neurons[z] = zn[z];
        if (zone_syn) zone_syn[z] = (int64_t)h[z];
        if (zone_out) zone_out[z] = (int64_t)h[nparts + z];
        if (zone_in) zone_in[z] = (int64_t)h[2 * nparts + z];
        total_cut += (int64_t)h[nparts + z];
    }
    if (cut) *cut = total_cut;
    return MGC_OK;
}

mgc_status mgc_get_info(mgc_sim* s, mgc_info* info)
{
    if (!s || !info) return fail(MGC_ERR_INVALID, "null argument");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    memset(info, 0, sizeof(*info));
    info->n_neurons = s->n;
    info->ring_len = s->M;
    info->min_delay = s->dmin;
    info->max_delay = s->dmax;
    info->n_synapses = s->S;
    CK(cudaMemcpy(&info->step, s->a.step, 8, cudaMemcpyDeviceToHost));
    unsigned long long ev = 0;
    CK(cudaMemcpy(&ev, s->a.events, 8, cudaMemcpyDeviceToHost));
    info->events = (int64_t)ev;
    info->mode = s->mode;
    info->graph_steps = s->graph_steps ? s->graph_steps : kGraphSteps;
    info->device_bytes = (int64_t)s->bytes;
    info->persistent = s->a.deferred && !sched_wanted(s) ? s->persistent : 0;
    info->first_neuron = s->a.src_base;
    info->total_neurons = s->n_src;
    info->window = s->fused ? s->window : 0;
    return MGC_OK;
}

mgc_status mgc_profile_steps(mgc_sim* s, int64_t steps, float* ms)
{
    if (!s || !ms || steps < 0) return fail(MGC_ERR_INVALID, "bad profile arguments");
    if (s->partition) return fail(MGC_ERR_INVALID, "partition handles run steps only between exchanges (mgc_run)");
    CK(cudaSetDevice(s->device));
    constexpr int kBatch = 64;
    std::vector<cudaEvent_t> ev(4 * kBatch);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    double acc[3] = {0, 0, 0};
    // External records become event-record nodes of the captured graph (a
    // plain record inside a capture only orders the capture's streams).
    auto rec = [&](cudaEvent_t ev_) { cudaEventRecordWithFlags(ev_, s->stream, cudaEventRecordExternal); };
    mgc_status st = MGC_OK;
    if (s->a.deferred && s->fused && !s->ahead) {
        k_deliver<<<s->deliver_grid, kPushBlock, 0, s->stream>>>(s->a);
        s->ahead = true;
    }
    // Each batch of steps is captured with its event records as one CUDA
    // graph and replayed, so kernels run back to back and the events time
    // the GPU, not the host's launch rate.
    for (int64_t done = 0; done < steps && st == MGC_OK;) {
        const int b = (int)std::min<int64_t>(kBatch, steps - done);
        if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            st = fail(MGC_ERR_CUDA, "profile: stream capture failed");
            break;
        }
        for (int i = 0; i < b; ++i) {
            cudaEvent_t* e = &ev[4 * i];
            // ms[0] neuron update, ms[1] event delivery (push or deferred), ms[2] STDP
            if (s->a.deferred && s->fused) {
                // the fused step timed as its two parts: neuron update of
                // step s, then delivery of the arrivals of step s+1
                rec(e[0]);
                k_neuron<<<s->neuron_grid, kNeuronBlock, 0, s->stream>>>(s->a);
                rec(e[1]);
                k_deliver<<<s->deliver_grid, kPushBlock, 0, s->stream>>>(s->a);
                rec(e[2]);
                rec(e[3]);
            } else if (s->a.deferred) {
                rec(e[0]);
                k_deliver<<<s->deliver_grid, kPushBlock, 0, s->stream>>>(s->a);
                rec(e[1]);
                k_neuron<<<s->neuron_grid, kNeuronBlock, 0, s->stream>>>(s->a);
                rec(e[2]);
                rec(e[3]);
            } else {
                rec(e[0]);
                k_neuron<<<s->neuron_grid, kNeuronBlock, 0, s->stream>>>(s->a);
                rec(e[1]);
                if (s->a.pull) {
                    k_pull<<<s->pull_grid, kPushBlock, 0, s->stream>>>(s->a);  // delivery + STDP
                } else {
                    k_push<<<s->push_grid, kPushBlock, 0, s->stream>>>(s->a);
                }
                rec(e[2]);
                if (s->stdp && !s->a.pull) k_stdp<<<s->stdp_grid, kPushBlock, 0, s->stream>>>(s->a);
                rec(e[3]);
            }
            s->launches += s->a.deferred ? 2 : kernels_per_step(s);
        }
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        cudaError_t err = cudaStreamEndCapture(s->stream, &g);
        if (err == cudaSuccess) err = cudaGraphInstantiate(&ge, g, 0);
        if (g) cudaGraphDestroy(g);
        if (err == cudaSuccess) err = cudaGraphLaunch(ge, s->stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(s->stream);
        if (ge) cudaGraphExecDestroy(ge);
        if (err != cudaSuccess) {
            st = fail(MGC_ERR_CUDA, "profile: %s", cudaGetErrorString(err));
            break;
        }
        for (int i = 0; i < b; ++i) {
            float t0 = 0, t1 = 0, t2 = 0;
            cudaEvent_t* e = &ev[4 * i];
            err = cudaEventElapsedTime(&t0, e[0], e[1]);
            if (err == cudaSuccess) err = cudaEventElapsedTime(&t1, e[1], e[2]);
            if (err == cudaSuccess) err = cudaEventElapsedTime(&t2, e[2], e[3]);
            if (err != cudaSuccess) {
                st = fail(MGC_ERR_CUDA, "profile: event time: %s", cudaGetErrorString(err));
                break;
            }
            if (s->a.deferred && s->fused) {
                acc[0] += t0;
                acc[1] += t1;
            } else if (s->a.deferred) {
                acc[1] += t0;
                acc[0] += t1;
            } else {
                acc[0] += t0;
                acc[1] += t1;
                if (s->stdp && !s->a.pull) acc[2] += t2;  // else no kernel between e[2] and e[3]
            }
        }
        done += b;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (int k = 0; k < 3; ++k) ms[k] = (float)acc[k];
    return st;
}

namespace {

// Launch configuration the autotuner varies: synapses per delivery task
// (deferred method) and resident blocks per SM of the step's main kernel
// (for the fused method: its instantiation for 2 or 3 blocks per SM).
struct TuneCand {
    int64_t chunk_target;
    int blocks_per_sm;
};

int& tuned_grid(mgc_sim* s)
{
    if (s->a.deferred) return s->fused ? s->fused_grid : s->deliver_grid;
    return s->a.pull ? s->pull_grid : s->push_grid;
}

mgc_status apply_cand(mgc_sim* s, const TuneCand& c, int sms)
{
    if (s->graph) {  // the graph holds the old launch parameters
        CK(cudaStreamSynchronize(s->stream));
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
        s->sched_graph = false;
    }
    if (s->a.deferred) set_chunking(s->a, s->max_gap, c.chunk_target);
    if (s->fused) {
        s->fused_variant = c.blocks_per_sm >= 3 ? 1 : 0;
        s->fused_grid = s->fused_grid_v[s->fused_variant];
        CKS(sched_put(s, &SchedState::static_variant, (int32_t)s->fused_variant));
    } else {
        tuned_grid(s) = sms * c.blocks_per_sm;
    }
    return MGC_OK;
}

}  // namespace

mgc_status mgc_set_persistent(mgc_sim* s, int32_t mode)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    if (mode < 0 || mode > 3) return fail(MGC_ERR_INVALID, "step-group mode %d (0, 1, 2 or 3)", mode);
    if (mode && !s->a.deferred) return fail(MGC_ERR_INVALID, "step groups need the deferred method");
    if (mode == 2 && !s->fused) return fail(MGC_ERR_INVALID, "the pipelined step group needs a minimum delay >= 4");
    if (mode == 2 && s->dmin < 4) return fail(MGC_ERR_INVALID, "the pipelined step group needs a minimum delay >= 4");
    if (mode == 3 && !s->fused) return fail(MGC_ERR_INVALID, "the windowed step group needs a minimum delay >= 2");
    if (s->graph && s->persistent != mode) {  // the scheduler's graph holds step groups of the old mode
        CK(cudaStreamSynchronize(s->stream));
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
        s->sched_graph = false;
    }
    s->persistent = mode;
    return MGC_OK;
}

mgc_status mgc_set_window(mgc_sim* s, int32_t steps)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    if (!s->fused) return fail(MGC_ERR_INVALID, "the windowed step group needs a minimum delay >= 2");
    const int most = std::min(kMaxWindow, s->dmin);
    if (steps < 1 || steps > most) return fail(MGC_ERR_INVALID, "window of %d steps (1 to %d)", steps, most);
    s->window = steps;
    return MGC_OK;
}

mgc_status mgc_autotune(mgc_sim* s, int64_t steps_per_trial, mgc_tune_report* rep)
{
    if (!s || !rep || steps_per_trial < 1) return fail(MGC_ERR_INVALID, "bad autotune arguments");
    if (s->partition) return fail(MGC_ERR_INVALID, "partition handles run steps only between exchanges (mgc_run)");
    CK(cudaSetDevice(s->device));
    memset(rep, 0, sizeof(*rep));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, s->device));
    const int sms = prop.multiProcessorCount;
    int occ = 1, occ_min = 1;
    if (s->fused) {
        occ_min = 2;  // the two instantiations of the fused kernel
        occ = 3;
    } else if (s->a.deferred) {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_deliver, kPushBlock, 0));
    } else {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, s->a.pull ? (const void*)k_pull : (const void*)k_push,
                                                         kPushBlock, 0));
    }
    occ = std::max(1, occ);
    // the builder's choice first, then the grid of chunk lengths x blocks per SM
    std::vector<TuneCand> cands;
    cands.push_back({s->a.deferred ? kDefaultChunk : 0,
                     s->fused ? (s->fused_variant == 1 ? 3 : 2) : std::max(1, tuned_grid(s) / sms)});
    const int64_t targets[] = {64, 128, 256, 512, 1024};
    for (int64_t t : s->a.deferred ? std::vector<int64_t>(targets, targets + 5) : std::vector<int64_t>{0})
        for (int b = occ_min; b <= occ; ++b) {
            if (t == cands[0].chunk_target && b == cands[0].blocks_per_sm) continue;
            if (s->a.deferred && t > kDefaultChunk && s->max_gap <= kDefaultChunk) continue;  // same chunking
            cands.push_back({t, b});
        }
    const int64_t steps = (steps_per_trial + kGraphSteps - 1) / kGraphSteps * kGraphSteps;
    s->persistent = 0;  // the shapes are timed as graphs of single-step kernels, step groups after
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double best = 1e300;
    size_t best_i = 0;
    mgc_status st = MGC_OK;
    for (size_t i = 0; i < cands.size() && st == MGC_OK; ++i) {
        st = apply_cand(s, cands[i], sms);
        if (st == MGC_OK) st = mgc_run(s, kGraphSteps);  // builds the graph, settles the state
        if (st != MGC_OK) break;
        cudaEventRecord(e0, s->stream);
        st = mgc_run(s, steps);
        cudaEventRecord(e1, s->stream);
        if (st != MGC_OK) break;
        float ms = 0.f;
        cudaError_t err = cudaEventSynchronize(e1);
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        if (err != cudaSuccess) {
            st = fail(MGC_ERR_CUDA, "autotune: %s", cudaGetErrorString(err));
            break;
        }
        const double per = (double)ms / (double)steps;
        if (i == 0) rep->default_ms_per_step = per;
        if (per < best) {
            best = per;
            best_i = i;
        }
        rep->trials += 1;
    }
    TuneCand best_c = cands[best_i];
    const int window0 = s->window;
    int best_window = window0;
    // step-group trials: p = 1, 2 of both instantiations, then the windows
    // 2..min(4, min delay) of the windowed group (p = 3) of both
    std::vector<std::pair<int, int>> groups;  // (mode, window)
    if (s->fused) {
        for (int p = 1; p <= 2; ++p)
            if (p == 1 || s->dmin >= 4) groups.push_back({p, window0}), groups.push_back({p, window0});
        for (int w = 2; w <= std::min(kMaxWindow, s->dmin); ++w) groups.push_back({3, w}), groups.push_back({3, w});
    } else {
        groups.push_back({1, window0});
    }
    for (size_t t = 0; t < groups.size() && st == MGC_OK && s->a.deferred && !sched_wanted(s); ++t) {
        // the best chunking once more as step groups of each kernel
        // instantiation: their best register budget can differ from the
        // single-step kernel's (a minimum delay of 1: the one step-group
        // form, k_steps1)
        const int p = groups[t].first;
        const TuneCand c = s->fused ? TuneCand{cands[best_i].chunk_target, t % 2 == 0 ? 2 : 3} : cands[best_i];
        st = apply_cand(s, c, sms);
        s->persistent = p;
        s->window = groups[t].second;
        if (st == MGC_OK) st = mgc_run(s, kGraphSteps);
        if (st == MGC_OK) {
            cudaEventRecord(e0, s->stream);
            st = mgc_run(s, steps);
            cudaEventRecord(e1, s->stream);
        }
        float ms = 0.f;
        if (st == MGC_OK && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) {
            const double per = (double)ms / (double)steps;
            rep->trials += 1;
            if (per < best) {
                best = per;
                rep->persistent = p;
                best_c = c;
                best_window = groups[t].second;
            }
        }
        if (st == MGC_OK) st = mgc_sync(s);
    }
    s->persistent = rep->persistent;
    s->window = best_window;
    rep->window = s->fused ? s->window : 0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != MGC_OK) return st;
    CKS(apply_cand(s, best_c, sms));
    rep->ms_per_step = best;
    rep->chunk_len = s->a.deferred ? s->a.chunk_len : 0;
    rep->blocks_per_sm = best_c.blocks_per_sm;
    rep->steps = (int64_t)rep->trials * (steps + kGraphSteps);
    return MGC_OK;
}

// ---- scheduler -------------------------------------------------------------

namespace {

mgc_status need_sched(mgc_sim* s)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    if (!s->sched) return fail(MGC_ERR_INVALID, "the step scheduler needs the fused deferred method (min delay >= 2)");
    CK(cudaSetDevice(s->device));
    return MGC_OK;
}

mgc_status read_sched(mgc_sim* s, SchedState* h)
{
    CK(cudaStreamSynchronize(s->stream));
    CK(cudaMemcpy(h, s->sched, sizeof(*h), cudaMemcpyDeviceToHost));
    return MGC_OK;
}

// Least-squares line t = a + b*x.
bool fit_line(const std::vector<double>& x, const std::vector<double>& t, double* a, double* b)
{
    const size_t n = x.size();
    if (n < 2) return false;
    double mx = 0, mt = 0;
    for (size_t i = 0; i < n; ++i) {
        mx += x[i];
        mt += t[i];
    }
    mx /= n;
    mt /= n;
    double sxx = 0, sxt = 0;
    for (size_t i = 0; i < n; ++i) {
        sxx += (x[i] - mx) * (x[i] - mx);
        sxt += (x[i] - mx) * (t[i] - mt);
    }
    *b = sxx > 0 ? sxt / sxx : 0.0;
    *a = mt - *b * mx;
    return true;
}

}  // namespace

mgc_status mgc_sched_set_mode(mgc_sim* s, int32_t mode)
{
    CKS(need_sched(s));
    if (mode < MGC_SCHED_STATIC || mode > MGC_SCHED_LEARNED) return fail(MGC_ERR_INVALID, "unknown schedule mode %d", mode);
    SchedState h;
    CKS(read_sched(s, &h));
    if (mode == MGC_SCHED_LEARNED && !h.trained) return fail(MGC_ERR_INVALID, "the scheduler's network is not trained");
    CKS(sched_put(s, &SchedState::have_prev, (int32_t)0));
    CKS(sched_put(s, &SchedState::mode, mode));
    s->sched_mode_h = mode;
    return refresh_graph(s);
}

mgc_status mgc_sched_set_threshold(mgc_sim* s, double threshold, int32_t hi_variant)
{
    CKS(need_sched(s));
    if (hi_variant < 0 || hi_variant > 1) return fail(MGC_ERR_INVALID, "variant must be 0 or 1");
    CKS(sched_put(s, &SchedState::threshold, (float)threshold));
    CKS(sched_put(s, &SchedState::hi_variant, hi_variant));
    return MGC_OK;
}

mgc_status mgc_sched_collect(mgc_sim* s, int32_t on, int32_t reset)
{
    CKS(need_sched(s));
    if (reset) CKS(sched_put(s, &SchedState::n_data, (int32_t)0));
    CKS(sched_put(s, &SchedState::collect, (int32_t)(on != 0)));
    s->sched_collect_h = on != 0;
    return refresh_graph(s);
}

mgc_status mgc_sched_calibrate(mgc_sim* s, int32_t groups, double* threshold)
{
    CKS(need_sched(s));
    if (s->partition) return fail(MGC_ERR_INVALID, "partition handles run steps only between exchanges (mgc_run)");
    if (groups < 4 || groups > kMaxDataset / 2) return fail(MGC_ERR_INVALID, "calibrate with 4..%d groups", kMaxDataset / 2);
    SchedState h;
    s->sched_forced_h = true;
    CKS(refresh_graph(s));
    CKS(mgc_run(s, kGraphSteps));  // builds the step-group graph, settles the state
    CKS(read_sched(s, &h));
    if (!s->sched_graph) return fail(MGC_ERR_CUDA, "the step-group graph has no scheduler branch");
    const int32_t collect0 = h.collect;
    CKS(sched_put(s, &SchedState::collect, (int32_t)1));
    if (h.n_data + groups + 2 > kMaxDataset) CKS(sched_put(s, &SchedState::n_data, (int32_t)0));
    CKS(read_sched(s, &h));
    const int32_t n0 = h.n_data;
    std::vector<cudaEvent_t> ev(2 * (groups + 1));
    for (auto& e : ev) CK(cudaEventCreate(&e));
    std::vector<float> ms(groups + 1, 0.f);
    mgc_status st = MGC_OK;
    for (int g = 0; g <= groups && st == MGC_OK; ++g) {
        st = sched_put(s, &SchedState::forced_variant, (int32_t)(g % 2));
        if (st != MGC_OK) break;
        cudaEventRecord(ev[2 * g], s->stream);
        st = mgc_run(s, kGraphSteps);
        cudaEventRecord(ev[2 * g + 1], s->stream);
    }
    if (st == MGC_OK) st = sched_put(s, &SchedState::forced_variant, (int32_t)-1);
    s->sched_forced_h = false;
    if (st == MGC_OK) st = refresh_graph(s);
    if (st == MGC_OK && cudaStreamSynchronize(s->stream) != cudaSuccess) st = fail(MGC_ERR_CUDA, "calibration run failed");
    for (int g = 0; g <= groups && st == MGC_OK; ++g) cudaEventElapsedTime(&ms[g], ev[2 * g], ev[2 * g + 1]);
    for (auto& e : ev) cudaEventDestroy(e);
    if (st != MGC_OK) return st;
    // features of group g were recorded when group g+1 started
    std::vector<float> rows((size_t)(groups + 1) * kTraceCols);
    CK(cudaMemcpy(rows.data(), s->sched_data + (size_t)n0 * kTraceCols, rows.size() * sizeof(float),
                  cudaMemcpyDeviceToHost));
    std::vector<double> x[2], t[2];
    for (int g = 0; g < groups; ++g) {
        const double load = std::expm1((double)rows[(size_t)(g + 1) * kTraceCols + kTracePops]);
        x[g % 2].push_back(load);
        t[g % 2].push_back((double)ms[g] / kGraphSteps);
    }
    double a0 = 0, b0 = 0, a1 = 0, b1 = 0;
    fit_line(x[0], t[0], &a0, &b0);
    fit_line(x[1], t[1], &a1, &b1);
    double lo = 1e300, hi = -1e300, m0 = 0, m1 = 0;
    for (int v = 0; v < 2; ++v)
        for (size_t i = 0; i < x[v].size(); ++i) {
            lo = std::min(lo, x[v][i]);
            hi = std::max(hi, x[v][i]);
            (v ? m1 : m0) += t[v][i] / x[v].size();
        }
    float thr = 1e30f;
    int32_t hi_v = m0 <= m1 ? 1 : 0;  // with thr = inf: always the faster variant on average
    if (b0 != b1) {
        const double xc = (a1 - a0) / (b0 - b1);
        if (xc > lo && xc < hi) {
            thr = (float)xc;
            hi_v = b1 < b0 ? 1 : 0;  // the flatter line wins at high load
        }
    }
    CKS(sched_put(s, &SchedState::threshold, thr));
    CKS(sched_put(s, &SchedState::hi_variant, hi_v));
    CKS(sched_put(s, &SchedState::collect, collect0));
    if (threshold) *threshold = thr;
    return MGC_OK;
}

mgc_status mgc_sched_train(mgc_sim* s, int32_t epochs, float lr, uint64_t seed, float* loss)
{
    CKS(need_sched(s));
    if (epochs < 1 || !(lr > 0.f)) return fail(MGC_ERR_INVALID, "bad training arguments");
    SchedState h;
    CKS(read_sched(s, &h));
    const int n_rows = h.n_data;
    const int n = n_rows - kGroupLag;
    if (n < 16) return fail(MGC_ERR_INVALID, "%d recorded groups; training needs at least %d", n_rows, kGroupLag + 16);
    std::vector<float> rows((size_t)n_rows * kTraceCols);
    CK(cudaMemcpy(rows.data(), s->sched_data, rows.size() * sizeof(float), cudaMemcpyDeviceToHost));
    // windows: kGroupLag consecutive groups (oldest first) -> the next group
    std::vector<float> X((size_t)n * kMlpIn), Y((size_t)n * kMlpOut);
    for (int t = 0; t < n; ++t) {
        for (int i = 0; i < kMlpIn; ++i) X[(size_t)t * kMlpIn + i] = rows[(size_t)t * kTraceCols + i];
        for (int o = 0; o < kMlpOut; ++o) Y[(size_t)t * kMlpOut + o] = rows[(size_t)(t + kGroupLag) * kTraceCols + o];
    }
    auto standardize = [&](std::vector<float>& M, int cols, float* mean, float* sd) {
        for (int c = 0; c < cols; ++c) {
            double m = 0, v = 0;
            for (int t = 0; t < n; ++t) m += M[(size_t)t * cols + c];
            m /= n;
            for (int t = 0; t < n; ++t) v += (M[(size_t)t * cols + c] - m) * (M[(size_t)t * cols + c] - m);
            const double d = std::max(std::sqrt(v / n), 1e-3);
            mean[c] = (float)m;
            sd[c] = (float)d;
            for (int t = 0; t < n; ++t) M[(size_t)t * cols + c] = (float)((M[(size_t)t * cols + c] - m) / d);
        }
    };
    standardize(X, kMlpIn, h.xm, h.xs);
    standardize(Y, kMlpOut, h.ym, h.ys);
    // Glorot-uniform initial weights from the seed, zero biases
    for (int k = 0; k < kMlpParams; ++k) {
        const bool w1 = k < mlp_b1(), w2 = k >= mlp_w2() && k < mlp_b2();
        const double lim = w1 ? std::sqrt(6.0 / (kMlpIn + kMlpHidden)) : std::sqrt(6.0 / (kMlpHidden + kMlpOut));
        const U32x4 r = philox4x32_10((uint32_t)k, 0u, 0u, 0x4D4C5049u /* "MLPI" */, (uint32_t)seed, (uint32_t)(seed >> 32));
        h.p[k] = (w1 || w2) ? (float)((2.0 * unit_open0(r.x) - 1.0) * lim) : 0.f;
    }
    h.trained = 0;
    CK(cudaMemcpy(s->sched, &h, sizeof(h), cudaMemcpyHostToDevice));
    DevTmp tx, ty, tl;
    float *dX, *dY, *dl;
    CKS(tmp_alloc(tx, &dX, X.size()));
    CKS(tmp_alloc(ty, &dY, Y.size()));
    CKS(tmp_alloc(tl, &dl, 1));
    CK(cudaMemcpy(dX, X.data(), X.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dY, Y.data(), Y.size() * sizeof(float), cudaMemcpyHostToDevice));
    k_mlp_train<<<1, 256, 0, s->stream>>>(s->sched, dX, dY, n, epochs, lr, seed, dl);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    float l = 0.f;
    CK(cudaMemcpy(&l, dl, sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
    CKS(sched_put(s, &SchedState::trained, (int32_t)1));
    return MGC_OK;
}

mgc_status mgc_sched_report(mgc_sim* s, mgc_sched_stats* r, int32_t reset)
{
    CKS(need_sched(s));
    if (!r) return fail(MGC_ERR_INVALID, "null report");
    SchedState h;
    CKS(read_sched(s, &h));
    memset(r, 0, sizeof(*r));
    r->mode = h.mode;
    r->trained = h.trained;
    r->groups = h.groups;
    r->misses = h.misses;
    r->variant_groups[0] = h.variant_groups[0];
    r->variant_groups[1] = h.variant_groups[1];
    r->mean_abs_log_err = h.err_groups ? h.abs_log_err / (double)h.err_groups : 0.0;
    r->threshold = h.threshold;
    r->hi_variant = h.hi_variant;
    r->static_variant = h.static_variant;
    r->recorded_groups = h.n_data;
    if (reset) {
        h.groups = h.misses = h.err_groups = 0;
        h.variant_groups[0] = h.variant_groups[1] = 0;
        h.abs_log_err = 0.0;
        h.have_prev = 0;
        CK(cudaMemcpy(s->sched, &h, sizeof(h), cudaMemcpyHostToDevice));
    }
    return MGC_OK;
}

mgc_status mgc_mlp_gradient(int32_t device, const float* params, const float* x, const float* y, int32_t n, float* grad,
                            float* loss)
{
    if (!params || !x || !y || !grad || !loss || n < 1 || n > kMaxGradSamples)
        return fail(MGC_ERR_INVALID, "mgc_mlp_gradient: 1..%d samples", kMaxGradSamples);
    CK(cudaSetDevice(device));
    DevTmp tp, tx, ty, tg, tl;
    float *dp, *dx, *dy, *dg, *dl;
    CKS(tmp_alloc(tp, &dp, kMlpParams));
    CKS(tmp_alloc(tx, &dx, (size_t)n * kMlpIn));
    CKS(tmp_alloc(ty, &dy, (size_t)n * kMlpOut));
    CKS(tmp_alloc(tg, &dg, kMlpParams));
    CKS(tmp_alloc(tl, &dl, 1));
    CK(cudaMemcpy(dp, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dx, x, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dy, y, sizeof(float) * n * kMlpOut, cudaMemcpyHostToDevice));
    k_mlp_gradient<<<1, 256>>>(dp, dx, dy, n, dg, dl);
    CK(cudaGetLastError());
    CK(cudaMemcpy(grad, dg, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(loss, dl, sizeof(float), cudaMemcpyDeviceToHost));
    return MGC_OK;
}

// ---- checkpoints -------------------------------------------------------------

namespace {

constexpr uint64_t kCheckpointMagic = 0x3130545043474d4dull;  // "MMGCPT01"

struct CheckpointHeader {
    uint64_t magic;
    int64_t n, ns, S;
    int32_t mode, M, H, D, stdp, ahead;
    int64_t bytes;  // whole checkpoint
};

struct Segment {
    void* dev;
    size_t bytes;
};

// The device state a step depends on, in a fixed order.
std::vector<Segment> state_segments(mgc_sim* s)
{
    StepArgs& a = s->a;
    const size_t ns = (size_t)a.ns, n = (size_t)s->n;
    std::vector<Segment> v = {
        {a.V, 4 * ns}, {a.Iexc, 4 * ns}, {a.Iinh, 4 * ns}, {a.refrac, 4 * ns}, {a.last_fired, 4 * ns},
        {a.fire_cnt, 4 * ns}, {const_cast<float*>(a.rate), 4 * ns}, {a.step, 16}, {a.events, 8},
        {a.spk_count, 4}};
    if (a.deferred) {
        v.push_back({a.acc_e, 4 * kAccBuffers * ns});
        v.push_back({a.acc_i, 4 * kAccBuffers * ns});
        v.push_back({a.hist_ids, 4 * (size_t)a.H * (size_t)s->n_src});
        v.push_back({a.hist_cnt, 4 * (size_t)a.H});
    } else {
        v.push_back({a.ring_e, 4 * (size_t)s->M * ns});
        v.push_back({a.ring_i, 4 * (size_t)s->M * ns});
        v.push_back({a.spk, 4 * n});
    }
    if (s->stdp) v.push_back({a.pull ? (void*)a.in_ent : (void*)a.syn, 8 * (size_t)s->S});  // plastic weights
    return v;
}

CheckpointHeader checkpoint_header(mgc_sim* s)
{
    CheckpointHeader h{};
    h.magic = kCheckpointMagic;
    h.n = s->n;
    h.ns = s->a.ns;
    h.S = s->S;
    h.mode = s->mode;
    h.M = s->M;
    h.H = s->a.H;
    h.D = s->a.D;
    h.stdp = s->stdp;
    h.ahead = s->ahead;
    h.bytes = sizeof(CheckpointHeader);
    for (const Segment& g : state_segments(s)) h.bytes += (int64_t)g.bytes;
    return h;
}

}  // namespace

mgc_status mgc_checkpoint_size(mgc_sim* s, int64_t* bytes)
{
    if (!s || !bytes) return fail(MGC_ERR_INVALID, "null argument");
    *bytes = checkpoint_header(s).bytes;
    return MGC_OK;
}

mgc_status mgc_checkpoint_save(mgc_sim* s, void* buf, int64_t bytes)
{
    if (!s || !buf) return fail(MGC_ERR_INVALID, "null argument");
    if (s->partition && s->pending)
        return fail(MGC_ERR_INVALID, "partition: save a checkpoint right after an exchange");
    CK(cudaSetDevice(s->device));
    const CheckpointHeader h = checkpoint_header(s);
    if (bytes < h.bytes) return fail(MGC_ERR_INVALID, "checkpoint buffer of %lld bytes, need %lld", (long long)bytes,
                                     (long long)h.bytes);
    CK(cudaStreamSynchronize(s->stream));
    char* p = static_cast<char*>(buf);
    memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    for (const Segment& g : state_segments(s)) {
        CK(cudaMemcpy(p, g.dev, g.bytes, cudaMemcpyDeviceToHost));
        p += g.bytes;
    }
    return MGC_OK;
}

mgc_status mgc_checkpoint_load(mgc_sim* s, const void* buf, int64_t bytes)
{
    if (!s || !buf) return fail(MGC_ERR_INVALID, "null argument");
    CK(cudaSetDevice(s->device));
    CheckpointHeader h;
    if (bytes < (int64_t)sizeof(h)) return fail(MGC_ERR_INVALID, "not a checkpoint");
    memcpy(&h, buf, sizeof(h));
    const CheckpointHeader mine = checkpoint_header(s);
    if (h.magic != kCheckpointMagic) return fail(MGC_ERR_INVALID, "not a checkpoint");
    if (h.n != mine.n || h.S != mine.S || h.mode != mine.mode || h.M != mine.M || h.H != mine.H || h.D != mine.D ||
        h.stdp != mine.stdp || h.bytes != mine.bytes || bytes < h.bytes)
        return fail(MGC_ERR_INVALID, "the checkpoint is of another network or method");
    CK(cudaStreamSynchronize(s->stream));
    const char* p = static_cast<const char*>(buf) + sizeof(h);
    for (const Segment& g : state_segments(s)) {
        CK(cudaMemcpy(g.dev, p, g.bytes, cudaMemcpyHostToDevice));
        p += g.bytes;
    }
    // the raster starts empty at the restored step; nothing is pending
    int64_t step = 0;
    const int64_t zero = 0;
    const int32_t zero32 = 0;
    CK(cudaMemcpy(&step, s->a.step, 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(s->a.raster_step0, &step, 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->a.raster_pos, &zero, 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->a.status, &zero32, 4, cudaMemcpyHostToDevice));
    if (s->a.ev_mark) {
        unsigned long long ev = 0;
        CK(cudaMemcpy(&ev, s->a.events, 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(s->a.ev_mark, &ev, 8, cudaMemcpyHostToDevice));
    }
    s->ahead = h.ahead != 0;
    s->pending = 0;  // a partition's checkpoint is taken between exchanges
    return MGC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Spike exchange between partitions.  A partition handle's history holds the
// spike ids (whole-network ids) of every neuron; its own neuron update writes
// its neurons' spikes, and the other partitions' spikes of the steps run since
// the last exchange are appended after them.  Deliveries of step x read the
// spikes of steps <= x - min_delay, so exchanging every <= min_delay - 1 steps
// hands each partition every spike before it is delivered.
// ---------------------------------------------------------------------------
namespace {

// History slot of the step `back` steps before the device's current one.
__device__ __forceinline__ int32_t slot_back(const StepArgs& a, int32_t back)
{
    const int32_t h = a.slots[1] - back;
    return h < 0 ? h + a.H : h;
}

// Block j: the spikes of step (current - count + j) into counts[j] and, when
// they fit, into ids after those of the earlier steps.
__global__ void k_part_export(StepArgs a, int32_t count, int32_t* counts, int32_t* ids, int64_t cap)
{
    const int32_t j = blockIdx.x;
    int64_t off = 0;
    for (int32_t q = 0; q < j; ++q) off += a.hist_cnt[slot_back(a, count - q)];
    const int32_t hs = slot_back(a, count - j);
    const int32_t c = a.hist_cnt[hs];
    if (threadIdx.x == 0) counts[j] = c;
    if (!ids || off + c > cap) return;  // the host reports the overflow from the counts
    const int32_t* src = a.hist_ids + (size_t)hs * (size_t)a.n_src;
    for (int32_t i = threadIdx.x; i < c; i += blockDim.x) ids[off + i] = src[i];
}

// Block (j, r), r != self: rank r's spikes of step (current - count + j),
// stored from ids + r * stride after its spikes of the earlier steps, go
// after the slot's own spikes and those of the ranks before r.  Rank q's
// count of step j is cnt[q * cnt_stride + j].  A rank whose window holds
// more than cap ids (its buffer cut them), a negative count, an id outside
// the network or a slot that would hold more than every neuron sets
// kStatusExchange and the counts stay as they were (k_part_commit), so no
// delivery reads what was written.
__global__ void k_part_import(StepArgs a, int32_t count, int32_t nranks, int32_t self, const int32_t* cnt,
                              int64_t cnt_stride, const int32_t* ids, int64_t stride, int64_t cap)
{
    const int32_t j = blockIdx.x, r = blockIdx.y;
    int64_t src = (int64_t)r * stride, rank_total = 0;
    bool bad = false;
    for (int32_t q = 0; q < count; ++q) {
        const int32_t c = cnt[(size_t)r * cnt_stride + q];
        bad |= c < 0;
        rank_total += c;
        if (q < j) src += c;
    }
    if (r == self) {  // its own window cut short makes the others refuse: refuse here too
        if (threadIdx.x == 0 && rank_total > cap) atomicOr(a.status, kStatusExchange);
        return;
    }
    const int32_t hs = slot_back(a, count - j);
    const int64_t own = a.hist_cnt[hs];
    int64_t dst = own, total = own;
    for (int32_t q = 0; q < nranks; ++q) {
        if (q == self) continue;
        const int32_t c = cnt[(size_t)q * cnt_stride + j];
        if (q < r) dst += c;
        total += c;
    }
    if (bad || rank_total > cap || total > a.n_src) {
        if (threadIdx.x == 0) atomicOr(a.status, kStatusExchange);
        return;
    }
    const int32_t c = cnt[(size_t)r * cnt_stride + j];
    int32_t* out = a.hist_ids + (size_t)hs * (size_t)a.n_src;
    for (int32_t i = threadIdx.x; i < c; i += blockDim.x) {
        const int32_t id = ids[src + i];
        if (id < 0 || id >= a.n_src) {
            atomicOr(a.status, kStatusExchange);
            continue;
        }
        out[dst + i] = id;
    }
}

// The slots' counts grow by the imported spikes, unless the import failed.
__global__ void k_part_commit(StepArgs a, int32_t count, int32_t nranks, int32_t self, const int32_t* cnt,
                              int64_t cnt_stride)
{
    if (*(volatile int32_t*)a.status & kStatusExchange) return;
    for (int32_t j = threadIdx.x; j < count; j += blockDim.x) {
        int32_t add = 0;
        for (int32_t q = 0; q < nranks; ++q)
            if (q != self) add += cnt[(size_t)q * cnt_stride + j];
        a.hist_cnt[slot_back(a, count - j)] += add;
    }
}

mgc_status xch_reserve(mgc_sim* s, int64_t count)
{
    if (s->xch_cap >= count) return MGC_OK;
    CKS(s->alloc(&s->xch, (size_t)count));
    s->xch_cap = count;
    return MGC_OK;
}

// Kernels read and write the exchange buffers directly: device memory of the
// handle's device, managed memory, or page-locked host memory mapped into
// the device's address space.
bool device_accessible(const void* p, int device)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (at.type == cudaMemoryTypeDevice) return at.device == device;
    if (at.type == cudaMemoryTypeManaged) return true;
    if (at.type == cudaMemoryTypeHost) return at.devicePointer == p;
    return false;
}

mgc_status check_window(mgc_sim* s, int32_t count)
{
    if (!s->partition) return fail(MGC_ERR_INVALID, "not a partition handle");
    if (count < 1 || count != s->pending)
        return fail(MGC_ERR_INVALID, "exchange the %d steps run since the last import (got %d)", s->pending, count);
    return MGC_OK;
}

}  // namespace

extern "C" {

mgc_status mgc_part_export(mgc_sim* s, int32_t count, int32_t* counts, int32_t* ids, int64_t ids_cap, int64_t* total)
{
    if (!s || !counts || !total || ids_cap < 0) return fail(MGC_ERR_INVALID, "null argument");
    CKS(check_window(s, count));
    CK(cudaSetDevice(s->device));
    if (ids_cap > 0 && (!ids || !device_accessible(ids, s->device)))
        return fail(MGC_ERR_INVALID, "spike id buffer is not device memory of device %d", s->device);
    CKS(xch_reserve(s, count));
    k_part_export<<<count, 256, 0, s->stream>>>(s->a, count, s->xch, ids_cap > 0 ? ids : nullptr, ids_cap);
    CK(cudaGetLastError());
    s->launches += 1;
    CK(cudaMemcpyAsync(counts, s->xch, 4 * (size_t)count, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    int64_t sum = 0;
    for (int32_t j = 0; j < count; ++j) sum += counts[j];
    *total = sum;
    if (sum > ids_cap) return fail(MGC_ERR_OVERFLOW, "%lld spike ids to export, room for %lld", (long long)sum,
                                   (long long)ids_cap);
    return MGC_OK;
}

mgc_status mgc_part_import(mgc_sim* s, int32_t count, int32_t nranks, int32_t self, const int32_t* counts,
                           const int32_t* ids, int64_t stride)
{
    if (!s || !counts || nranks < 1 || self < 0 || self >= nranks || stride < 0)
        return fail(MGC_ERR_INVALID, "bad import arguments");
    CKS(check_window(s, count));
    bool any = false;
    for (int32_t r = 0; r < nranks; ++r) {
        int64_t sum = 0;
        for (int32_t j = 0; j < count; ++j) {
            const int32_t c = counts[(size_t)r * count + j];
            if (c < 0 || c > s->n_src) return fail(MGC_ERR_INVALID, "rank %d step %d: bad spike count %d", r, j, c);
            sum += c;
        }
        if (sum > stride) return fail(MGC_ERR_INVALID, "rank %d sends %lld ids in a stride of %lld", r,
                                      (long long)sum, (long long)stride);
        any |= r != self && sum > 0;
    }
    CK(cudaSetDevice(s->device));
    if (any && (!ids || !device_accessible(ids, s->device)))
        return fail(MGC_ERR_INVALID, "spike id buffer is not device memory of device %d", s->device);
    CKS(xch_reserve(s, (int64_t)nranks * count));
    CK(cudaMemcpyAsync(s->xch, counts, 4 * (size_t)nranks * count, cudaMemcpyHostToDevice, s->stream));
    if (any) {
        k_part_import<<<dim3(count, nranks), 256, 0, s->stream>>>(s->a, count, nranks, self, s->xch, count, ids,
                                                                   stride, stride);
        k_part_commit<<<1, 256, 0, s->stream>>>(s->a, count, nranks, self, s->xch, count);
        CK(cudaGetLastError());
        s->launches += 2;
    }
    CK(cudaStreamSynchronize(s->stream));  // the counts were staged from the caller's memory
    int32_t st = 0;
    CK(cudaMemcpy(&st, s->a.status, 4, cudaMemcpyDeviceToHost));
    if (st & kStatusExchange) return fail(MGC_ERR_INVALID, "an imported spike id was out of range (exchange refused)");
    s->pending = 0;
    return MGC_OK;
}

mgc_status mgc_part_export_dev(mgc_sim* s, int32_t count, int32_t* buf, int64_t cap)
{
    if (!s || !buf || cap < 0) return fail(MGC_ERR_INVALID, "bad export arguments");
    CKS(check_window(s, count));
    CK(cudaSetDevice(s->device));
    if (!device_accessible(buf, s->device))
        return fail(MGC_ERR_INVALID, "exchange buffer is not device memory of device %d", s->device);
    k_part_export<<<count, 256, 0, s->stream>>>(s->a, count, buf, buf + count, cap);
    CK(cudaGetLastError());
    s->launches += 1;
    return MGC_OK;
}

mgc_status mgc_part_import_dev(mgc_sim* s, int32_t count, int32_t nranks, int32_t self, const int32_t* bufs, int64_t cap)
{
    if (!s || nranks < 1 || self < 0 || self >= nranks || cap < 0) return fail(MGC_ERR_INVALID, "bad import arguments");
    CKS(check_window(s, count));
    CK(cudaSetDevice(s->device));
    if (nranks > 1) {
        if (!bufs || !device_accessible(bufs, s->device))
            return fail(MGC_ERR_INVALID, "exchange buffer is not device memory of device %d", s->device);
        const int64_t blk = count + cap;  // one rank's export: counts, then ids
        k_part_import<<<dim3(count, nranks), 256, 0, s->stream>>>(s->a, count, nranks, self, bufs, blk, bufs + count,
                                                                   blk, cap);
        k_part_commit<<<1, 256, 0, s->stream>>>(s->a, count, nranks, self, bufs, blk);
        CK(cudaGetLastError());
        s->launches += 2;
    }
    s->pending = 0;
    return MGC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Failure handling without a GPU fault: host-side allocation failures, and
// the step groups' bounded waits run against a counter that nothing advances.
// ---------------------------------------------------------------------------
namespace {

// which = 0: the pipelined group's phase wait for phase 1 (gridDim.x
// arrivals on counter 1; none come).  which = 1: the per-step grid barrier
// with block 0 alone arriving (the other blocks leave).  Both give up after
// their spin limit with kStatusBarrier.
__global__ void k_wait_selftest(StepArgs a, int32_t which)
{
    __shared__ int abort_flag;
    if (threadIdx.x == 0) abort_flag = 0;
    __syncthreads();
    if (which == 0) {
        wait_phase(a, 1, &abort_flag);
    } else {
        if (blockIdx.x != 0) return;
        grid_barrier(a, &abort_flag);
    }
}

}  // namespace

extern "C" {

mgc_status mgc_fault_inject_alloc(int64_t n)
{
    if (n < 0) return fail(MGC_ERR_INVALID, "allocation count must be >= 0");
    g_fail_alloc.store(n);
    return MGC_OK;
}

mgc_status mgc_selftest_wait_timeout(int32_t device, int32_t which, int32_t* status, double* ms)
{
    if (!status || !ms || which < 0 || which > 1) return fail(MGC_ERR_INVALID, "bad self-test arguments");
    CKS(pick_device(device));
    DevTmp tb, ts;
    unsigned int* bar;
    int32_t* st;
    CKS(tmp_alloc(tb, &bar, 4));
    CKS(tmp_alloc(ts, &st, 1));
    CK(cudaMemset(bar, 0, 4 * sizeof(unsigned int)));
    CK(cudaMemset(st, 0, sizeof(int32_t)));
    StepArgs a{};
    a.bar = bar;
    a.status = st;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0));
    k_wait_selftest<<<which == 0 ? 1 : 2, 32>>>(a, which);
    const cudaError_t le = cudaGetLastError();
    CK(cudaEventRecord(e1));
    const cudaError_t se = cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(le);
    CK(se);
    CK(cudaMemcpy(status, st, sizeof(int32_t), cudaMemcpyDeviceToHost));
    *ms = t;
    return MGC_OK;
}

mgc_status mgc_get_stream(mgc_sim* s, void** stream)
{
    if (!s || !stream) return fail(MGC_ERR_INVALID, "null argument");
    *stream = (void*)s->stream;
    return MGC_OK;
}

int64_t mgc_effective_steps(int64_t steps, int32_t min_delay)
{
    if (min_delay < 1 || steps < 0) return -1;
    const int64_t cycles = steps / min_delay + (steps % min_delay == 0 ? 1 : 0);
    return std::min(steps, cycles * (int64_t)min_delay);
}

void mgc_destroy(mgc_sim* s) { delete s; }

const char* mgc_last_error(void) { return g_last_error.c_str(); }

int64_t mgc_kernel_launches(mgc_sim* s) { return s ? s->launches : 0; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Ceilings of event delivery on this device: scattered fp32 reductions fed by
// streamed 8-byte event records, and a plain stream of the same records.

namespace {

__global__ void k_scatter_records(uint2* rec, int64_t n, uint32_t n_targets, uint64_t seed)
{
    GRID_STRIDE(i, n)
    {
        const U32x4 r = philox4x32_10((uint32_t)i, (uint32_t)((uint64_t)i >> 32), 0u, 0x43454C53u /* "CELS" */,
                                      (uint32_t)seed, (uint32_t)(seed >> 32));
        rec[i] = make_uint2(scale_u32(r.x, n_targets), __float_as_uint(1e-4f));
    }
}

__global__ void k_scatter_reduce(const uint2* rec, int64_t n, float* acc)
{
    GRID_STRIDE(i, n)
    {
        const uint2 r = __ldcs(rec + i);
        red_add(acc + r.x, __uint_as_float(r.y));
    }
}

__global__ void k_scatter_read(const uint2* rec, int64_t n, float* sink)
{
    float s = 0.f;
    GRID_STRIDE(i, n)
    {
        const uint2 r = __ldcs(rec + i);
        s += __uint_as_float(r.y) * (float)(r.x & 1u);
    }
    if (s == -1.f) sink[0] = s;  // keeps the loads; never true for these records
}

}  // namespace

extern "C" mgc_status mgc_measure_scatter(int32_t device, int64_t n_events, int32_t n_targets, int32_t reps,
                                          double* red_events_per_s, double* read_bytes_per_s)
{
    if (n_events < 1 || n_targets < 1 || reps < 1 || !red_events_per_s || !read_bytes_per_s)
        return fail(MGC_ERR_INVALID, "mgc_measure_scatter: bad arguments");
    CK(cudaSetDevice(device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    DevTmp t_rec, t_acc;
    uint2* rec = nullptr;
    float* acc = nullptr;
    CKS(tmp_alloc(t_rec, &rec, (size_t)n_events));
    CKS(tmp_alloc(t_acc, &acc, (size_t)n_targets));
    CK(cudaMemset(acc, 0, sizeof(float) * (size_t)n_targets));
    const int grid = prop.multiProcessorCount * 8;
    k_scatter_records<<<grid, 256>>>(rec, n_events, (uint32_t)n_targets, 12345u);
    CK(cudaGetLastError());
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best_red = 1e30f, best_read = 1e30f;
    cudaError_t err = cudaSuccess;
    for (int r = 0; r <= reps && err == cudaSuccess; ++r) {  // r = 0 warms up
        float ms = 0.f;
        cudaEventRecord(e0);
        k_scatter_reduce<<<grid, 256>>>(rec, n_events, acc);
        cudaEventRecord(e1);
        err = cudaEventSynchronize(e1);
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        if (r) best_red = std::min(best_red, ms);
        cudaEventRecord(e0);
        k_scatter_read<<<grid, 256>>>(rec, n_events, acc);
        cudaEventRecord(e1);
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        if (r) best_read = std::min(best_read, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) return fail(MGC_ERR_CUDA, "mgc_measure_scatter: %s", cudaGetErrorString(err));
    *red_events_per_s = (double)n_events / (best_red * 1e-3);
    *read_bytes_per_s = 8.0 * (double)n_events / (best_read * 1e-3);
    return MGC_OK;
}

// ---------------------------------------------------------------------------
// CSR row offsets of a device-resident synapse list without any allocation:
// the scan's scratch is a fixed static device array.

namespace {

constexpr int kRoThreads = 256;
constexpr int kRoPerThread = 16;
constexpr int64_t kRoTile = kRoThreads * kRoPerThread;        // offsets scanned per block
constexpr int64_t kRoMaxTiles = 32768;                        // 256 KB of tile sums
constexpr int64_t kRoMaxNeurons = kRoMaxTiles * kRoTile - 1;  // 134,217,727
constexpr int kRoMaxDevices = 64;

// [0, kRoMaxTiles): tile sums, scanned in place into tile offsets;
// [kRoMaxTiles]: number of synapses whose source is out of range.
__device__ __align__(256) unsigned long long g_ro_scratch[kRoMaxTiles + 32];

std::mutex g_ro_mutex[kRoMaxDevices];              // one call per device at a time
unsigned long long* g_ro_addr[kRoMaxDevices] = {};  // scratch address on each device

__global__ void k_ro_count(const int32_t* src, int64_t S, int32_t n, unsigned long long* cnt,
                           unsigned long long* bad)
{
    GRID_STRIDE(k, S)
    {
        const int32_t v = src[k];
        if (v >= 0 && v < n) atomicAdd(cnt + v, 1ull);
        else atomicAdd(bad, 1ull);
    }
}

// Sum of each tile of kRoTile entries.
__global__ void __launch_bounds__(kRoThreads) k_ro_tile_sums(const unsigned long long* v, int64_t count,
                                                             unsigned long long* tile_sum)
{
    typedef cub::BlockReduce<unsigned long long, kRoThreads> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    const int64_t base = blockIdx.x * kRoTile;
    unsigned long long s = 0;
    for (int j = 0; j < kRoPerThread; ++j) {
        const int64_t i = base + (int64_t)j * kRoThreads + threadIdx.x;
        if (i < count) s += v[i];
    }
    s = Reduce(tmp).Sum(s);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = s;
}

// Exclusive scan of the tile sums in place (one block of 1024 threads).
__global__ void __launch_bounds__(1024) k_ro_scan_tiles(unsigned long long* t, int64_t tiles)
{
    typedef cub::BlockScan<unsigned long long, 1024> Scan;
    __shared__ typename Scan::TempStorage tmp;
    const int64_t per = (tiles + 1023) / 1024;
    const int64_t lo = threadIdx.x * per, hi = min(lo + per, tiles);
    unsigned long long s = 0;
    for (int64_t i = lo; i < hi; ++i) s += t[i];
    unsigned long long pre;
    Scan(tmp).ExclusiveSum(s, pre);
    for (int64_t i = lo; i < hi; ++i) {
        const unsigned long long x = t[i];
        t[i] = pre;
        pre += x;
    }
}

// Exclusive scan of each tile in place, plus the tile's offset.
__global__ void __launch_bounds__(kRoThreads) k_ro_apply(unsigned long long* v, int64_t count,
                                                         const unsigned long long* tile_off)
{
    typedef cub::BlockScan<unsigned long long, kRoThreads> Scan;
    __shared__ typename Scan::TempStorage tmp;
    const int64_t base = blockIdx.x * kRoTile + (int64_t)threadIdx.x * kRoPerThread;
    unsigned long long x[kRoPerThread];
    unsigned long long s = 0;
#pragma unroll
    for (int j = 0; j < kRoPerThread; ++j) {
        x[j] = base + j < count ? v[base + j] : 0ull;
        s += x[j];
    }
    unsigned long long pre;
    Scan(tmp).ExclusiveSum(s, pre);
    pre += tile_off[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kRoPerThread; ++j) {
        if (base + j < count) v[base + j] = pre;
        pre += x[j];
    }
}

}  // namespace

extern "C" mgc_status mgc_row_offsets_static(const int32_t* src, int64_t n_synapses, int32_t n_neurons,
                                             int64_t* row_ptr, void* stream)
{
    if (n_neurons < 0 || n_synapses < 0 || !row_ptr || (n_synapses > 0 && !src))
        return fail(MGC_ERR_INVALID, "mgc_row_offsets_static: bad arguments");
    if (n_neurons > kRoMaxNeurons)
        return fail(MGC_ERR_INVALID,
                    "mgc_row_offsets_static: %d neurons exceed the static scratch limit of %lld neurons",
                    n_neurons, (long long)kRoMaxNeurons);
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kRoMaxDevices)
        return fail(MGC_ERR_INVALID, "mgc_row_offsets_static: device %d beyond the %d supported", dev,
                    kRoMaxDevices);
    // Calls on one device share its scratch array: hold the device's lock
    // until this call's work has finished.
    std::lock_guard<std::mutex> lock(g_ro_mutex[dev]);
    if (!g_ro_addr[dev]) CK(cudaGetSymbolAddress(reinterpret_cast<void**>(&g_ro_addr[dev]), g_ro_scratch));
    unsigned long long* scratch = g_ro_addr[dev];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t count = (int64_t)n_neurons + 1;
    const int64_t tiles = (count + kRoTile - 1) / kRoTile;
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(row_ptr);
    unsigned long long* bad = scratch + kRoMaxTiles;
    unsigned long long nbad = 0;
    // Once the first operation is enqueued, every exit waits for the stream
    // (whatever that wait returns) before the lock is released, so that no
    // work of this call can still write the shared scratch array when the
    // next call on this device starts.
    const mgc_status rc = [&]() -> mgc_status {
        // must start at zero: the row counts (kept in row_ptr) and the bad-source count
        CK(cudaMemsetAsync(cnt, 0, sizeof(int64_t) * count, st));
        CK(cudaMemsetAsync(bad, 0, sizeof(unsigned long long), st));
        if (n_synapses) k_ro_count<<<grid_for(n_synapses), 256, 0, st>>>(src, n_synapses, n_neurons, cnt, bad);
        k_ro_tile_sums<<<(unsigned)tiles, kRoThreads, 0, st>>>(cnt, count, scratch);
        k_ro_scan_tiles<<<1, 1024, 0, st>>>(scratch, tiles);
        k_ro_apply<<<(unsigned)tiles, kRoThreads, 0, st>>>(cnt, count, scratch);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return MGC_OK;
    }();
    if (rc != MGC_OK) {
        cudaStreamSynchronize(st);
        return rc;
    }
    if (nbad)
        return fail(MGC_ERR_INVALID, "mgc_row_offsets_static: %llu synapse sources outside [0, %d)", nbad,
                    n_neurons);
    return MGC_OK;
}
