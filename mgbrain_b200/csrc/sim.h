// Internal declarations shared by the library's translation units: the
// simulation handle, error reporting, device allocation, the kernel
// selectors and the host helpers one part of the library calls in another.
// Not part of the C ABI (include/mgc.h).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mgc.h"
#include "kernels.cuh"
#include "sched_state.h"

namespace mgc {

// Sets the calling thread's last-error text; returns st.
mgc_status fail(mgc_status st, const char* fmt, ...);

// cudaMalloc, unless the host-side fault injector (mgc_fault_inject_alloc)
// makes this allocation fail as out of memory.
cudaError_t dev_malloc(void** p, size_t bytes);

#define CK(expr)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            if (e_ == cudaErrorMemoryAllocation) {                                                \
                cudaGetLastError();                                                               \
                return ::mgc::fail(MGC_ERR_NOMEM, "%s: %s", #expr, cudaGetErrorString(e_));       \
            }                                                                                     \
            return ::mgc::fail(MGC_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_),     \
                               __FILE__, __LINE__);                                               \
        }                                                                                         \
    } while (0)

#define CKS(expr)                    \
    do {                             \
        mgc_status s_ = (expr);      \
        if (s_ != MGC_OK) return s_; \
    } while (0)

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

constexpr int64_t kDefaultRasterSteps = 1 << 16;
constexpr int kGraphSteps = 64;
constexpr size_t kMaxBucketBytes = size_t(16) << 30;  // deferred bucket table budget
constexpr int64_t kDefaultChunk = 128;                // synapses per delivery task
constexpr int64_t kMaxChunks = 64;                    // tasks per (spike, delay) segment
constexpr int32_t kPersistentSteps = 1024;            // steps per cooperative launch

inline int bits_for(int64_t n)
{
    int b = 1;
    while ((int64_t(1) << b) < n) ++b;
    return b;
}

inline int grid_for(int64_t n, int block = 256)
{
    int64_t g = (n + block - 1) / block;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

}  // namespace mgc

struct mgc_sim {
    int device = 0;
    cudaStream_t stream = nullptr;
    mgc::StepArgs a{};
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
    int neuron_grid = 1, push_grid = 1, deliver_grid = 1, fused_grid = 1;
    bool fused = false;  // one launch per step (deferred, min delay >= 2)
    bool explicit_net = false;  // built from a synapse list (mgc_create)
    int pull_grid = 1;
    int64_t* in_syn64 = nullptr;  // synapse-list index of each incoming-row position (pull)
    bool ahead = true;   // arrivals of the current device step are already delivered
    std::vector<void*> allocs;
    std::vector<size_t> alloc_bytes;  // size of each of allocs
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
    mgc::SchedState* sched = nullptr; // device
    float* sched_data = nullptr;      // device [kMaxDataset][kTraceCols]
    bool sched_graph = false;         // the step-group graph branches on the scheduler's choice
    int persistent = 0;               // fused method as cooperative step groups: 1 barrier per
                                      // step, 2 pipelined (min delay >= 4), 3 windowed
    int group_grid_v[2][2] = {{1, 1}, {1, 1}};  // [persistent-1][variant] co-resident grids
    int window = 1;                   // steps per window of the windowed group (<= min delay, <= 8)
    int window_grid_v[2][2] = {{1, 1}, {1, 1}};  // its co-resident grids [window > 4][variant]
    size_t window_smem[2] = {0, 0};   // its dynamic shared memory [window > 4]: the delivery prefixes
    int acc_buffers = 4;              // accumulator buffers allocated (8 for a minimum delay >= 5)
    int group_grid1 = 1;              // minimum delay 1: the step group's grid
    int32_t fx_shift = 0;             // fixed-point shift the builder picked for this network's weights
    bool hetero = false;              // some neuron receives unequal weights of one sign
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
        CK(mgc::dev_malloc(&v, b));
        allocs.push_back(v);
        alloc_bytes.push_back(b);
        bytes += b;
        if (zero) CK(cudaMemsetAsync(v, 0, b, stream));
        *p = static_cast<T*>(v);
        return MGC_OK;
    }

    // Frees one of the handle's buffers (after the stream is idle).
    void release(void* p)
    {
        for (size_t i = 0; i < allocs.size(); ++i)
            if (allocs[i] == p) {
                cudaFree(p);
                bytes -= alloc_bytes[i];
                allocs.erase(allocs.begin() + i);
                alloc_bytes.erase(alloc_bytes.begin() + i);
                return;
            }
    }

    template <class T>
    mgc_status upload(T** p, const T* host, size_t count)
    {
        CKS(alloc(p, count, host == nullptr));
        if (host && count) CK(cudaMemcpyAsync(*p, host, count * sizeof(T), cudaMemcpyHostToDevice, stream));
        return MGC_OK;
    }
};

namespace mgc {

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

// ---- kernel selectors (step_kernels.cu, inst_*.cu) --------------------------
using StepKernel = void (*)(StepArgs);
using GroupKernel = void (*)(StepArgs, int32_t);
using WindowKernel = void (*)(StepArgs, int32_t, int32_t);

StepKernel neuron_kernel(const mgc_sim* s);
StepKernel deliver_kernel(const mgc_sim* s);
StepKernel push_kernel(const mgc_sim* s);
StepKernel pull_kernel(const mgc_sim* s);
// The fused step kernel for this network (with or without LIF/LIFE
// currents), variant 0 compiled for 2 resident blocks per SM, 1 for 3.
StepKernel fused_kernel(const mgc_sim* s, int v);
// The step-group kernels of the same variant: p = 1 one barrier per step,
// p = 2 pipelined; a minimum delay of 1 has its own group (k_steps1).
GroupKernel steps_kernel(const mgc_sim* s, int p, int v);
GroupKernel pipe_kernel(const mgc_sim* s, int v);
// The windowed step group of variant v: for windows of up to 4 steps, or
// (wide) of up to 8; with pull steps (mgc_set_pull) or without.
WindowKernel window_kernel(const mgc_sim* s, int v, bool wide, bool pull);
// The scheduler's decision kernel (sched.cu).
const void* sched_decide_kernel();

// ---- network construction (build.cu) ----------------------------------------
mgc_status pick_device(int device);
// Grids of the kernels the handle launches (after the kernel selection changed).
mgc_status launch_shapes(mgc_sim* s);
// The builders' steps, in order: neuron arrays and constants; the method
// (CSR word layout, delivery method, fixed-point plan: hetero = some neuron
// receives unequal weights of one sign); the CSR layout; the CSR from a
// device-resident synapse list (src, tar, weight, delay in steps, plastic
// flags or null; src is overwritten); the method's buffers and launch shapes.
mgc_status build_neurons(mgc_sim* s, int32_t n, const int8_t* type, const float* rate, const float* v_init,
                         const float* lifc, const float* stdpc, uint64_t seed, int64_t raster_steps,
                         int64_t raster_ids);
mgc_status build_method(mgc_sim* s, int requested, bool hetero, int32_t fx_shift);
// The fixed-point plan alone (a builder that learns it after the method).
mgc_status build_set_fx(mgc_sim* s, bool hetero, int32_t fx_shift);
mgc_status begin_list_layout(mgc_sim* s);
mgc_status csr_from_list(mgc_sim* s, int32_t* src, int32_t* tar, float* w, int32_t* dl, uint8_t* pl);
mgc_status build_finish(mgc_sim* s);
// The fixed-point shift rule (kernels.cuh): sums of up to `bound` fit 61
// bits; with `exact`, no finer than the smallest weight's last mantissa bit
// (min_exp: its frexp exponent).
int32_t fx_shift_rule(double bound, int min_exp, bool exact);
// The incoming rows and history bitmaps of the deferred method's pull steps,
// built once (mgc_set_pull).
mgc_status build_in_rows(mgc_sim* s);
// Frees them again (pull steps off; the stream idle first).
void release_in_rows(mgc_sim* s);
// Segments of up to `gap` synapses cut into chunks of about `target`.
void set_chunking(StepArgs& a, int64_t gap, int64_t target);

// ---- stepping (run.cu) ------------------------------------------------------
int kernels_per_step(const mgc_sim* s);
mgc_status enqueue_step(mgc_sim* s);
mgc_status build_graph(mgc_sim* s);
mgc_status build_sched_graph(mgc_sim* s);
bool sched_wanted(const mgc_sim* s);
mgc_status refresh_graph(mgc_sim* s);
// The step-group mode the scheduler's graph runs for mode p.
int graph_group_mode(const mgc_sim* s, int p);
// The accumulator cycle the next steps run with: 7 (eight buffers) while
// windowed groups of more than 4 steps run, else 3.
int32_t wanted_acc_mask(const mgc_sim* s);
// Switch the accumulator cycle to `mask`: with `move`, the buffer holding the
// current step's arrivals moves to its place in the new cycle (on the
// stream); graphs holding the old cycle are dropped.
mgc_status set_acc_mask(mgc_sim* s, int32_t mask, bool move);

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

}  // namespace mgc
