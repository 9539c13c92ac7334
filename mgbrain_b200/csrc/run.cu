// The step driver: one step's launches, CUDA graphs of 64 steps (with the
// scheduler's conditional node when it is on), cooperative step groups, and
// the run / sync / rate entry points.  Replaces the step loop of
// MGSimulator::simulate_sparse (src/simulator/mgsim/adj/mgsim.cpp:794-857)
// calling mgsim_step_sparse (mgcore.cu:535-554).
#include "sim.h"

using namespace mgc;

namespace {

// New POISSON probabilities into the neurons' V slots.
__global__ void k_rate_to_v(const int8_t* type, const float* rate, float* V, int32_t n)
{
    GRID_STRIDE(i, n)
    {
        if (type[i] == kPOISSON) V[i] = rate[i];
    }
}

// The current step's arrivals from buffer s & from_mask to s & to_mask (both
// accumulators; `words`: 32-bit words per entry).  Between runs only that
// buffer holds input that an update reads (the step kernels clear a buffer
// when its step's update reads it, and every step form ends with nothing
// delivered past the current step; the windowed update leaves the slots of
// groups of four POISSON neurons, whose update ignores them), so the target
// holds nothing read and the source is left zero.
__global__ void k_acc_move(float* acc_e, float* acc_i, const int64_t* step, int32_t from_mask, int32_t to_mask,
                           int64_t ns, int32_t words)
{
    const int64_t s = *step;
    const int64_t from = s & from_mask, to = s & to_mask;
    if (from == to) return;
    const int64_t n = ns * words;
    uint32_t* bufs[2] = {reinterpret_cast<uint32_t*>(acc_e), reinterpret_cast<uint32_t*>(acc_i)};
    for (uint32_t* b : bufs) {
        uint32_t* src = b + from * n;
        uint32_t* dst = b + to * n;
        GRID_STRIDE(i, n)
        {
            dst[i] = src[i];
            src[i] = 0u;
        }
    }
}

// The windowed update's rotation of neuron groups over lane positions
// (StepArgs::upd_rot) for a grid of `grid` blocks: the lanes whose last pass
// is the pass before the others' extra one take the POISSON groups, whose
// draws make theirs the costliest passes, when those neurons form one range
// of the network and fit there; else 0.  A multiple of 32 before it is taken
// modulo the groups.
int64_t update_rotation(const mgc_sim* s, int grid)
{
    const int64_t groups = s->a.ns >> 2;
    const int64_t lanes = (int64_t)grid * kPushBlock;
    if (s->pois_idx.empty() || groups < 1 || lanes < 1) return 0;
    const int64_t first = s->pois_idx.front(), last = s->pois_idx.back();
    if (last - first + 1 != (int64_t)s->pois_idx.size() || first % 4 != 0) return 0;
    const int64_t ga = first / 4, gb = (last + 4) / 4;  // the POISSON groups [ga, gb)
    const int64_t passes = groups / lanes, extra = groups % lanes;
    if (passes < 1 || extra == 0) return 0;  // every lane runs as many passes
    const int64_t t0 = (passes - 1) * lanes + extra;  // lanes without the extra pass, in their last one
    const int64_t rot0 = ga - t0;
    const int64_t rot = rot0 - (((rot0 % 32) + 32) % 32);
    if ((gb - ga) + 31 > passes * lanes - t0) return 0;
    return ((rot % groups) + groups) % groups;
}

}  // namespace

namespace mgc {

// The step-group mode the scheduler's graph runs for mode p: the windowed
// group keeps no schedule trace, so the graph takes the pipelined group (or
// the barrier per step, for a minimum delay below 4) in its place.
int graph_group_mode(const mgc_sim* s, int p) { return p == 3 ? (s->dmin >= 4 ? 2 : 1) : p; }

int32_t wanted_acc_mask(const mgc_sim* s)
{
    const bool wide = s->acc_buffers == kAccBuffersWide && s->persistent == 3 && s->window > kAccBuffers;
    return wide && !sched_wanted(s) ? kAccBuffersWide - 1 : kAccBuffers - 1;
}

mgc_status set_acc_mask(mgc_sim* s, int32_t mask, bool move)
{
    StepArgs& a = s->a;
    if (!a.deferred || mask == a.acc_mask) return MGC_OK;
    if (mask + 1 > s->acc_buffers) return fail(MGC_ERR_INVALID, "%d accumulator buffers, not %d", s->acc_buffers,
                                               mask + 1);
    if (s->graph) {  // its launches hold the old cycle
        CK(cudaStreamSynchronize(s->stream));
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
        s->sched_graph = false;
    }
    if (move) {
        k_acc_move<<<grid_for(a.ns), 256, 0, s->stream>>>(a.acc_e, a.acc_i, a.step, a.acc_mask, mask, a.ns,
                                                          a.fx ? 2 : 1);
        CK(cudaGetLastError());
        s->launches += 1;
    }
    a.acc_mask = mask;
    return MGC_OK;
}


int kernels_per_step(const mgc_sim* s)
{
    if (s->a.deferred) return s->fused ? 1 : 2;
    return 2;  // neuron update, then the push (with STDP fused) or the pull
}

mgc_status enqueue_step(mgc_sim* s)
{
    if (s->a.deferred) {
        if (s->fused) {
            if (!s->ahead) {  // arrivals of this step not yet delivered
                deliver_kernel(s)<<<s->deliver_grid, kPushBlock, 0, s->stream>>>(s->a);
                s->launches += 1;
            }
            fused_kernel(s, s->fused_variant)<<<s->fused_grid, kPushBlock, 0, s->stream>>>(s->a);
            s->ahead = true;
            s->launches += 1;
        } else {
            deliver_kernel(s)<<<s->deliver_grid, kPushBlock, 0, s->stream>>>(s->a);
            neuron_kernel(s)<<<s->neuron_grid, kNeuronBlock, 0, s->stream>>>(s->a);
            s->launches += 2;
        }
    } else {
        neuron_kernel(s)<<<s->neuron_grid, kNeuronBlock, 0, s->stream>>>(s->a);
        if (s->a.pull) {
            pull_kernel(s)<<<s->pull_grid, kPushBlock, 0, s->stream>>>(s->a);
        } else {
            push_kernel(s)<<<s->push_grid, kPushBlock, 0, s->stream>>>(s->a);
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
    kp.func = const_cast<void*>(sched_decide_kernel());
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


}  // namespace mgc

extern "C" {

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
    if (left > 0) CKS(set_acc_mask(s, wanted_acc_mask(s), true));
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
                // a window of w steps holds w buffers; each instantiation
                // is compiled for one cycle (3, or 7 above 4 steps)
                const int wide = w > kAccBuffers;
                if (s->a.acc_mask != (wide ? kAccBuffersWide : kAccBuffers) - 1)
                    return fail(MGC_ERR_INVALID, "a window of %d steps in the %d-buffer cycle", w, s->a.acc_mask + 1);
                ga.upd_rot = s->a.pull_min > 0 ? 0 : update_rotation(s, s->window_grid_v[wide][v]);
                void* wargs[] = {&ga, &n, &w};
                e = cudaLaunchCooperativeKernel((const void*)window_kernel(s, v, wide, s->a.pull_min > 0),
                                                dim3(s->window_grid_v[wide][v]), dim3(kPushBlock), wargs,
                                                s->window_smem[wide], s->stream);
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
