// Measurement and launch-shape selection: per-kernel timing of steps with
// CUDA events (mgc_profile_steps), the autotuner, and the step-group mode and
// window setters.
#include "sim.h"

using namespace mgc;

extern "C" {

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
        deliver_kernel(s)<<<s->deliver_grid, kPushBlock, 0, s->stream>>>(s->a);
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
                neuron_kernel(s)<<<s->neuron_grid, kNeuronBlock, 0, s->stream>>>(s->a);
                rec(e[1]);
                deliver_kernel(s)<<<s->deliver_grid, kPushBlock, 0, s->stream>>>(s->a);
                rec(e[2]);
                rec(e[3]);
            } else if (s->a.deferred) {
                rec(e[0]);
                deliver_kernel(s)<<<s->deliver_grid, kPushBlock, 0, s->stream>>>(s->a);
                rec(e[1]);
                neuron_kernel(s)<<<s->neuron_grid, kNeuronBlock, 0, s->stream>>>(s->a);
                rec(e[2]);
                rec(e[3]);
            } else {
                rec(e[0]);
                neuron_kernel(s)<<<s->neuron_grid, kNeuronBlock, 0, s->stream>>>(s->a);
                rec(e[1]);
                if (s->a.pull) {
                    pull_kernel(s)<<<s->pull_grid, kPushBlock, 0, s->stream>>>(s->a);  // delivery + STDP
                } else {
                    push_kernel(s)<<<s->push_grid, kPushBlock, 0, s->stream>>>(s->a);
                }
                rec(e[2]);
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
                (void)t2;  // STDP runs inside the push or the pull (ms[1])
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
    int grid = 0;  // ring and pull methods: a grid of fewer blocks than SMs (0: blocks_per_sm per SM)
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
        tuned_grid(s) = c.grid > 0 ? c.grid : sms * c.blocks_per_sm;
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

mgc_status mgc_set_pull(mgc_sim* s, int32_t min_pairs)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    if (min_pairs < 0) return fail(MGC_ERR_INVALID, "pull threshold %d (0 turns pull steps off)", min_pairs);
    StepArgs& a = s->a;
    if (min_pairs > 0) {
        if (!s->fused) return fail(MGC_ERR_INVALID, "pull steps need the deferred method with a minimum delay >= 2");
        if (s->partition) return fail(MGC_ERR_INVALID, "pull steps are not available for partition handles");
        if (s->hetero && !a.fx)
            return fail(MGC_ERR_INVALID, "pull steps with unequal weights of one sign need fixed-point accumulation");
    }
    CK(cudaSetDevice(s->device));
    if (s->graph) {  // its launches hold the old arguments
        CK(cudaStreamSynchronize(s->stream));
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
        s->sched_graph = false;
    }
    if (min_pairs > 0) CKS(build_in_rows(s));
    a.pull_min = min_pairs;
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
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, deliver_kernel(s), kPushBlock, 0));
    } else {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, s->a.pull ? (const void*)pull_kernel(s) : (const void*)push_kernel(s),
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
    // the ring and pull methods also at grids below one block per SM: a small
    // network's step has few tasks, and every block of the push joins the
    // step's epilogue counter
    if (!s->a.deferred)
        for (int g : {16, 37, 74}) cands.push_back({0, 1, g});
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
    // 2..min(4, min delay) of the windowed group (p = 3) of both, and the
    // longest, min(8, min delay), when above 4 (windows of 5 to 7 steps load
    // their inputs in a second, partial batch and measured slower than both
    // 4 and 8 on the benchmark networks)
    std::vector<std::pair<int, int>> groups;  // (mode, window)
    if (s->fused) {
        for (int p = 1; p <= 2; ++p)
            if (p == 1 || s->dmin >= 4) groups.push_back({p, window0}), groups.push_back({p, window0});
        for (int w = 2; w <= std::min(kAccBuffers, s->dmin); ++w) groups.push_back({3, w}), groups.push_back({3, w});
        const int widest = std::min(kMaxWindow, s->dmin);
        if (widest > kAccBuffers) groups.push_back({3, widest}), groups.push_back({3, widest});
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
    // pull steps of the windowed group (mgc_set_pull) at thresholds of n/3,
    // n/8 and n/20 arriving (spike, delay) pairs per step, on networks whose
    // incoming rows are cheap to copy (a pull step reads all of them, so it
    // pays only where that read costs less than a step's events: small dense
    // networks in bursts)
    int32_t best_pull = 0;
    const bool pull_ok = s->fused && !s->partition && !(s->hetero && !s->a.fx) && s->S > 0 &&
                         s->S <= (int64_t(1) << 27) && !sched_wanted(s);
    const bool had_rows = s->a.in_ent != nullptr;
    const int pull_window = rep->persistent == 3 ? best_window : std::min(kMaxWindow, s->dmin);
    const int32_t ths[3] = {std::max(1, s->n / 3), std::max(1, s->n / 8), std::max(1, s->n / 20)};
    for (int t = 0; t < 3 && st == MGC_OK && pull_ok; ++t) {
        st = apply_cand(s, best_c, sms);
        s->persistent = 3;
        s->window = pull_window;
        if (st == MGC_OK) st = mgc_set_pull(s, ths[t]);
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
                rep->persistent = 3;
                best_window = pull_window;
                best_pull = ths[t];
            }
        }
        if (st == MGC_OK) st = mgc_sync(s);
    }
    if (pull_ok && st == MGC_OK) st = mgc_set_pull(s, 0);
    s->persistent = rep->persistent;
    s->window = best_window;
    rep->window = s->fused ? s->window : 0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != MGC_OK) return st;
    CKS(apply_cand(s, best_c, sms));
    if (best_pull > 0)
        CKS(mgc_set_pull(s, best_pull));
    else if (pull_ok && !had_rows)
        release_in_rows(s);  // the trials' incoming rows, not needed
    rep->pull_min = best_pull;
    rep->ms_per_step = best;
    rep->chunk_len = s->a.deferred ? s->a.chunk_len : 0;
    rep->blocks_per_sm = best_c.grid > 0 ? 0 : best_c.blocks_per_sm;
    rep->steps = (int64_t)rep->trials * (steps + kGraphSteps);
    return MGC_OK;
}

mgc_status mgc_autotune_rewind(mgc_sim* s, int64_t steps_per_trial, mgc_tune_report* rep)
{
    if (!s || !rep || steps_per_trial < 1) return fail(MGC_ERR_INVALID, "bad autotune arguments");
    if (s->partition) return fail(MGC_ERR_INVALID, "partition handles run steps only between exchanges (mgc_run)");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    // the raster restarts at the restored step, so a recording handle's
    // raster must hold nothing unread
    int64_t clock[3] = {0, 0, 0};
    if (s->a.record) {
        CK(cudaMemcpy(&clock[0], s->a.step, 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&clock[1], s->a.raster_step0, 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&clock[2], s->a.raster_pos, 8, cudaMemcpyDeviceToHost));
    }
    if (clock[0] != clock[1] || clock[2] != 0)
        return fail(MGC_ERR_INVALID, "autotune with rewind: read the raster first (%lld steps unread)",
                    (long long)(clock[0] - clock[1]));
    int64_t bytes = 0;
    CKS(mgc_checkpoint_size(s, &bytes));
    std::vector<char> saved((size_t)bytes);
    CKS(mgc_checkpoint_save(s, saved.data(), bytes));
    const mgc_status st = mgc_autotune(s, steps_per_trial, rep);
    // the state goes back even when a trial failed, so that the handle
    // continues from where the call found it
    const mgc_status back = mgc_checkpoint_load(s, saved.data(), bytes);
    return st != MGC_OK ? st : back;
}

}  // extern "C"
