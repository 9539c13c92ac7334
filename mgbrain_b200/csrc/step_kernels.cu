// The single-step kernels of the ring and pull methods and of the deferred
// method's separate launches, and the selectors the host uses to launch them:
// k_neuron (neuron update), k_deliver (deferred delivery), k_push (ring
// push), k_push_stdp (ring push with STDP fused) and k_pull (per-target
// pass with STDP fused).
#include "sim.h"

namespace mgc {

// ---------------------------------------------------------------------------
// Pull method, after k_neuron of step s: one warp per target walks its
// incoming row.  Synapses whose source spiked at s add their (pre-update)
// weight to ring slot (s + delay) % M of the target, in the order the
// reference's push visits them for one slot (source ascending, then
// synapse-list order), so sums are the same fp32 sequence whatever the
// weights; the same pass applies the reference's STDP (mgcore.cu:365-412):
// dt = s - last_fired[target] when the source spiked, dt = last_fired[source]
// - s when the target spiked (both: dt = 0 twice).  No atomics: the warp owns
// the target's ring entries and incoming weights.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kPushBlock) k_pull(StepArgs a)
{
    const int64_t s = *a.step;
    const int32_t slot0 = a.slots[0];
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long ev = 0;
    for (int64_t T = warp; T < a.n; T += nwarps) {
        const int64_t rb = a.in_ptr[T], re = a.in_ptr[T + 1];
        if (rb == re) continue;
        const bool post = bit_of(a.fired_bits, (int32_t)T);
        const int32_t lfT = a.last_fired[T];
        // lane 0 keeps the running sums of the ring entries of one delay
        int32_t cur_d = -1;
        float ce = 0.0f, ci = 0.0f;
        bool te = false, ti = false;
        for (int64_t q0 = rb; q0 < re; q0 += 32) {
            const int64_t q = q0 + lane;
            const bool ok = q < re;
            const uint2 e = ok ? a.in_ent[q] : make_uint2(0u, 0u);
            const int32_t src = (int32_t)(e.x & a.tmask);
            const int32_t d = (int32_t)(e.x >> a.tbits);
            const float w = as_f(e.y);
            const bool in_range = !ok || MGC_OK_INDEX(src < a.n && d >= 1 && d < a.M);
            const bool pre = ok && in_range && bit_of(a.fired_bits, src);
            const unsigned m = __ballot_sync(0xffffffffu, pre);
            unsigned mm = m;
            while (mm) {  // spiking sources in row order
                const int l = __ffs(mm) - 1;
                mm &= mm - 1;
                const int32_t dl = __shfl_sync(0xffffffffu, d, l);
                const float wl = __shfl_sync(0xffffffffu, w, l);
                if (lane == 0) {
                    if (dl != cur_d) {
                        if (cur_d >= 0) {
                            int32_t sl = slot0 + cur_d;
                            if (sl >= a.M) sl -= a.M;
                            if (te) a.ring_e[(size_t)sl * a.ns + T] = ce;
                            if (ti) a.ring_i[(size_t)sl * a.ns + T] = ci;
                        }
                        cur_d = dl;
                        te = ti = false;
                    }
                    int32_t sl = slot0 + dl;
                    if (sl >= a.M) sl -= a.M;
                    if (wl > 0.0f) {
                        if (!te) {
                            ce = a.ring_e[(size_t)sl * a.ns + T];
                            te = true;
                        }
                        ce = __fadd_rn(ce, wl);
                    } else {
                        if (!ti) {
                            ci = a.ring_i[(size_t)sl * a.ns + T];
                            ti = true;
                        }
                        ci = __fadd_rn(ci, wl);
                    }
                }
            }
            if (lane == 0) ev += (unsigned long long)__popc(m);
            if (a.stdp && ok && in_range && (pre || post) && (!a.in_plastic || a.in_plastic[q])) {
                float nw = w;
                if (pre) nw = stdp_weight((int32_t)s - lfT, nw, a.P);
                if (post) nw = stdp_weight(a.last_fired[src] - (int32_t)s, nw, a.P);
                a.in_ent[q].y = as_u(nw);
            }
        }
        if (lane == 0 && cur_d >= 0) {
            int32_t sl = slot0 + cur_d;
            if (sl >= a.M) sl -= a.M;
            if (te) a.ring_e[(size_t)sl * a.ns + T] = ce;
            if (ti) a.ring_i[(size_t)sl * a.ns + T] = ci;
        }
    }
    if (lane == 0 && ev) atomicAdd(a.events, ev);
    if (last_block(a.done)) step_epilogue(a);
}


// ---------------------------------------------------------------------------
// Ring method with STDP: the event push (mgsim_syn_fast_core +
// pushInnerSpike, mgcore.cu:271-305, :112-115) and both sides of
// mgsim_stdp_core (mgcore.cu:365-412) in one pass over the step's spikes.
// Tasks: (spike, 128-synapse chunk of its outgoing row), then (spike,
// 128-entry chunk of its incoming list).  An outgoing synapse's weight is
// added to the ring before its update (the reference pushes before its STDP
// kernel), and the same lane then stores the depressed weight (dt =
// last_fired[self] - last_fired[target]).  The incoming side potentiates
// (dt = last_fired[source] - last_fired[self]) every plastic synapse whose
// source did not spike this step; those whose source did belong to that
// source's push task (both sides give dt = 0 there, and the clipped weight
// is the same once or twice), so no synapse is written by two tasks and
// every push reads its weight before any update of this step.
// ---------------------------------------------------------------------------
template <bool FX>
__global__ void __launch_bounds__(kPushBlock) k_push_stdp(StepArgs a)
{
    const int32_t cnt = *(volatile int32_t*)a.spk_count;
    const int32_t slot0 = a.slots[0];
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t tasks_out = (int64_t)cnt * a.chunks_per_spike;
    const int64_t tasks = tasks_out + (int64_t)cnt * a.chunks_in_per_spike;
    unsigned long long ev = 0;
    const int64_t rpos = a.record ? *a.raster_pos : 0;
    for (int64_t task = warp; task < tasks; task += nwarps) {
        if (task < tasks_out) {
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
            const int32_t lfn = a.last_fired[nid];
            uint2 w[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int64_t k = b + lane + 32 * u;
                w[u] = k < e ? a.syn[k] : make_uint2(0u, 0u);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int64_t k = b + lane + 32 * u;
                if (k >= e) continue;
                const uint32_t tgt = w[u].x & a.tmask;
                int32_t slot = slot0 + (int32_t)(w[u].x >> a.tbits);
                if (slot >= a.M) slot -= a.M;
                if (!MGC_OK_INDEX(tgt < (uint32_t)a.n && slot >= 0 && slot < a.M)) continue;
                const float wt = as_f(w[u].y);
                float* ring = wt > 0.0f ? a.ring_e : a.ring_i;
                const size_t at = (size_t)slot * (size_t)a.ns + tgt;
                if (FX)
                    red_add_fx(reinterpret_cast<unsigned long long*>(ring) + at, to_fx(wt, a.fx_scale));
                else
                    red_add(ring + at, wt);
                if (!a.plastic || a.plastic[k])
                    a.syn[k].y = as_u(stdp_weight(lfn - a.last_fired[tgt], wt, a.P));
            }
        } else {
            const int64_t t2 = task - tasks_out;
            const int32_t j = (int32_t)(t2 / a.chunks_in_per_spike);
            const int32_t c = (int32_t)(t2 - (int64_t)j * a.chunks_in_per_spike);
            const int32_t nid = a.spk[j];
            if (!MGC_OK_INDEX(nid >= 0 && nid < a.n)) continue;
            const int32_t lfn = a.last_fired[nid];
            const int64_t qb = a.dend_off[nid] + (int64_t)c * kChunk;
            const int64_t qe = min(a.dend_off[nid + 1], qb + (int64_t)kChunk);
            for (int64_t q = qb + lane; q < qe; q += 32) {
                const int64_t k = a.dend_pos[q];
                if (!MGC_OK_INDEX(k >= 0 && k < a.n_syn && a.csr_src[k] >= 0 && a.csr_src[k] < a.n)) continue;
                if (a.plastic && !a.plastic[k]) continue;
                const int32_t src = a.csr_src[k];
                if (bit_of(a.fired_bits, src)) continue;  // the source's push task updates it
                a.syn[k].y = as_u(stdp_weight(a.last_fired[src] - lfn, as_f(a.syn[k].y), a.P));
            }
        }
    }
    if (lane == 0 && ev) atomicAdd(a.events, ev);
    if (last_block(a.done)) step_epilogue(a);
}

StepKernel neuron_kernel(const mgc_sim* s) { return s->a.fx ? k_neuron<true> : k_neuron<false>; }
StepKernel deliver_kernel(const mgc_sim* s) { return s->a.fx ? k_deliver<true> : k_deliver<false>; }
StepKernel push_kernel(const mgc_sim* s)
{
    if (s->stdp) return s->a.fx ? k_push_stdp<true> : k_push_stdp<false>;
    return s->a.fx ? k_push<true> : k_push<false>;
}
StepKernel pull_kernel(const mgc_sim*) { return k_pull; }

}  // namespace mgc
