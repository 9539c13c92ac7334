// The single-step kernels of the ring and pull methods and of the deferred
// method's separate launches, and the selectors the host uses to launch them:
// k_neuron (neuron update), k_deliver (deferred delivery), k_push (ring
// push), k_pull (per-target pass with STDP fused) and k_stdp (ring STDP).
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
        if (!MGC_OK_INDEX(nid >= 0 && nid < a.n)) continue;
        const int32_t lfn = a.last_fired[nid];
        for (int64_t k = a.row_ptr[nid] + lane; k < a.row_ptr[nid + 1]; k += 32) {
            if (a.plastic && !a.plastic[k]) continue;
            const uint2 e = a.syn[k];
            if (!MGC_OK_INDEX(k < a.n_syn && (e.x & a.tmask) < (uint32_t)a.n)) continue;
            const int32_t dt = lfn - a.last_fired[e.x & a.tmask];
            a.syn[k].y = as_u(stdp_weight(dt, as_f(e.y), a.P));
        }
        for (int64_t q = a.dend_off[nid] + lane; q < a.dend_off[nid + 1]; q += 32) {
            const int64_t k = a.dend_pos[q];
            if (!MGC_OK_INDEX(k >= 0 && k < a.n_syn && a.csr_src[k] >= 0 && a.csr_src[k] < a.n)) continue;
            if (a.plastic && !a.plastic[k]) continue;
            const int32_t dt = a.last_fired[a.csr_src[k]] - lfn;
            a.syn[k].y = as_u(stdp_weight(dt, as_f(a.syn[k].y), a.P));
        }
    }
    if (last_block(a.done)) step_epilogue(a);
}

StepKernel neuron_kernel(const mgc_sim* s) { return s->a.fx ? k_neuron<true> : k_neuron<false>; }
StepKernel deliver_kernel(const mgc_sim* s) { return s->a.fx ? k_deliver<true> : k_deliver<false>; }
StepKernel push_kernel(const mgc_sim* s) { return s->a.fx ? k_push<true> : k_push<false>; }
StepKernel pull_kernel(const mgc_sim*) { return k_pull; }
StepKernel stdp_kernel(const mgc_sim*) { return k_stdp; }

}  // namespace mgc
