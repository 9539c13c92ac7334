// Learned step scheduler: a per-group trace of spikes and delivered events,
// a small MLP that predicts the next group's load from the last groups, and
// the device-side choice between the two instantiations of the fused step
// kernel (compiled for 2 or 3 resident blocks per SM) through a conditional
// SWITCH node of the step-group graph.  The choice changes no arithmetic:
// both variants run the same code on the same data.
//
// No reference counterpart: the reference launches a fixed schedule
// (mgcore.cu:535-554).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"
#include "philox.cuh"
#include "sched_state.h"

namespace mgc {

__device__ __forceinline__ int choose_variant(const SchedState& st, float events_per_step)
{
    return events_per_step > st.threshold ? st.hi_variant : 1 - st.hi_variant;
}

// One warp: aggregates the trace of the steps since the previous decision,
// scores that decision, decides the variant of the next group and sets the
// graph's conditional handle.
__global__ void k_sched_decide(StepArgs a, SchedState* st, float* data, cudaGraphConditionalHandle handle,
                               int32_t set_handle)
{
    const int lane = threadIdx.x;
    const int64_t s0 = *a.step;
    const int64_t since = s0 - st->last_s0;
    const int64_t n = since < kTraceSteps ? since : kTraceSteps;
    float f[kTraceCols];
#pragma unroll
    for (int c = 0; c < kTraceCols; ++c) {
        float sum = 0.f;
        for (int64_t r = lane; r < n; r += 32)
            sum += a.trace[((s0 - n + r) & (kTraceSteps - 1)) * kTraceCols + c];
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        f[c] = n > 0 ? log1pf(sum / (float)n) : 0.f;
    }
    // learned: lane j computes hidden unit j of the MLP on the last
    // kGroupLag groups, the one that just ended included
    float pred_log = 0.f;
    const bool learn = st->mode == kSchedLearned && st->trained && st->n_hist + (n > 0) >= kGroupLag;
    __syncwarp();  // every lane has read the state before lane 0 changes it
    if (lane == 0 && n > 0) {
        // score the decision taken for the group that just ended
        if (st->have_prev) {
            const int best = choose_variant(*st, expm1f(f[kTracePops]));
            st->groups += 1;
            st->misses += best != st->prev_variant;
            if (st->mode == kSchedLearned && st->trained) {
                st->abs_log_err += fabs((double)st->prev_pred - (double)f[kTracePops]);
                st->err_groups += 1;
            }
        }
        for (int c = 0; c < kTraceCols; ++c) st->hist[st->hist_pos][c] = f[c];
        st->hist_pos = (st->hist_pos + 1) % kGroupHist;
        st->n_hist = min(st->n_hist + 1, kGroupHist);
        if (st->collect && st->n_data < kMaxDataset) {
            for (int c = 0; c < kTraceCols; ++c) data[(size_t)st->n_data * kTraceCols + c] = f[c];
            st->n_data += 1;
        }
    }
    __syncwarp();
    if (learn) {
        float z = st->p[mlp_b1() + lane];
        for (int g = 0; g < kGroupLag; ++g) {
            const int slot = (st->hist_pos - kGroupLag + g + 2 * kGroupHist) % kGroupHist;
            for (int c = 0; c < kTraceCols; ++c) {
                const int i = g * kTraceCols + c;
                const float x = (st->hist[slot][c] - st->xm[i]) / st->xs[i];
                z += st->p[mlp_w1() + lane * kMlpIn + i] * x;
            }
        }
        const float h = fmaxf(z, 0.f);
        float y = st->p[mlp_w2() + kTracePops * kMlpHidden + lane] * h;  // events output only
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        y += st->p[mlp_b2() + kTracePops];
        pred_log = y * st->ys[kTracePops] + st->ym[kTracePops];
    }
    if (lane == 0) {
        int v;
        if (st->forced_variant >= 0) {
            v = st->forced_variant;
        } else if (st->mode == kSchedThreshold && st->n_hist > 0) {
            const int last = (st->hist_pos + kGroupHist - 1) % kGroupHist;
            v = choose_variant(*st, expm1f(st->hist[last][kTracePops]));
        } else if (learn) {
            v = choose_variant(*st, expm1f(pred_log));
            st->prev_pred = pred_log;
        } else {
            v = st->static_variant;
        }
        st->have_prev = st->forced_variant < 0 && (st->mode == kSchedThreshold || learn);
        st->prev_variant = v;
        st->variant_groups[v] += 1;
        st->last_s0 = s0;
        if (set_handle) cudaGraphSetConditional(handle, (unsigned int)v);
    }
}

// ---------------------------------------------------------------------------
// MLP training: forward, backward and Adam in one block, deterministic
// (fixed summation order; minibatches follow a seeded affine permutation).
// ---------------------------------------------------------------------------

// Gradient of L = (1/nb) sum_b sum_o (y_bo - t_bo)^2 / 2 over the samples
// rows[0..nb) of X/Y, accumulated into g (zeroed by the caller).  z: [nb][H]
// scratch, dy: [nb][OUT], se: [nb*OUT] squared errors.  blockDim.x threads.
__device__ void mlp_batch_grad(const float* p, const float* X, const float* Y, const int* rows, int nb, float* g,
                               float* z, float* dy, float* se)
{
    const int t0 = threadIdx.x, nt = blockDim.x;
    for (int k = t0; k < nb * kMlpHidden; k += nt) {
        const int b = k / kMlpHidden, j = k % kMlpHidden;
        const float* x = X + (size_t)rows[b] * kMlpIn;
        float acc = p[mlp_b1() + j];
        for (int i = 0; i < kMlpIn; ++i) acc += p[mlp_w1() + j * kMlpIn + i] * x[i];
        z[k] = acc;
    }
    __syncthreads();
    for (int k = t0; k < nb * kMlpOut; k += nt) {
        const int b = k / kMlpOut, o = k % kMlpOut;
        float y = p[mlp_b2() + o];
        for (int j = 0; j < kMlpHidden; ++j) y += p[mlp_w2() + o * kMlpHidden + j] * fmaxf(z[b * kMlpHidden + j], 0.f);
        const float d = y - Y[(size_t)rows[b] * kMlpOut + o];
        dy[k] = d / (float)nb;
        se[k] = 0.5f * d * d / (float)nb;
    }
    __syncthreads();
    for (int k = t0; k < kMlpOut * kMlpHidden; k += nt) {
        const int o = k / kMlpHidden, j = k % kMlpHidden;
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc += dy[b * kMlpOut + o] * fmaxf(z[b * kMlpHidden + j], 0.f);
        g[mlp_w2() + k] += acc;
    }
    for (int o = t0; o < kMlpOut; o += nt) {
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc += dy[b * kMlpOut + o];
        g[mlp_b2() + o] += acc;
    }
    __syncthreads();
    // z becomes dL/dz (the ReLU mask taken from z itself)
    for (int k = t0; k < nb * kMlpHidden; k += nt) {
        const int b = k / kMlpHidden, j = k % kMlpHidden;
        float acc = 0.f;
        for (int o = 0; o < kMlpOut; ++o) acc += p[mlp_w2() + o * kMlpHidden + j] * dy[b * kMlpOut + o];
        z[k] = z[k] > 0.f ? acc : 0.f;
    }
    __syncthreads();
    for (int k = t0; k < kMlpHidden * kMlpIn; k += nt) {
        const int j = k / kMlpIn, i = k % kMlpIn;
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc += z[b * kMlpHidden + j] * X[(size_t)rows[b] * kMlpIn + i];
        g[mlp_w1() + k] += acc;
    }
    for (int j = t0; j < kMlpHidden; j += nt) {
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc += z[b * kMlpHidden + j];
        g[mlp_b1() + j] += acc;
    }
    __syncthreads();
}

// Full-batch loss and gradient at `params` (n <= kMaxGradSamples samples).
__global__ void k_mlp_gradient(const float* params, const float* X, const float* Y, int n, float* grad, float* loss)
{
    __shared__ float p[kMlpParams], g[kMlpParams];
    __shared__ float z[kMaxGradSamples * kMlpHidden], dy[kMaxGradSamples * kMlpOut], se[kMaxGradSamples * kMlpOut];
    __shared__ int rows[kMaxGradSamples];
    for (int k = threadIdx.x; k < kMlpParams; k += blockDim.x) {
        p[k] = params[k];
        g[k] = 0.f;
    }
    for (int b = threadIdx.x; b < n; b += blockDim.x) rows[b] = b;
    __syncthreads();
    mlp_batch_grad(p, X, Y, rows, n, g, z, dy, se);
    for (int k = threadIdx.x; k < kMlpParams; k += blockDim.x) grad[k] = g[k];
    if (threadIdx.x == 0) {
        float l = 0.f;
        for (int k = 0; k < n * kMlpOut; ++k) l += se[k];
        *loss = l;
    }
}

// `epochs` passes of Adam over n samples in minibatches of kTrainBatch;
// params (and Adam moments, zero at the start) live in shared memory and are
// written back to st->p at the end.  loss_out: mean loss of the last epoch.
__global__ void k_mlp_train(SchedState* st, const float* X, const float* Y, int n, int epochs, float lr, uint64_t seed,
                            float* loss_out)
{
    __shared__ float p[kMlpParams], g[kMlpParams], m1[kMlpParams], m2[kMlpParams];
    __shared__ float z[kTrainBatch * kMlpHidden], dy[kTrainBatch * kMlpOut], se[kTrainBatch * kMlpOut];
    __shared__ int rows[kTrainBatch];
    __shared__ uint32_t perm_a, perm_c;
    __shared__ float epoch_loss;
    for (int k = threadIdx.x; k < kMlpParams; k += blockDim.x) {
        p[k] = st->p[k];
        m1[k] = m2[k] = 0.f;
    }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float b1t = 1.f, b2t = 1.f;
    for (int e = 0; e < epochs; ++e) {
        if (threadIdx.x == 0) {
            // permutation r -> (a*r + c) mod n with a coprime to n
            const U32x4 r = philox4x32_10((uint32_t)e, 0u, 0u, 0x4D4C5054u /* "MLPT" */, (uint32_t)seed,
                                          (uint32_t)(seed >> 32));
            uint32_t a = (r.x % (uint32_t)n) | 1u;
            auto gcd = [](uint32_t x, uint32_t y) {
                while (y) {
                    const uint32_t t = x % y;
                    x = y;
                    y = t;
                }
                return x;
            };
            while (gcd(a, (uint32_t)n) != 1u) a += 2u;
            perm_a = a % (uint32_t)n;
            perm_c = r.y % (uint32_t)n;
            epoch_loss = 0.f;
        }
        __syncthreads();
        for (int b0 = 0; b0 < n; b0 += kTrainBatch) {
            const int nb = min(kTrainBatch, n - b0);
            for (int b = threadIdx.x; b < nb; b += blockDim.x)
                rows[b] = (int)(((uint64_t)perm_a * (uint64_t)(b0 + b) + perm_c) % (uint64_t)n);
            for (int k = threadIdx.x; k < kMlpParams; k += blockDim.x) g[k] = 0.f;
            __syncthreads();
            mlp_batch_grad(p, X, Y, rows, nb, g, z, dy, se);
            if (threadIdx.x == 0) {
                float l = 0.f;
                for (int k = 0; k < nb * kMlpOut; ++k) l += se[k];
                epoch_loss += l * (float)nb / (float)n;
            }
            b1t *= b1;
            b2t *= b2;
            for (int k = threadIdx.x; k < kMlpParams; k += blockDim.x) {
                m1[k] = b1 * m1[k] + (1.f - b1) * g[k];
                m2[k] = b2 * m2[k] + (1.f - b2) * g[k] * g[k];
                const float mh = m1[k] / (1.f - b1t), vh = m2[k] / (1.f - b2t);
                p[k] -= lr * mh / (sqrtf(vh) + eps);
            }
            __syncthreads();
        }
    }
    for (int k = threadIdx.x; k < kMlpParams; k += blockDim.x) st->p[k] = p[k];
    if (threadIdx.x == 0) *loss_out = epoch_loss;
}

}  // namespace mgc
