// Scheduler state and MLP shape shared by the host side of the library and
// the scheduler's kernels (sched.cuh).  No reference counterpart: the
// reference launches a fixed schedule (mgcore.cu:535-554).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"

namespace mgc {

constexpr int kGroupLag = 4;                       // groups of history the MLP sees
constexpr int kMlpIn = kGroupLag * kTraceCols;     // 20
constexpr int kMlpHidden = 32;
constexpr int kMlpOut = kTraceCols;                // next group: per-population spikes, events
constexpr int kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + kMlpOut * kMlpHidden + kMlpOut;
constexpr int kGroupHist = 16;
constexpr int kMaxDataset = 16384;                 // group feature rows kept for training
constexpr int kTrainBatch = 64;
constexpr int kMaxGradSamples = 128;

enum : int32_t { kSchedStatic = 0, kSchedThreshold = 1, kSchedLearned = 2 };

// Scheduler state in device memory (one per handle).  Feature of a group:
// log1p of the per-step mean of each trace column over the group's steps.
struct SchedState {
    int32_t mode;
    int32_t static_variant;
    int32_t forced_variant;   // >= 0: every group runs it (calibration)
    int32_t collect;          // append group features to the dataset
    float threshold;          // events per step where the better variant changes
    int32_t hi_variant;       // variant chosen above the threshold
    int32_t trained;
    int64_t last_s0;          // step at the previous decision
    int32_t have_prev;        // the previous decision awaits evaluation
    int32_t prev_variant;
    float prev_pred;          // learned: predicted log1p(events/step) of the running group
    int32_t n_hist;
    int32_t hist_pos;
    int32_t n_data;
    int64_t groups;           // evaluated decisions
    int64_t misses;           // decisions that differ from the threshold on the actual load
    int64_t variant_groups[2];
    double abs_log_err;       // learned: sum |predicted - actual| of log1p(events/step)
    int64_t err_groups;
    float hist[kGroupHist][kTraceCols];
    // MLP: y = W2 relu(W1 x + b1) + b2 on standardized x and y
    float p[kMlpParams];
    float xm[kMlpIn], xs[kMlpIn], ym[kMlpOut], ys[kMlpOut];
};

// Parameter blocks inside a flat parameter vector.
__host__ __device__ constexpr int mlp_w1() { return 0; }
__host__ __device__ constexpr int mlp_b1() { return kMlpHidden * kMlpIn; }
__host__ __device__ constexpr int mlp_w2() { return mlp_b1() + kMlpHidden; }
__host__ __device__ constexpr int mlp_b2() { return mlp_w2() + kMlpOut * kMlpHidden; }

}  // namespace mgc
