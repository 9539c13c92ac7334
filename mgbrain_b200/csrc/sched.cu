// The step scheduler's entry points: mode, threshold, calibration, training
// of its MLP on the GPU, reports; its kernels are in sched.cuh.
#include <cmath>

#include "sched.cuh"
#include "sim.h"

using namespace mgc;

namespace mgc {
const void* sched_decide_kernel() { return (const void*)k_sched_decide; }
}  // namespace mgc

extern "C" {

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


}  // extern "C"
