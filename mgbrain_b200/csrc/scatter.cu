// The ceilings of event delivery on a device: scattered fp32 reductions fed
// by streamed 8-byte event records, and a plain stream of the same records.
#include "sim.h"

using namespace mgc;

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

