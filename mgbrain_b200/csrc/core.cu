// Error reporting, device allocation with host-side fault injection, the
// step groups' wait self-test and the small entry points of the C ABI.
#include <cstdarg>
#include <cstdio>

#include "sim.h"

using namespace mgc;

namespace mgc {

static thread_local std::string g_last_error;

// Host-side fault injection (mgc_fault_inject_alloc): when positive, the
// device allocation that brings the count to zero fails as if the device
// were out of memory.
static std::atomic<int64_t> g_fail_alloc{0};

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


const char* last_error_text() { return g_last_error.c_str(); }

}  // namespace mgc

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

const char* mgc_last_error(void) { return last_error_text(); }

int64_t mgc_kernel_launches(mgc_sim* s) { return s ? s->launches : 0; }

}  // extern "C"
