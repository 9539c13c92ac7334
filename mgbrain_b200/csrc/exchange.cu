// Spike exchange between the partitions of one network (one handle per
// partition), host-staged and device-resident forms.
#include "sim.h"

using namespace mgc;

// ---------------------------------------------------------------------------
// Spike exchange between partitions.  A partition handle's history holds the
// spike ids (whole-network ids) of every neuron; its own neuron update writes
// its neurons' spikes, and the other partitions' spikes of the steps run since
// the last exchange are appended after them.  Deliveries of step x read the
// spikes of steps <= x - min_delay, so exchanging every <= min_delay - 1 steps
// hands each partition every spike before it is delivered.
// ---------------------------------------------------------------------------
namespace {

// History slot of the step `back` steps before the device's current one.
__device__ __forceinline__ int32_t slot_back(const StepArgs& a, int32_t back)
{
    const int32_t h = a.slots[1] - back;
    return h < 0 ? h + a.H : h;
}

// Block j: the spikes of step (current - count + j) into counts[j] and, when
// they fit, into ids after those of the earlier steps.
__global__ void k_part_export(StepArgs a, int32_t count, int32_t* counts, int32_t* ids, int64_t cap)
{
    const int32_t j = blockIdx.x;
    int64_t off = 0;
    for (int32_t q = 0; q < j; ++q) off += a.hist_cnt[slot_back(a, count - q)];
    const int32_t hs = slot_back(a, count - j);
    const int32_t c = a.hist_cnt[hs];
    if (threadIdx.x == 0) counts[j] = c;
    if (!ids || off + c > cap) return;  // the host reports the overflow from the counts
    const int32_t* src = a.hist_ids + (size_t)hs * (size_t)a.n_src;
    for (int32_t i = threadIdx.x; i < c; i += blockDim.x) ids[off + i] = src[i];
}

// Block (j, r), r != self: rank r's spikes of step (current - count + j),
// stored from ids + r * stride after its spikes of the earlier steps, go
// after the slot's own spikes and those of the ranks before r.  Rank q's
// count of step j is cnt[q * cnt_stride + j].  A rank whose window holds
// more than cap ids (its buffer cut them), a negative count, an id outside
// the network or a slot that would hold more than every neuron sets
// kStatusExchange and the counts stay as they were (k_part_commit), so no
// delivery reads what was written.
__global__ void k_part_import(StepArgs a, int32_t count, int32_t nranks, int32_t self, const int32_t* cnt,
                              int64_t cnt_stride, const int32_t* ids, int64_t stride, int64_t cap)
{
    const int32_t j = blockIdx.x, r = blockIdx.y;
    int64_t src = (int64_t)r * stride, rank_total = 0;
    bool bad = false;
    for (int32_t q = 0; q < count; ++q) {
        const int32_t c = cnt[(size_t)r * cnt_stride + q];
        bad |= c < 0;
        rank_total += c;
        if (q < j) src += c;
    }
    if (r == self) {  // its own window cut short makes the others refuse: refuse here too
        if (threadIdx.x == 0 && rank_total > cap) atomicOr(a.status, kStatusExchange);
        return;
    }
    const int32_t hs = slot_back(a, count - j);
    const int64_t own = a.hist_cnt[hs];
    int64_t dst = own, total = own;
    for (int32_t q = 0; q < nranks; ++q) {
        if (q == self) continue;
        const int32_t c = cnt[(size_t)q * cnt_stride + j];
        if (q < r) dst += c;
        total += c;
    }
    if (bad || rank_total > cap || total > a.n_src) {
        if (threadIdx.x == 0) atomicOr(a.status, kStatusExchange);
        return;
    }
    const int32_t c = cnt[(size_t)r * cnt_stride + j];
    int32_t* out = a.hist_ids + (size_t)hs * (size_t)a.n_src;
    for (int32_t i = threadIdx.x; i < c; i += blockDim.x) {
        const int32_t id = ids[src + i];
        if (id < 0 || id >= a.n_src) {
            atomicOr(a.status, kStatusExchange);
            continue;
        }
        out[dst + i] = id;
    }
}

// The slots' counts grow by the imported spikes, unless the import failed.
__global__ void k_part_commit(StepArgs a, int32_t count, int32_t nranks, int32_t self, const int32_t* cnt,
                              int64_t cnt_stride)
{
    if (*(volatile int32_t*)a.status & kStatusExchange) return;
    for (int32_t j = threadIdx.x; j < count; j += blockDim.x) {
        int32_t add = 0;
        for (int32_t q = 0; q < nranks; ++q)
            if (q != self) add += cnt[(size_t)q * cnt_stride + j];
        a.hist_cnt[slot_back(a, count - j)] += add;
    }
}

mgc_status xch_reserve(mgc_sim* s, int64_t count)
{
    if (s->xch_cap >= count) return MGC_OK;
    CKS(s->alloc(&s->xch, (size_t)count));
    s->xch_cap = count;
    return MGC_OK;
}

// Kernels read and write the exchange buffers directly: device memory of the
// handle's device, managed memory, or page-locked host memory mapped into
// the device's address space.
bool device_accessible(const void* p, int device)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (at.type == cudaMemoryTypeDevice) return at.device == device;
    if (at.type == cudaMemoryTypeManaged) return true;
    if (at.type == cudaMemoryTypeHost) return at.devicePointer == p;
    return false;
}

mgc_status check_window(mgc_sim* s, int32_t count)
{
    if (!s->partition) return fail(MGC_ERR_INVALID, "not a partition handle");
    if (count < 1 || count != s->pending)
        return fail(MGC_ERR_INVALID, "exchange the %d steps run since the last import (got %d)", s->pending, count);
    return MGC_OK;
}

}  // namespace

extern "C" {

mgc_status mgc_part_export(mgc_sim* s, int32_t count, int32_t* counts, int32_t* ids, int64_t ids_cap, int64_t* total)
{
    if (!s || !counts || !total || ids_cap < 0) return fail(MGC_ERR_INVALID, "null argument");
    CKS(check_window(s, count));
    CK(cudaSetDevice(s->device));
    if (ids_cap > 0 && (!ids || !device_accessible(ids, s->device)))
        return fail(MGC_ERR_INVALID, "spike id buffer is not device memory of device %d", s->device);
    CKS(xch_reserve(s, count));
    k_part_export<<<count, 256, 0, s->stream>>>(s->a, count, s->xch, ids_cap > 0 ? ids : nullptr, ids_cap);
    CK(cudaGetLastError());
    s->launches += 1;
    CK(cudaMemcpyAsync(counts, s->xch, 4 * (size_t)count, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    int64_t sum = 0;
    for (int32_t j = 0; j < count; ++j) sum += counts[j];
    *total = sum;
    if (sum > ids_cap) return fail(MGC_ERR_OVERFLOW, "%lld spike ids to export, room for %lld", (long long)sum,
                                   (long long)ids_cap);
    return MGC_OK;
}

mgc_status mgc_part_import(mgc_sim* s, int32_t count, int32_t nranks, int32_t self, const int32_t* counts,
                           const int32_t* ids, int64_t stride)
{
    if (!s || !counts || nranks < 1 || self < 0 || self >= nranks || stride < 0)
        return fail(MGC_ERR_INVALID, "bad import arguments");
    CKS(check_window(s, count));
    bool any = false;
    for (int32_t r = 0; r < nranks; ++r) {
        int64_t sum = 0;
        for (int32_t j = 0; j < count; ++j) {
            const int32_t c = counts[(size_t)r * count + j];
            if (c < 0 || c > s->n_src) return fail(MGC_ERR_INVALID, "rank %d step %d: bad spike count %d", r, j, c);
            sum += c;
        }
        if (sum > stride) return fail(MGC_ERR_INVALID, "rank %d sends %lld ids in a stride of %lld", r,
                                      (long long)sum, (long long)stride);
        any |= r != self && sum > 0;
    }
    CK(cudaSetDevice(s->device));
    if (any && (!ids || !device_accessible(ids, s->device)))
        return fail(MGC_ERR_INVALID, "spike id buffer is not device memory of device %d", s->device);
    CKS(xch_reserve(s, (int64_t)nranks * count));
    CK(cudaMemcpyAsync(s->xch, counts, 4 * (size_t)nranks * count, cudaMemcpyHostToDevice, s->stream));
    if (any) {
        k_part_import<<<dim3(count, nranks), 256, 0, s->stream>>>(s->a, count, nranks, self, s->xch, count, ids,
                                                                   stride, stride);
        k_part_commit<<<1, 256, 0, s->stream>>>(s->a, count, nranks, self, s->xch, count);
        CK(cudaGetLastError());
        s->launches += 2;
    }
    CK(cudaStreamSynchronize(s->stream));  // the counts were staged from the caller's memory
    int32_t st = 0;
    CK(cudaMemcpy(&st, s->a.status, 4, cudaMemcpyDeviceToHost));
    if (st & kStatusExchange) return fail(MGC_ERR_INVALID, "an imported spike id was out of range (exchange refused)");
    s->pending = 0;
    return MGC_OK;
}

mgc_status mgc_part_export_dev(mgc_sim* s, int32_t count, int32_t* buf, int64_t cap)
{
    if (!s || !buf || cap < 0) return fail(MGC_ERR_INVALID, "bad export arguments");
    CKS(check_window(s, count));
    CK(cudaSetDevice(s->device));
    if (!device_accessible(buf, s->device))
        return fail(MGC_ERR_INVALID, "exchange buffer is not device memory of device %d", s->device);
    k_part_export<<<count, 256, 0, s->stream>>>(s->a, count, buf, buf + count, cap);
    CK(cudaGetLastError());
    s->launches += 1;
    return MGC_OK;
}

mgc_status mgc_part_import_dev(mgc_sim* s, int32_t count, int32_t nranks, int32_t self, const int32_t* bufs, int64_t cap)
{
    if (!s || nranks < 1 || self < 0 || self >= nranks || cap < 0) return fail(MGC_ERR_INVALID, "bad import arguments");
    CKS(check_window(s, count));
    CK(cudaSetDevice(s->device));
    if (nranks > 1) {
        if (!bufs || !device_accessible(bufs, s->device))
            return fail(MGC_ERR_INVALID, "exchange buffer is not device memory of device %d", s->device);
        const int64_t blk = count + cap;  // one rank's export: counts, then ids
        k_part_import<<<dim3(count, nranks), 256, 0, s->stream>>>(s->a, count, nranks, self, bufs, blk, bufs + count,
                                                                   blk, cap);
        k_part_commit<<<1, 256, 0, s->stream>>>(s->a, count, nranks, self, bufs, blk);
        CK(cudaGetLastError());
        s->launches += 2;
    }
    s->pending = 0;
    return MGC_OK;
}

}  // extern "C"
