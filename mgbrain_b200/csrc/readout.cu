// Readout: the raster (read, or staged on the device and collected), neuron
// state, weights, the CSR, partition statistics and handle information.
#include <memory>
#include <thread>

#include "sim.h"

using namespace mgc;

namespace {

constexpr int32_t kRasterBits = kStatusRasterIds | kStatusRasterSteps;

// ns steps' counts c32 and their ni ids hid (step after step) into the
// caller's arrays, each step's ids sorted, the steps split over host threads.
mgc_status finish_raster(int64_t step0, int64_t ns, int64_t ni, const int32_t* c32, int32_t* hid, bool truncated,
                         int32_t status, int64_t* first_step, int64_t* counts, int64_t counts_cap, int32_t* ids,
                         int64_t ids_cap, int64_t* n_steps, int64_t* n_ids)
{
    truncated = truncated || ns > counts_cap || ni > ids_cap;
    std::vector<int64_t> off(ns + 1, 0);
    for (int64_t i = 0; i < ns; ++i) {
        off[i + 1] = off[i] + c32[i];
        if (counts && i < counts_cap) counts[i] = c32[i];
    }
    auto sort_steps = [&](int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; ++i)
            if (off[i + 1] <= ni) std::sort(hid + off[i], hid + off[i + 1]);
    };
    const int64_t nt = std::min<int64_t>(std::max(1u, std::thread::hardware_concurrency()), 16);
    if (ni > (1 << 16) && ns > 1 && nt > 1) {
        std::vector<std::thread> pool;
        for (int64_t t = 0; t < nt; ++t) pool.emplace_back(sort_steps, ns * t / nt, ns * (t + 1) / nt);
        for (auto& th : pool) th.join();
    } else {
        sort_steps(0, ns);
    }
    if (ids && hid != ids) memcpy(ids, hid, 4 * std::min(ni, ids_cap));
    if (first_step) *first_step = step0;
    if (n_steps) *n_steps = std::min(ns, counts_cap);
    if (n_ids) *n_ids = std::min(ni, ids_cap);
    if (truncated) return fail(MGC_ERR_OVERFLOW, "raster truncated (device status %d)", status);
    return MGC_OK;
}

// The raster so far into a stage (block-strided copies), then the clock of
// the next raster (k_raster_restart, after every block has read).
__global__ void k_raster_stage(StepArgs a, int32_t* ids, int32_t* counts, int64_t steps_cap, int64_t ids_cap)
{
    const int64_t ns = min(*a.step - *a.raster_step0, steps_cap);
    const int64_t ni = min(*a.raster_pos, ids_cap);
    GRID_STRIDE(i, ns) counts[i] = a.raster_counts[i];
    GRID_STRIDE(i, ni) ids[i] = a.raster_ids[i];
}

__global__ void k_raster_restart(StepArgs a, int64_t* meta, int64_t steps_cap, int64_t ids_cap)
{
    const int64_t step = *a.step, step0 = *a.raster_step0;
    meta[0] = step0;
    meta[1] = min(step - step0, steps_cap);
    meta[2] = min(*a.raster_pos, ids_cap);
    meta[3] = *a.status & kRasterBits;
    *a.raster_step0 = step;
    *a.raster_pos = 0;
    atomicAnd(a.status, ~kRasterBits);
}

}  // namespace

extern "C" {

mgc_status mgc_read_raster(mgc_sim* s, int64_t* first_step, int64_t* counts, int64_t counts_cap, int32_t* ids,
                           int64_t ids_cap, int64_t* n_steps, int64_t* n_ids)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    if (!s->a.record) return fail(MGC_ERR_INVALID, "raster recording is off for this handle");
    if (s->staged) return fail(MGC_ERR_INVALID, "collect the staged rasters first (mgc_raster_collect)");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    int64_t step = 0, step0 = 0, pos = 0;
    int32_t status = 0;
    CK(cudaMemcpy(&step, s->a.step, 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&step0, s->a.raster_step0, 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&pos, s->a.raster_pos, 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&status, s->a.status, 4, cudaMemcpyDeviceToHost));
    const int64_t ns = std::min(step - step0, s->raster_steps_cap);
    const int64_t ni = std::min(pos, s->raster_ids_cap);
    std::vector<int32_t> c32(ns);
    if (ns) CK(cudaMemcpy(c32.data(), s->a.raster_counts, 4 * ns, cudaMemcpyDeviceToHost));
    // the ids land in the caller's buffer when it holds them all (else in a
    // staging buffer)
    std::unique_ptr<int32_t[]> staging;
    int32_t* hid = ids;
    if (!ids || ids_cap < ni) {
        staging.reset(new int32_t[std::max<int64_t>(ni, 1)]);
        hid = staging.get();
    }
    if (ni) CK(cudaMemcpy(hid, s->a.raster_ids, 4 * ni, cudaMemcpyDeviceToHost));
    // the next raster starts here; only the raster's status bits are cleared
    const int64_t zero = 0;
    const int32_t kept = status & ~kRasterBits;
    CK(cudaMemcpy(s->a.raster_step0, &step, 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->a.raster_pos, &zero, 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->a.status, &kept, 4, cudaMemcpyHostToDevice));
    return finish_raster(step0, ns, ni, c32.data(), hid, (status & kRasterBits) != 0, status, first_step, counts,
                         counts_cap, ids, ids_cap, n_steps, n_ids);
}

mgc_status mgc_raster_stage(mgc_sim* s)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    if (!s->a.record) return fail(MGC_ERR_INVALID, "raster recording is off for this handle");
    if (s->staged == 2) return fail(MGC_ERR_INVALID, "two rasters are staged already: collect one first");
    CK(cudaSetDevice(s->device));
    mgc_sim::RasterStage& g = s->stages[(s->stage_head + s->staged) & 1];
    if (!g.ids) {
        CKS(s->alloc(&g.ids, (size_t)s->raster_ids_cap, false));
        CKS(s->alloc(&g.counts, (size_t)s->raster_steps_cap, false));
        CKS(s->alloc(&g.meta, 4));
        CK(cudaEventCreateWithFlags(&g.ev, cudaEventDisableTiming));
    }
    if (!s->copy_stream) CK(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
    k_raster_stage<<<grid_for(s->raster_ids_cap), 256, 0, s->stream>>>(s->a, g.ids, g.counts, s->raster_steps_cap,
                                                                        s->raster_ids_cap);
    k_raster_restart<<<1, 1, 0, s->stream>>>(s->a, g.meta, s->raster_steps_cap, s->raster_ids_cap);
    CK(cudaGetLastError());
    CK(cudaEventRecord(g.ev, s->stream));
    s->launches += 2;
    s->staged += 1;
    return MGC_OK;
}

mgc_status mgc_raster_collect(mgc_sim* s, int64_t* first_step, int64_t* counts, int64_t counts_cap, int32_t* ids,
                              int64_t ids_cap, int64_t* n_steps, int64_t* n_ids)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    if (!s->staged) return fail(MGC_ERR_INVALID, "no raster is staged (mgc_raster_stage)");
    CK(cudaSetDevice(s->device));
    mgc_sim::RasterStage& g = s->stages[s->stage_head];
    // the stage's copies are done; the steps enqueued after it keep running
    CK(cudaStreamWaitEvent(s->copy_stream, g.ev, 0));
    int64_t meta[4];
    CK(cudaMemcpyAsync(meta, g.meta, sizeof(meta), cudaMemcpyDeviceToHost, s->copy_stream));
    CK(cudaStreamSynchronize(s->copy_stream));
    const int64_t step0 = meta[0], ns = meta[1], ni = meta[2];
    const int32_t status = (int32_t)meta[3];
    std::vector<int32_t> c32(ns);
    std::unique_ptr<int32_t[]> staging;
    int32_t* hid = ids;
    if (!ids || ids_cap < ni) {
        staging.reset(new int32_t[std::max<int64_t>(ni, 1)]);
        hid = staging.get();
    }
    if (ns) CK(cudaMemcpyAsync(c32.data(), g.counts, 4 * ns, cudaMemcpyDeviceToHost, s->copy_stream));
    if (ni) CK(cudaMemcpyAsync(hid, g.ids, 4 * ni, cudaMemcpyDeviceToHost, s->copy_stream));
    CK(cudaStreamSynchronize(s->copy_stream));
    s->stage_head ^= 1;
    s->staged -= 1;
    return finish_raster(step0, ns, ni, c32.data(), hid, status != 0, status, first_step, counts, counts_cap, ids,
                         ids_cap, n_steps, n_ids);
}

mgc_status mgc_read_state(mgc_sim* s, float* v, float* i_exc, float* i_inh, int32_t* refrac, int32_t* last_fired,
                          int32_t* fire_cnt)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    const size_t n = s->n;
    if (v) {
        CK(cudaMemcpy(v, s->a.V, 4 * n, cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < s->pois_idx.size(); ++k) v[s->pois_idx[k]] = s->pois_v[k];
    }
    if (i_exc) CK(cudaMemcpy(i_exc, s->a.Iexc, 4 * n, cudaMemcpyDeviceToHost));
    if (i_inh) CK(cudaMemcpy(i_inh, s->a.Iinh, 4 * n, cudaMemcpyDeviceToHost));
    if (refrac) CK(cudaMemcpy(refrac, s->a.refrac, 4 * n, cudaMemcpyDeviceToHost));
    if (last_fired) CK(cudaMemcpy(last_fired, s->a.last_fired, 4 * n, cudaMemcpyDeviceToHost));
    if (fire_cnt) CK(cudaMemcpy(fire_cnt, s->a.fire_cnt, 4 * n, cudaMemcpyDeviceToHost));
    return MGC_OK;
}

mgc_status mgc_read_weights(mgc_sim* s, float* weight)
{
    if (!s || !weight) return fail(MGC_ERR_INVALID, "null argument");
    if (!s->csr_syn64) return fail(MGC_ERR_INVALID, "procedural networks have no synapse-list order");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    std::vector<uint2> syn(s->S);
    std::vector<int64_t> idx(s->S);
    // the pull method keeps the live weights in its incoming rows
    const uint2* src_words = s->a.pull ? s->a.in_ent : s->a.syn;
    const int64_t* src_idx = s->a.pull ? s->in_syn64 : s->csr_syn64;
    if (s->S) {
        CK(cudaMemcpy(syn.data(), src_words, 8 * s->S, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(idx.data(), src_idx, 8 * s->S, cudaMemcpyDeviceToHost));
    }
    for (int64_t p = 0; p < s->S; ++p) memcpy(&weight[idx[p]], &syn[p].y, 4);
    return MGC_OK;
}

mgc_status mgc_export_csr(mgc_sim* s, int64_t* row_ptr, int32_t* tgt, float* weight, int32_t* delay)
{
    if (!s) return fail(MGC_ERR_INVALID, "null handle");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    if (row_ptr) CK(cudaMemcpy(row_ptr, s->a.row_ptr, 8 * ((size_t)s->n_src + 1), cudaMemcpyDeviceToHost));
    if (tgt || weight || delay) {
        // in pieces, so a large CSR needs no second full-size host copy
        const int64_t piece = int64_t(1) << 24;
        std::vector<uint2> buf((size_t)std::min<int64_t>(piece, std::max<int64_t>(s->S, 1)));
        for (int64_t p0 = 0; p0 < s->S; p0 += piece) {
            const int64_t c = std::min(piece, s->S - p0);
            CK(cudaMemcpy(buf.data(), s->a.syn + p0, 8 * c, cudaMemcpyDeviceToHost));
            for (int64_t q = 0; q < c; ++q) {
                if (tgt) tgt[p0 + q] = (int32_t)(buf[q].x & s->a.tmask);
                if (delay) delay[p0 + q] = (int32_t)(buf[q].x >> s->a.tbits);
                if (weight) memcpy(&weight[p0 + q], &buf[q].y, 4);
            }
        }
    }
    return MGC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Partition statistics on the device: one warp per source row of the CSR,
// the zones' counters in shared memory, flushed once per block.
// ---------------------------------------------------------------------------
namespace {

constexpr int kMaxZones = 4096;

__global__ void k_partition_stats(const int64_t* row_ptr, const uint2* syn, int32_t n_src, uint32_t tmask,
                                  int32_t tar_base, const int32_t* part, int32_t nparts, unsigned long long* out)
{
    extern __shared__ unsigned int zc[];  // [3][nparts]: syn by source zone, out by source zone, in by target zone
    for (int z = threadIdx.x; z < 3 * nparts; z += blockDim.x) zc[z] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t src = warp; src < n_src; src += nwarps) {
        const int64_t b = row_ptr[src], e = row_ptr[src + 1];
        if (e == b) continue;
        const int32_t zs = part[src];
        unsigned int crossing = 0;
        for (int64_t q = b + lane; q < e; q += 32) {
            const int32_t zt = part[(int32_t)(syn[q].x & tmask) + tar_base];
            if (zt != zs) {
                ++crossing;
                atomicAdd(&zc[2 * nparts + zt], 1u);
            }
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) crossing += __shfl_xor_sync(0xffffffffu, crossing, o);
        if (lane == 0) {
            atomicAdd(&zc[zs], (unsigned int)(e - b));
            atomicAdd(&zc[nparts + zs], crossing);
        }
    }
    __syncthreads();
    for (int z = threadIdx.x; z < 3 * nparts; z += blockDim.x)
        if (zc[z]) atomicAdd(out + z, (unsigned long long)zc[z]);
}

}  // namespace

extern "C" {

mgc_status mgc_partition_stats(mgc_sim* s, const int32_t* part, int32_t nparts, int64_t* cut, int64_t* zone_neurons,
                               int64_t* zone_syn, int64_t* zone_out, int64_t* zone_in)
{
    if (!s || !part) return fail(MGC_ERR_INVALID, "null argument");
    if (nparts < 1 || nparts > kMaxZones) return fail(MGC_ERR_INVALID, "1..%d zones (got %d)", kMaxZones, nparts);
    const int32_t n = s->n_src;
    std::vector<int64_t> zn(nparts, 0);
    for (int32_t i = 0; i < n; ++i) {
        if (part[i] < 0 || part[i] >= nparts)
            return fail(MGC_ERR_INVALID, "neuron %d in zone %d, outside 0..%d", i, part[i], nparts - 1);
        zn[part[i]] += 1;
    }
    CK(cudaSetDevice(s->device));
    DevTmp tp, to;
    int32_t* dpart;
    unsigned long long* dout;
    CKS(tmp_alloc(tp, &dpart, (size_t)n));
    CKS(tmp_alloc(to, &dout, 3 * (size_t)nparts));
    CK(cudaMemcpyAsync(dpart, part, 4 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemsetAsync(dout, 0, 8 * 3 * (size_t)nparts, s->stream));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, s->device));
    const size_t smem = 4 * 3 * (size_t)nparts;
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(k_partition_stats, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // a partition handle's targets are local ids; their zones are those of
    // the whole-network ids from its first neuron on
    k_partition_stats<<<prop.multiProcessorCount * 4, 256, smem, s->stream>>>(s->a.row_ptr, s->a.syn, n, s->a.tmask,
                                                                              s->a.src_base, dpart, nparts, dout);
    CK(cudaGetLastError());
    s->launches += 1;
    std::vector<unsigned long long> h(3 * (size_t)nparts);
    CK(cudaMemcpyAsync(h.data(), dout, 8 * h.size(), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    int64_t total_cut = 0;
    for (int32_t z = 0; z < nparts; ++z) {
        if (zone_neurons) zone_neurons[z] = zn[z];
        if (zone_syn) zone_syn[z] = (int64_t)h[z];
        if (zone_out) zone_out[z] = (int64_t)h[nparts + z];
        if (zone_in) zone_in[z] = (int64_t)h[2 * nparts + z];
        total_cut += (int64_t)h[nparts + z];
    }
    if (cut) *cut = total_cut;
    return MGC_OK;
}

mgc_status mgc_get_info(mgc_sim* s, mgc_info* info)
{
    if (!s || !info) return fail(MGC_ERR_INVALID, "null argument");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    memset(info, 0, sizeof(*info));
    info->n_neurons = s->n;
    info->ring_len = s->M;
    info->min_delay = s->dmin;
    info->max_delay = s->dmax;
    info->n_synapses = s->S;
    CK(cudaMemcpy(&info->step, s->a.step, 8, cudaMemcpyDeviceToHost));
    unsigned long long ev = 0;
    CK(cudaMemcpy(&ev, s->a.events, 8, cudaMemcpyDeviceToHost));
    info->events = (int64_t)ev;
    info->mode = s->mode;
    info->graph_steps = s->graph_steps ? s->graph_steps : kGraphSteps;
    info->device_bytes = (int64_t)s->bytes;
    info->persistent = s->a.deferred && !sched_wanted(s) ? s->persistent : 0;
    info->first_neuron = s->a.src_base;
    info->total_neurons = s->n_src;
    info->window = s->fused ? s->window : 0;
    info->accumulation = s->a.fx ? MGC_ACC_FIXED : MGC_ACC_FLOAT;
    info->fx_shift = s->fx_shift;
    return MGC_OK;
}


}  // extern "C"
