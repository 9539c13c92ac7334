// CSR row offsets of a device-resident synapse list without any allocation.
#include <cub/cub.cuh>

#include <mutex>

#include "sim.h"

using namespace mgc;

// ---------------------------------------------------------------------------
// CSR row offsets of a device-resident synapse list without any allocation:
// the scan's scratch is a fixed static device array.

namespace {

constexpr int kRoThreads = 256;
constexpr int kRoPerThread = 16;
constexpr int64_t kRoTile = kRoThreads * kRoPerThread;        // offsets scanned per block
constexpr int64_t kRoMaxTiles = 32768;                        // 256 KB of tile sums
constexpr int64_t kRoMaxNeurons = kRoMaxTiles * kRoTile - 1;  // 134,217,727
constexpr int kRoMaxDevices = 64;

// [0, kRoMaxTiles): tile sums, scanned in place into tile offsets;
// [kRoMaxTiles]: number of synapses whose source is out of range.
__device__ __align__(256) unsigned long long g_ro_scratch[kRoMaxTiles + 32];

std::mutex g_ro_mutex[kRoMaxDevices];              // one call per device at a time
unsigned long long* g_ro_addr[kRoMaxDevices] = {};  // scratch address on each device

__global__ void k_ro_count(const int32_t* src, int64_t S, int32_t n, unsigned long long* cnt,
                           unsigned long long* bad)
{
    GRID_STRIDE(k, S)
    {
        const int32_t v = src[k];
        if (v >= 0 && v < n) atomicAdd(cnt + v, 1ull);
        else atomicAdd(bad, 1ull);
    }
}

// Sum of each tile of kRoTile entries.
__global__ void __launch_bounds__(kRoThreads) k_ro_tile_sums(const unsigned long long* v, int64_t count,
                                                             unsigned long long* tile_sum)
{
    typedef cub::BlockReduce<unsigned long long, kRoThreads> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    const int64_t base = blockIdx.x * kRoTile;
    unsigned long long s = 0;
    for (int j = 0; j < kRoPerThread; ++j) {
        const int64_t i = base + (int64_t)j * kRoThreads + threadIdx.x;
        if (i < count) s += v[i];
    }
    s = Reduce(tmp).Sum(s);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = s;
}

// Exclusive scan of the tile sums in place (one block of 1024 threads).
__global__ void __launch_bounds__(1024) k_ro_scan_tiles(unsigned long long* t, int64_t tiles)
{
    typedef cub::BlockScan<unsigned long long, 1024> Scan;
    __shared__ typename Scan::TempStorage tmp;
    const int64_t per = (tiles + 1023) / 1024;
    const int64_t lo = threadIdx.x * per, hi = min(lo + per, tiles);
    unsigned long long s = 0;
    for (int64_t i = lo; i < hi; ++i) s += t[i];
    unsigned long long pre;
    Scan(tmp).ExclusiveSum(s, pre);
    for (int64_t i = lo; i < hi; ++i) {
        const unsigned long long x = t[i];
        t[i] = pre;
        pre += x;
    }
}

// Exclusive scan of each tile in place, plus the tile's offset.
__global__ void __launch_bounds__(kRoThreads) k_ro_apply(unsigned long long* v, int64_t count,
                                                         const unsigned long long* tile_off)
{
    typedef cub::BlockScan<unsigned long long, kRoThreads> Scan;
    __shared__ typename Scan::TempStorage tmp;
    const int64_t base = blockIdx.x * kRoTile + (int64_t)threadIdx.x * kRoPerThread;
    unsigned long long x[kRoPerThread];
    unsigned long long s = 0;
#pragma unroll
    for (int j = 0; j < kRoPerThread; ++j) {
        x[j] = base + j < count ? v[base + j] : 0ull;
        s += x[j];
    }
    unsigned long long pre;
    Scan(tmp).ExclusiveSum(s, pre);
    pre += tile_off[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kRoPerThread; ++j) {
        if (base + j < count) v[base + j] = pre;
        pre += x[j];
    }
}

}  // namespace

extern "C" mgc_status mgc_row_offsets_static(const int32_t* src, int64_t n_synapses, int32_t n_neurons,
                                             int64_t* row_ptr, void* stream)
{
    if (n_neurons < 0 || n_synapses < 0 || !row_ptr || (n_synapses > 0 && !src))
        return fail(MGC_ERR_INVALID, "mgc_row_offsets_static: bad arguments");
    if (n_neurons > kRoMaxNeurons)
        return fail(MGC_ERR_INVALID,
                    "mgc_row_offsets_static: %d neurons exceed the static scratch limit of %lld neurons",
                    n_neurons, (long long)kRoMaxNeurons);
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kRoMaxDevices)
        return fail(MGC_ERR_INVALID, "mgc_row_offsets_static: device %d beyond the %d supported", dev,
                    kRoMaxDevices);
    // Calls on one device share its scratch array: hold the device's lock
    // until this call's work has finished.
    std::lock_guard<std::mutex> lock(g_ro_mutex[dev]);
    if (!g_ro_addr[dev]) CK(cudaGetSymbolAddress(reinterpret_cast<void**>(&g_ro_addr[dev]), g_ro_scratch));
    unsigned long long* scratch = g_ro_addr[dev];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t count = (int64_t)n_neurons + 1;
    const int64_t tiles = (count + kRoTile - 1) / kRoTile;
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(row_ptr);
    unsigned long long* bad = scratch + kRoMaxTiles;
    unsigned long long nbad = 0;
    // Once the first operation is enqueued, every exit waits for the stream
    // (whatever that wait returns) before the lock is released, so that no
    // work of this call can still write the shared scratch array when the
    // next call on this device starts.
    const mgc_status rc = [&]() -> mgc_status {
        // must start at zero: the row counts (kept in row_ptr) and the bad-source count
        CK(cudaMemsetAsync(cnt, 0, sizeof(int64_t) * count, st));
        CK(cudaMemsetAsync(bad, 0, sizeof(unsigned long long), st));
        if (n_synapses) k_ro_count<<<grid_for(n_synapses), 256, 0, st>>>(src, n_synapses, n_neurons, cnt, bad);
        k_ro_tile_sums<<<(unsigned)tiles, kRoThreads, 0, st>>>(cnt, count, scratch);
        k_ro_scan_tiles<<<1, 1024, 0, st>>>(scratch, tiles);
        k_ro_apply<<<(unsigned)tiles, kRoThreads, 0, st>>>(cnt, count, scratch);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return MGC_OK;
    }();
    if (rc != MGC_OK) {
        cudaStreamSynchronize(st);
        return rc;
    }
    if (nbad)
        return fail(MGC_ERR_INVALID, "mgc_row_offsets_static: %llu synapse sources outside [0, %d)", nbad,
                    n_neurons);
    return MGC_OK;
}

