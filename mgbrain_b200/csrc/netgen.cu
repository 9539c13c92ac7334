// Network generation on the device by NetGen's rules (include/mgc.h,
// mgc_create_generated): the synapse list NetGen::gen_net would make
// (src/model/netgen.cpp:39-229), generated in device memory in gen_net's
// order and handed to the CSR construction without a host copy.
//
// The fixed-probability rule (netgen.cpp:169-186) takes pair k of the
// row-major sn x tn pairs, while fewer than gen_num are taken, when the k-th
// output of NetGen's mt19937 modulo sn*tn is below gen_num * 1.1.  The k-th
// output depends on all before it, so the candidate pairs are cut into
// stretches of C pairs and each stretch starts from the generator jumped
// ahead by its first index (MGBrain::MtJump, computed on the host: jumps by
// C, 2C, 4C, ... from the stretches already placed).  A block runs one
// stretch: MT19937's block twist of 624 words in shared memory (three
// dependent phases of at most 227 independent words), then the 624 tempered
// outputs tested at once.  A first pass counts each stretch's taken pairs,
// the host turns the counts into offsets and finds the stretch that reaches
// gen_num, and a second pass writes each taken pair at its offset, in order
// (block scan of the taken flags of each round of outputs).
#include <cub/cub.cuh>

#include <cmath>
#include <memory>
#include <thread>

#include "mgbrain/mt19937.h"
#include "sim.h"

using namespace mgc;

namespace {

constexpr int kMtN = 624;
constexpr int kGenThreads = 256;
constexpr uint64_t kStretchMin = uint64_t(1) << 22;  // candidate pairs per stretch, at least

__device__ __forceinline__ uint32_t mt_next(uint32_t a, uint32_t b, uint32_t c)
{
    const uint32_t y = (a & 0x80000000u) | (b & 0x7fffffffu);
    return c ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}

__device__ __forceinline__ uint32_t mt_temper(uint32_t y)
{
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    return y ^ (y >> 18);
}

// One block twist of the 624 words x (shared memory): new[j] = next(old[j],
// old[j+1], old[j+397]) for j < 227; next(old[j], old[j+1], new[j-227]) for
// 227 <= j < 623; next(old[623], new[0], new[396]).  Three phases in order
// (each reads what the one before wrote); inside a phase every thread reads
// its inputs before any thread writes.  Needs blockDim.x >= 227; ends with a
// barrier, so x holds the new words.
__device__ __forceinline__ void mt_twist(uint32_t* x)
{
    const int j = threadIdx.x;
    uint32_t v = 0;
    if (j < 227) v = mt_next(x[j], x[j + 1], x[j + 397]);
    __syncthreads();
    if (j < 227) x[j] = v;
    __syncthreads();
    if (j < 227) v = mt_next(x[227 + j], x[228 + j], x[j]);
    __syncthreads();
    if (j < 227) x[227 + j] = v;
    __syncthreads();
    if (j < 170) {
        const int jj = 454 + j;
        v = mt_next(x[jj], jj + 1 < kMtN ? x[jj + 1] : x[0], x[jj - 227]);
    }
    __syncthreads();
    if (j < 170) x[454 + j] = v;
    __syncthreads();
}

// draw % max_num for a 32-bit draw: the draw itself when max_num exceeds
// every draw, else Lemire's remainder by multiplication (exact for 32-bit
// operands), as the host NetGen computes it.
struct DrawMod {
    uint32_t d;
    uint64_t M;
    bool big;
    __device__ __forceinline__ uint64_t operator()(uint32_t a) const
    {
        if (big) return a;
        return __umul64hi(M * (uint64_t)a, (uint64_t)d);
    }
};

DrawMod make_mod(uint64_t max_num)
{
    DrawMod m;
    m.big = max_num > 0xffffffffull;
    m.d = (uint32_t)max_num;
    m.M = m.big ? 0 : UINT64_MAX / m.d + 1;
    return m;
}

__device__ __forceinline__ void load_state(uint32_t* x, const uint32_t* starts)
{
    for (int j = threadIdx.x; j < kMtN; j += blockDim.x) x[j] = starts[(size_t)blockIdx.x * kMtN + j];
    __syncthreads();
}

// Pass 1: taken pairs of stretch blockIdx.x (candidates [b*C, min((b+1)*C, max_num))).
__global__ void __launch_bounds__(kGenThreads) k_prob_count(const uint32_t* starts, uint64_t max_num, uint64_t C,
                                                            DrawMod mod, uint64_t limit, unsigned long long* counts)
{
    __shared__ uint32_t x[kMtN];
    __shared__ unsigned long long total;
    if (threadIdx.x == 0) total = 0;
    load_state(x, starts);
    const uint64_t lo = (uint64_t)blockIdx.x * C, hi = min(max_num, lo + C);
    unsigned long long mine = 0;
    for (uint64_t k0 = lo; k0 < hi; k0 += kMtN) {
        mt_twist(x);  // the next twist's first barrier comes after every read below
        for (int j = threadIdx.x; j < kMtN; j += blockDim.x)
            if (k0 + j < hi && mod(mt_temper(x[j])) < limit) ++mine;
    }
    typedef cub::BlockReduce<unsigned long long, kGenThreads> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    const unsigned long long sum = Reduce(tmp).Sum(mine);
    if (threadIdx.x == 0) counts[blockIdx.x] = sum;
}

// Pass 2: the taken pairs of stretch blockIdx.x, in order, at positions
// offset[b]...; pairs at positions >= gen_num are not written, and the pair
// at position gen_num - 1 records its candidate index in *last_k.
__global__ void __launch_bounds__(kGenThreads) k_prob_emit(const uint32_t* starts, uint64_t max_num, uint64_t C,
                                                           DrawMod mod, uint64_t limit, const unsigned long long* offset,
                                                           uint64_t gen_num, uint32_t tn, int32_t src0, int32_t tar0,
                                                           int32_t* src, int32_t* tar, unsigned long long* last_k)
{
    __shared__ uint32_t x[kMtN];
    typedef cub::BlockScan<int, kGenThreads> Scan;
    __shared__ typename Scan::TempStorage tmp;
    uint64_t base = offset[blockIdx.x];
    if (base >= gen_num) return;  // uniform over the block
    load_state(x, starts);
    const uint64_t lo = (uint64_t)blockIdx.x * C, hi = min(max_num, lo + C);
    for (uint64_t k0 = lo; k0 < hi && base < gen_num; k0 += kMtN) {
        mt_twist(x);
        for (int r = 0; r < kMtN; r += kGenThreads) {
            const int j = r + threadIdx.x;
            const uint64_t k = k0 + j;
            const int taken = (j < kMtN && k < hi && mod(mt_temper(x[j])) < limit) ? 1 : 0;
            int excl = 0, round_total = 0;
            Scan(tmp).ExclusiveSum(taken, excl, round_total);
            const uint64_t pos = base + excl;
            if (taken && pos < gen_num) {
                const uint64_t m = k / tn;
                src[pos] = src0 + (int32_t)m;
                tar[pos] = tar0 + (int32_t)(k - m * tn);
                if (pos == gen_num - 1) *last_k = k;
            }
            base += round_total;
            __syncthreads();  // the scan's storage is reused by the next round
        }
    }
}

// Pairs of the rules that need no sequential generator, synapse t of the
// projection: all pairs, one to one, all but self, fixed in-degree.
__global__ void k_rule_pairs(int rule, int64_t count, int32_t sn, int32_t tn, int32_t src0, int32_t tar0, int32_t k,
                             uint64_t seed, uint32_t rid, int32_t dmin, uint32_t dspan, int32_t* src, int32_t* tar,
                             int32_t* delay)
{
    GRID_STRIDE(t, count)
    {
        int64_t m = 0, n = 0;
        if (rule == MGC_RULE_ALL) {
            m = t / tn;
            n = t - m * tn;
        } else if (rule == MGC_RULE_ONE) {
            m = n = t;
        } else if (rule == MGC_RULE_ALL_BUT_SELF) {
            // rows m < min(sn, tn) skip column m (tn - 1 pairs), later rows have tn
            const int64_t rows_skip = sn < tn ? sn : tn;
            const int64_t first = rows_skip * (tn - 1);
            if (t < first) {
                m = t / (tn - 1);
                const int64_t j = t - m * (tn - 1);
                n = j < m ? j : j + 1;
            } else {
                const int64_t u = t - first;
                m = rows_skip + u / tn;
                n = u - (m - rows_skip) * tn;
            }
        } else {  // MGC_RULE_FIXED_INDEGREE: draw j of target n
            n = t / k;
            const int32_t j = (int32_t)(t - n * k);
            const U32x4 r = conn_draw(seed, (uint32_t)(tar0 + n), (uint32_t)j, rid);
            m = scale_u32(r.x, (uint32_t)sn);
            delay[t] = dmin + (int32_t)scale_u32(r.y, dspan);
        }
        src[t] = src0 + (int32_t)m;
        tar[t] = tar0 + (int32_t)n;
    }
}

__global__ void k_fill(int64_t count, int32_t* a, int32_t va, int32_t* b, int32_t vb)
{
    GRID_STRIDE(t, count)
    {
        a[t] = va;
        if (b) b[t] = vb;
    }
}

__global__ void k_fill_f(int64_t count, float* a, float v)
{
    GRID_STRIDE(t, count) a[t] = v;
}

// Per target: the least and largest |w| of each sign (as float bits, which
// order like the values for non-negative floats), the sum of |w| (of
// max(|w|, wlim) for a plastic synapse: the bound of one step's input), and
// the least exponent of a nonzero weight.
__global__ void k_fx_stats(const int32_t* tar, const float* w, const uint8_t* plastic, float wlim, int64_t S,
                           uint32_t* emin, uint32_t* emax, uint32_t* imin, uint32_t* imax, double* sum, int* min_exp)
{
    GRID_STRIDE(q, S)
    {
        const float x = w[q];
        const int32_t t = tar[q];
        const uint32_t bits = __float_as_uint(fabsf(x));
        if (x > 0.0f) {
            atomicMin(emin + t, bits);
            atomicMax(emax + t, bits);
        } else {
            atomicMin(imin + t, bits);
            atomicMax(imax + t, bits);
        }
        atomicAdd(sum + t, (double)((plastic && plastic[q]) ? fmaxf(fabsf(x), wlim) : fabsf(x)));
        if (x != 0.0f) {
            int e = 0;
            frexpf(x, &e);
            atomicMin(min_exp, e);
        }
    }
}

// Synapses projection r generates; -1 when it is malformed.
int64_t proj_count(const mgc_gen_desc* d, int32_t r)
{
    if (!d || r < 0 || r >= d->n_proj || !d->proj || !d->pop_num) return -1;
    const mgc_gen_proj& p = d->proj[r];
    if (p.src < 0 || p.src >= d->n_pops || p.tar < 0 || p.tar >= d->n_pops) return -1;
    const int64_t sn = d->pop_num[p.src], tn = d->pop_num[p.tar];
    switch (p.rule) {
    case MGC_RULE_PROB: {
        // round(max_num * ctype) in single precision, as gen_net computes it
        const uint64_t max_num = (uint64_t)sn * (uint64_t)tn;
        return (int64_t)std::round((float)max_num * p.prob);
    }
    case MGC_RULE_ALL: return sn * tn;
    case MGC_RULE_ONE: return sn == tn ? sn : -1;
    case MGC_RULE_ALL_BUT_SELF: return sn * tn - std::min(sn, tn);
    case MGC_RULE_FIXED_INDEGREE: return p.k >= 0 && (p.k == 0 || sn > 0) ? tn * p.k : -1;
    default: return -1;
    }
}

// Start states of B stretches of C draws from g: T^(bC) g, placed by jumps
// of C, 2C, 4C, ... from the states already placed (host threads).
std::vector<MGBrain::Mt19937> stretch_starts(const MGBrain::Mt19937& g, size_t B, uint64_t C)
{
    std::vector<MGBrain::Mt19937> st(B, g);
    if (B < 2) return st;
    MGBrain::MtJump jump(C);
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    size_t have = 1;
    while (have < B) {
        const size_t todo = std::min(have, B - have);
        std::vector<std::thread> pool;
        const size_t T = std::min<size_t>(hw, todo);
        for (size_t w = 0; w < T; ++w)
            pool.emplace_back([&, w] {
                for (size_t i = w; i < todo; i += T) {
                    st[have + i] = st[i];
                    jump.apply(st[have + i]);
                }
            });
        for (auto& th : pool) th.join();
        have += todo;
        if (have < B) jump = jump.doubled();
    }
    return st;
}

// The fixed-probability pairs of one projection into src/tar (gen_num
// entries), advancing g past the draws the rule consumes.
mgc_status gen_prob(mgc_sim* s, MGBrain::Mt19937& g, uint64_t max_num, uint64_t gen_num, int32_t tn, int32_t src0,
                    int32_t tar0, int32_t* src, int32_t* tar)
{
    if (gen_num == 0 || max_num == 0) {
        if (gen_num) k_fill<<<grid_for((int64_t)gen_num), 256, 0, s->stream>>>((int64_t)gen_num, src, src0, tar, tar0);
        return MGC_OK;
    }
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, s->device));
    const uint64_t want = (max_num + kStretchMin - 1) / kStretchMin;
    const size_t B = (size_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)prop.multiProcessorCount));
    const uint64_t C = (max_num + B - 1) / B;
    const std::vector<MGBrain::Mt19937> st = stretch_starts(g, B, C);
    std::vector<uint32_t> words(B * kMtN);
    for (size_t b = 0; b < B; ++b) st[b].state_words(words.data() + b * kMtN);
    DevTmp t_w, t_c, t_o, t_l;
    uint32_t* dwords;
    unsigned long long *dcounts, *doff, *dlast;
    CKS(tmp_alloc(t_w, &dwords, words.size()));
    CKS(tmp_alloc(t_c, &dcounts, B));
    CKS(tmp_alloc(t_o, &doff, B));
    CKS(tmp_alloc(t_l, &dlast, 1));
    CK(cudaMemcpyAsync(dwords, words.data(), 4 * words.size(), cudaMemcpyHostToDevice, s->stream));
    const DrawMod mod = make_mod(max_num);
    const uint64_t limit = (uint64_t)std::ceil((double)gen_num * 1.1);  // k < gen_num*1.1 <=> k < ceil(...)
    k_prob_count<<<(unsigned)B, kGenThreads, 0, s->stream>>>(dwords, max_num, C, mod, limit, dcounts);
    CK(cudaGetLastError());
    std::vector<unsigned long long> counts(B), off(B);
    CK(cudaMemcpyAsync(counts.data(), dcounts, 8 * B, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    unsigned long long total = 0;
    for (size_t b = 0; b < B; ++b) {
        off[b] = total;
        total += counts[b];
    }
    CK(cudaMemcpyAsync(doff, off.data(), 8 * B, cudaMemcpyHostToDevice, s->stream));
    k_prob_emit<<<(unsigned)B, kGenThreads, 0, s->stream>>>(dwords, max_num, C, mod, limit, doff, gen_num,
                                                             (uint32_t)tn, src0, tar0, src, tar, dlast);
    CK(cudaGetLastError());
    uint64_t consumed = max_num;
    if (total >= gen_num) {
        unsigned long long last = 0;
        CK(cudaMemcpyAsync(&last, dlast, 8, cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        consumed = last + 1;
    } else {  // the list's slots left over hold pair (0, 0) (netgen.cpp:210-222)
        const int64_t rest = (int64_t)(gen_num - total);
        k_fill<<<grid_for(rest), 256, 0, s->stream>>>(rest, src + total, src0, tar + total, tar0);
        CK(cudaGetLastError());
    }
    // the generator after the consumed draws: the start of their last stretch, advanced
    const size_t kc = (size_t)((consumed - 1) / C);
    g = st[kc];
    g.discard(consumed - kc * C);
    CK(cudaStreamSynchronize(s->stream));
    return MGC_OK;
}

}  // namespace

extern "C" int64_t mgc_gen_count(const mgc_gen_desc* d, int32_t r) { return proj_count(d, r); }

extern "C" mgc_status mgc_create_generated(const mgc_gen_desc* d, mgc_sim** out)
{
    if (!d || !out) return fail(MGC_ERR_INVALID, "null argument");
    *out = nullptr;
    if (d->n_pops <= 0 || !d->pop_num || !d->pop_type || d->n_proj < 0 || (d->n_proj > 0 && !d->proj))
        return fail(MGC_ERR_INVALID, "the network needs populations (and projections)");
    if (d->mode < MGC_MODE_AUTO || d->mode > MGC_MODE_PULL) return fail(MGC_ERR_INVALID, "unknown mode %d", d->mode);
    std::vector<int64_t> first(d->n_pops + 1, 0);
    for (int p = 0; p < d->n_pops; ++p) {
        if (d->pop_num[p] < 0) return fail(MGC_ERR_INVALID, "population %d has %d neurons", p, d->pop_num[p]);
        first[p + 1] = first[p] + d->pop_num[p];
    }
    if (first[d->n_pops] <= 0 || first[d->n_pops] > 0x7fffffff)
        return fail(MGC_ERR_INVALID, "the network needs 1 to 2^31-1 neurons");
    const int32_t n = (int32_t)first[d->n_pops];
    // synapses per projection, the delay range, the list's length
    std::vector<int64_t> cnt(d->n_proj), base(d->n_proj + 1, 0);
    int32_t dmin = 0x7fffffff, dmax = 0;
    bool any_plastic = false;
    for (int r = 0; r < d->n_proj; ++r) {
        const mgc_gen_proj& p = d->proj[r];
        cnt[r] = proj_count(d, r);
        if (cnt[r] < 0) return fail(MGC_ERR_INVALID, "projection %d is malformed", r);
        base[r + 1] = base[r] + cnt[r];
        if (!cnt[r]) continue;
        if (p.rule == MGC_RULE_FIXED_INDEGREE) {
            if (p.delay < 1 || p.delay_max < p.delay) return fail(MGC_ERR_INVALID, "projection %d: delays", r);
            dmin = std::min(dmin, p.delay);
            dmax = std::max(dmax, p.delay_max);
        } else if (p.delays) {
            for (int64_t q = 0; q < cnt[r]; ++q) {
                dmin = std::min(dmin, p.delays[q]);
                dmax = std::max(dmax, p.delays[q]);
            }
        } else {
            dmin = std::min(dmin, p.delay);
            dmax = std::max(dmax, p.delay);
        }
        any_plastic |= d->stdp && p.plastic;
    }
    const int64_t S = base[d->n_proj];
    if (S > (int64_t)0x7fffffff) return fail(MGC_ERR_INVALID, "%lld synapses: more than one sort takes", (long long)S);
    if (S == 0) dmin = dmax = 1;
    if (dmin < 1) return fail(MGC_ERR_INVALID, "synaptic delay below one step (%d)", dmin);
    CKS(pick_device(d->device));
    std::unique_ptr<mgc_sim> s(new mgc_sim);
    s->device = d->device;
    CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->n = n;
    s->S = S;
    s->stdp = d->stdp != 0;
    s->explicit_net = true;
    std::vector<int8_t> type(n);
    for (int p = 0; p < d->n_pops; ++p)
        for (int64_t i = first[p]; i < first[p + 1]; ++i) type[i] = d->pop_type[p];
    CKS(build_neurons(s.get(), n, type.data(), d->rate, d->v_init, d->lifconst, d->stdpconst, d->seed,
                      d->raster_steps, d->raster_ids));
    StepArgs& a = s->a;
    a.stdp = s->stdp;
    s->tpop_host.resize(n);
    for (int32_t i = 0; i < n; ++i) {
        const int t = type[i];
        s->tpop_host[i] = t == MGC_POISSON ? 0 : (t == MGC_LIF || t == MGC_LIFE || t == MGC_LIFB ? 1 : 2);
    }
    s->dmin = dmin;
    s->dmax = dmax;
    s->M = dmax + 1;
    CKS(build_method(s.get(), d->mode, false, 0));  // the accumulation plan follows from the list below
    CKS(begin_list_layout(s.get()));
    MGBrain::Mt19937 g;
    {
        // the caller's words are the logical order: ring position 0
        uint32_t w[kMtN];
        memcpy(w, d->mt_state, sizeof(w));
        g.set_state_words(w);
    }
    if (S > 0) {
        DevTmp t_src, t_tar, t_w, t_d, t_pl;
        int32_t *src, *tar, *dl;
        float* w;
        uint8_t* pl = nullptr;
        CKS(tmp_alloc(t_src, &src, S));
        CKS(tmp_alloc(t_tar, &tar, S));
        CKS(tmp_alloc(t_w, &w, S));
        CKS(tmp_alloc(t_d, &dl, S));
        if (d->stdp) CKS(tmp_alloc(t_pl, &pl, S));  // every synapse's flag (null would mean all plastic)
        for (int r = 0; r < d->n_proj; ++r) {
            const mgc_gen_proj& p = d->proj[r];
            const int64_t c = cnt[r], b0 = base[r];
            if (!c) continue;
            const int32_t sn = d->pop_num[p.src], tn = d->pop_num[p.tar];
            const int32_t src0 = (int32_t)first[p.src], tar0 = (int32_t)first[p.tar];
            if (p.rule == MGC_RULE_PROB) {
                CKS(gen_prob(s.get(), g, (uint64_t)sn * (uint64_t)tn, (uint64_t)c, tn, src0, tar0, src + b0, tar + b0));
            } else {
                k_rule_pairs<<<grid_for(c), 256, 0, s->stream>>>(
                    p.rule, c, sn, tn, src0, tar0, p.k, p.conn_seed, (uint32_t)r, p.delay,
                    (uint32_t)std::max(1, p.delay_max - p.delay + 1), src + b0, tar + b0, dl + b0);
                CK(cudaGetLastError());
            }
            if (p.weights)
                CK(cudaMemcpyAsync(w + b0, p.weights, 4 * c, cudaMemcpyHostToDevice, s->stream));
            else
                k_fill_f<<<grid_for(c), 256, 0, s->stream>>>(c, w + b0, p.weight);
            if (p.rule != MGC_RULE_FIXED_INDEGREE) {
                if (p.delays)
                    CK(cudaMemcpyAsync(dl + b0, p.delays, 4 * c, cudaMemcpyHostToDevice, s->stream));
                else
                    k_fill<<<grid_for(c), 256, 0, s->stream>>>(c, dl + b0, p.delay, nullptr, 0);
            }
            if (pl) CK(cudaMemsetAsync(pl + b0, (d->stdp && p.plastic) ? 1 : 0, c, s->stream));
            CK(cudaGetLastError());
        }
        // the accumulation plan of the list (as mgc_create computes it)
        {
            DevTmp t_a, t_b, t_c, t_dd, t_s, t_e;
            uint32_t *emin, *emax, *imin, *imax;
            double* sum;
            int* min_exp;
            CKS(tmp_alloc(t_a, &emin, n));
            CKS(tmp_alloc(t_b, &emax, n));
            CKS(tmp_alloc(t_c, &imin, n));
            CKS(tmp_alloc(t_dd, &imax, n));
            CKS(tmp_alloc(t_s, &sum, n));
            CKS(tmp_alloc(t_e, &min_exp, 1));
            CK(cudaMemsetAsync(emin, 0xff, 4 * (size_t)n, s->stream));
            CK(cudaMemsetAsync(imin, 0xff, 4 * (size_t)n, s->stream));
            CK(cudaMemsetAsync(emax, 0, 4 * (size_t)n, s->stream));
            CK(cudaMemsetAsync(imax, 0, 4 * (size_t)n, s->stream));
            CK(cudaMemsetAsync(sum, 0, 8 * (size_t)n, s->stream));
            const int big = 1 << 20;
            CK(cudaMemcpyAsync(min_exp, &big, 4, cudaMemcpyHostToDevice, s->stream));
            const float wlim = std::max(std::fabs(d->stdpconst[4]), std::fabs(d->stdpconst[5]));
            k_fx_stats<<<grid_for(S), 256, 0, s->stream>>>(tar, w, pl, wlim, S, emin, emax, imin, imax, sum, min_exp);
            CK(cudaGetLastError());
            std::vector<uint32_t> h[4];
            for (auto& v : h) v.resize(n);
            std::vector<double> hs(n);
            int hexp = big;
            CK(cudaMemcpyAsync(h[0].data(), emin, 4 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
            CK(cudaMemcpyAsync(h[1].data(), emax, 4 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
            CK(cudaMemcpyAsync(h[2].data(), imin, 4 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
            CK(cudaMemcpyAsync(h[3].data(), imax, 4 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
            CK(cudaMemcpyAsync(hs.data(), sum, 8 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
            CK(cudaMemcpyAsync(&hexp, min_exp, 4, cudaMemcpyDeviceToHost, s->stream));
            CK(cudaStreamSynchronize(s->stream));
            bool hetero = any_plastic;
            double bound = 0.0;
            for (int32_t t = 0; t < n; ++t) {
                hetero |= (h[1][t] && h[0][t] != h[1][t]) || (h[3][t] && h[2][t] != h[3][t]);
                bound = std::max(bound, hs[t]);
            }
            CKS(build_set_fx(s.get(), hetero, fx_shift_rule(bound, hexp, !any_plastic)));
        }
        CKS(csr_from_list(s.get(), src, tar, w, dl, pl));
    }
    if (d->mt_state_out) g.state_words(d->mt_state_out);
    CKS(build_finish(s.get()));
    *out = s.release();
    return MGC_OK;
}
