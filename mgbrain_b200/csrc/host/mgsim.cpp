// MGBrain C++ API: MGSimulator over the C ABI of the CUDA core.
#include "mgbrain/mgsim.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <iostream>

#include "mgc.h"

namespace MGBrain {

namespace {

// Steps per mgc_run between raster drains (the raster holds 65536 steps and
// 64 spikes per neuron).
constexpr long long kChunkSteps = 4096;

// LIFECONSTS the reference's kernels run with when the network brings
// none: copy_consts_gpu(max_delay, dt) uploads this array with DT = dt
// and V_THRESH 15 (mgcore.cu:685-734); when only STDP constants were set
// the __constant__ initialiser stays, with DT 0.0001 and V_THRESH 0.02
// (mgcore.cu:32-63, :735-748).
std::array<float, 30> default_lifconst(bool stdp_set, float dt)
{
    std::array<float, 30> c{};
    c[5] = 0.25f;
    c[6] = 10.0f;
    c[8] = 0.0004f;
    c[10] = 1.0f;
    c[11] = 1.0f;
    c[21] = 0.951229453f;
    c[22] = 0.967216074f;
    c[23] = 0.0799999982f;
    c[24] = 0.0599999987f;
    c[25] = 0.90483743f;
    if (stdp_set) {
        c[0] = 0.0001f;
        c[4] = 0.02f;
    } else {
        c[0] = dt;
        c[4] = 15.0f;
    }
    return c;
}

}  // namespace

void MGSimulator::check(int status, const char* what)
{
    if (status == MGC_OK) return;
    const char* msg = mgc_last_error();
    if (Config::THROW_ON_ERROR) throw Error(status, std::string(what) + ": " + msg);
    // the reference's CUDACHECK prints and exits (cudamem.cuh:8-18)
    printf("Error:%s,code:%d, reason:%s\n", what, status, msg);
    exit(1);
}

// The network of a Config::DEVICE_NETGEN recipe, generated on the device
// (mgc_create_generated) as one handle.
void MGSimulator::build_generated(Network& net)
{
    const size_t n = net.neurons.size();
    n_neurons = (int)n;
    std::vector<float> rate(n), v0(n);
    for (size_t i = 0; i < n; ++i) {
        rate[i] = net.neurons[i].rate;
        v0[i] = net.v_init.size() == n ? net.v_init[i] : net.lifconst[1];
    }
    std::vector<int32_t> pop_num(net.pops.size());
    std::vector<int8_t> pop_type(net.pops.size());
    for (size_t p = 0; p < net.pops.size(); ++p) {
        pop_num[p] = net.pops[p].num;
        pop_type[p] = (int8_t)net.pops[p].type;
    }
    const Network::GenRecipe& rc = net.recipe;
    std::vector<mgc_gen_proj> pr(rc.projs.size());
    for (size_t r = 0; r < rc.projs.size(); ++r) {
        const Network::GenProjection& g = rc.projs[r];
        mgc_gen_proj& q = pr[r];
        q.src = g.src;
        q.tar = g.tar;
        q.rule = g.rule;
        q.prob = g.prob;
        q.k = g.k;
        q.conn_seed = g.seed;
        q.weight = g.weight;
        q.delay = g.delay;
        q.delay_max = g.delay_max;
        q.weights = g.weights.empty() ? nullptr : g.weights.data();
        q.delays = g.delays.empty() ? nullptr : g.delays.data();
        // Config::STDP makes every synapse plastic unless STDP_BY_TYPE gates it by projection
        q.plastic = Config::STDP_BY_TYPE ? (g.plastic ? 1 : 0) : 1;
    }
    mgc_gen_desc d{};
    d.n_pops = (int32_t)pop_num.size();
    d.pop_num = pop_num.data();
    d.pop_type = pop_type.data();
    d.n_proj = (int32_t)pr.size();
    d.proj = pr.data();
    for (int k = 0; k < 624; ++k) d.mt_state[k] = rc.mt[k];
    d.rate = rate.data();
    d.v_init = v0.data();
    const std::array<float, 30> lc = net.nlifconst ? net.lifconst : default_lifconst(net.nstdpconst, Config::DT);
    for (int i = 0; i < 30; ++i) d.lifconst[i] = lc[i];
    const std::array<float, 6> sc =
        net.nstdpconst ? net.stdpconst : std::array<float, 6>{0.1f, -0.01f, 17, 34, 40, 0};
    for (int i = 0; i < 6; ++i) d.stdpconst[i] = sc[i];
    d.stdp = Config::STDP ? 1 : 0;
    d.mode = MGC_MODE_AUTO;
    if (Config::SEED >= 0) {
        d.seed = (uint64_t)Config::SEED;
    } else {
        srand((unsigned)time(0));  // as init_state does (mgcore.cu:665-669)
        d.seed = (uint64_t)rand();
    }
    d.device = Config::DEVICE;
    d.raster_steps = 65536;
    d.raster_ids = 0;
    if (npart > 1)
        std::cerr << "mgbrain_b200: a network generated on the device runs as one handle; the " << npart
                  << " partitions run together" << std::endl;
    std::cout << (npart == 1 ? "run single-net on single-GPU" : "run multi-net on single-GPU") << std::endl;
    Piece pc;
    pc.count = (int)n;
    pc.device = Config::DEVICE;
    check(mgc_create_generated(&d, &pc.sim), "mgc_create_generated");
    pieces.push_back(pc);
    sim = pc.sim;
    mgc_info info;
    check(mgc_get_info(sim, &info), "mgc_get_info");
    min_delay = info.min_delay;
    max_delay = info.max_delay;
}

MGSimulator::MGSimulator(Network& net, std::vector<int>& part, int nparts)
{
    npart = nparts < 1 ? 1 : nparts;
    this->part = part;
    if (net.recipe.active) {
        build_generated(net);
        return;
    }
    const size_t n = net.neurons.size();
    const size_t S = net.synapses.size();
    n_neurons = (int)n;
    std::vector<int8_t> type(n);
    std::vector<float> rate(n), v0(n);
    for (size_t i = 0; i < n; ++i) {
        type[i] = (int8_t)net.neurons[i].type;
        rate[i] = net.neurons[i].rate;
        // mgsim.cpp:97: every neuron starts at lifconst[1]
        v0[i] = net.v_init.size() == n ? net.v_init[i] : net.lifconst[1];
    }
    std::vector<int32_t> src(S), tar(S), delay(S);
    std::vector<float> w(S);
    min_delay = S ? 0x7fffffff : 1;
    max_delay = S ? 0 : 1;
    for (size_t k = 0; k < S; ++k) {
        const Synapse& s = net.synapses[k];
        src[k] = s.src;
        tar[k] = s.tar;
        w[k] = s.weight;
        delay[k] = (int32_t)std::round(s.delay / Config::STEP);  // mgsim.cpp:49
        min_delay = std::min(min_delay, delay[k]);
        max_delay = std::max(max_delay, delay[k]);
        if ((size_t)s.src >= n || (size_t)s.tar >= n) check(MGC_ERR_INVALID, "synapse endpoint out of range");
    }
    if (min_delay < 1)
        check(MGC_ERR_INVALID, "a synaptic delay rounds to 0 steps (the reference divides by min_delay)");
    mgc_net_desc d{};
    d.n_neurons = (int32_t)n;
    d.type = type.data();
    d.rate = rate.data();
    d.v_init = v0.data();
    d.n_synapses = (int64_t)S;
    d.syn_src = src.data();
    d.syn_tar = tar.data();
    d.syn_weight = w.data();
    d.syn_delay = delay.data();
    std::vector<uint8_t> plastic;
    if (Config::STDP && Config::STDP_BY_TYPE && net.plastic.size() == S) {
        plastic.assign(net.plastic.begin(), net.plastic.end());
        d.syn_plastic = plastic.data();
    }
    const std::array<float, 30> lc =
        net.nlifconst ? net.lifconst : default_lifconst(net.nstdpconst, Config::DT);
    for (int i = 0; i < 30; ++i) d.lifconst[i] = lc[i];
    const std::array<float, 6> sc =
        net.nstdpconst ? net.stdpconst : std::array<float, 6>{0.1f, -0.01f, 17, 34, 40, 0};
    for (int i = 0; i < 6; ++i) d.stdpconst[i] = sc[i];
    d.stdp = Config::STDP ? 1 : 0;
    d.mode = MGC_MODE_AUTO;
    if (Config::SEED >= 0) {
        d.seed = (uint64_t)Config::SEED;
    } else {
        srand((unsigned)time(0));  // as init_state does (mgcore.cu:665-669)
        d.seed = (uint64_t)rand();
    }
    d.device = Config::DEVICE;
    d.raster_steps = 65536;
    d.raster_ids = 0;
    this->part = part;

    // the partitions as separate handles: each a run of consecutive ids
    std::vector<std::pair<int, int>> ranges;  // (first, count) of the non-empty zones
    const char* why = nullptr;
    if (npart > 1 && !Config::SINGLE_GPU) {
        bool consecutive = part.size() == n;
        for (size_t i = 0; consecutive && i < n; ++i)
            consecutive = part[i] >= 0 && part[i] < npart && (i == 0 || part[i] >= part[i - 1]);
        if (!consecutive)
            why = "the partitions are not runs of consecutive neuron ids";
        else if (Config::STDP)
            why = "plastic weights (STDP) run in one handle";
        else if (min_delay < 2)
            why = "a minimum delay of one step leaves no exchange window";
        for (size_t i = 0; !why && i < n;) {
            size_t j = i;
            while (j < n && part[j] == part[i]) ++j;
            ranges.emplace_back((int)i, (int)(j - i));
            i = j;
        }
    }
    if (why) {
        std::cerr << "mgbrain_b200: " << why << "; the " << npart << " partitions run as one handle" << std::endl;
        ranges.clear();
    }
    if (ranges.size() > 1) {
        int devices = 1;
        if (cudaGetDeviceCount(&devices) != cudaSuccess || devices < 1) devices = 1;
        std::cout << "run multi-net on " << (devices > 1 ? "multi-GPU" : "single-GPU") << std::endl;
        for (size_t p = 0; p < ranges.size(); ++p) {
            Piece pc;
            pc.first = ranges[p].first;
            pc.count = ranges[p].second;
            pc.device = (Config::DEVICE + (int)p) % devices;
            d.device = pc.device;
            d.mode = MGC_MODE_DEFERRED;
            check(mgc_create_partition(&d, pc.first, pc.count, &pc.sim), "mgc_create_partition");
            pieces.push_back(pc);
            const size_t cap = (size_t)(min_delay - 1) * (size_t)pc.count;
            cudaSetDevice(pc.device);
            if (cudaMalloc(&pieces.back().xout, 4 * std::max<size_t>(cap, 1)) != cudaSuccess)
                check(MGC_ERR_NOMEM, "exchange buffer");
        }
        syn_tar = tar;
    } else {
        std::cout << (npart == 1 ? "run single-net on single-GPU" : "run multi-net on single-GPU") << std::endl;
        Piece pc;
        pc.count = (int)n;
        pc.device = Config::DEVICE;
        check(mgc_create(&d, &pc.sim), "mgc_create");
        pieces.push_back(pc);
    }
    sim = pieces[0].sim;
}

MGSimulator::~MGSimulator()
{
    for (Piece& p : pieces) {
        if (p.xout || p.xin) cudaSetDevice(p.device);
        if (p.xout) cudaFree(p.xout);
        if (p.xin) cudaFree(p.xin);
        if (p.sim) mgc_destroy(p.sim);
    }
}

// The partitions' spike ids of the last `steps` steps, each partition's
// appended to every other's history (through host memory, so the partitions
// may sit on any devices).
void MGSimulator::exchange(int steps)
{
    const int R = (int)pieces.size();
    std::vector<int32_t> counts((size_t)R * steps);
    std::vector<int64_t> total(R);
    std::vector<std::vector<int32_t>> ids(R);
    for (int r = 0; r < R; ++r) {
        Piece& p = pieces[r];
        const int64_t cap = (int64_t)(min_delay - 1) * p.count;
        check(mgc_part_export(p.sim, steps, counts.data() + (size_t)r * steps, p.xout, cap, &total[r]),
              "mgc_part_export");
        ids[r].resize(std::max<int64_t>(total[r], 1));
        cudaSetDevice(p.device);
        if (total[r] && cudaMemcpy(ids[r].data(), p.xout, 4 * (size_t)total[r], cudaMemcpyDeviceToHost) != cudaSuccess)
            check(MGC_ERR_CUDA, "exchange copy");
    }
    const int64_t stride = std::max<int64_t>(1, *std::max_element(total.begin(), total.end()));
    std::vector<int32_t> all((size_t)R * stride, 0);
    for (int r = 0; r < R; ++r) std::copy(ids[r].begin(), ids[r].begin() + total[r], all.begin() + (size_t)r * stride);
    for (int r = 0; r < R; ++r) {
        Piece& p = pieces[r];
        cudaSetDevice(p.device);
        if (p.xin_cap < (long long)all.size()) {
            if (p.xin) cudaFree(p.xin);
            p.xin = nullptr;
            if (cudaMalloc(&p.xin, 4 * all.size()) != cudaSuccess) check(MGC_ERR_NOMEM, "exchange buffer");
            p.xin_cap = (long long)all.size();
        }
        if (cudaMemcpy(p.xin, all.data(), 4 * all.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            check(MGC_ERR_CUDA, "exchange copy");
        check(mgc_part_import(p.sim, steps, R, r, counts.data(), p.xin, stride), "mgc_part_import");
    }
}

void MGSimulator::drain_raster()
{
    const long long before = (long long)raster_counts.size();
    std::vector<std::vector<int64_t>> pc(pieces.size());
    std::vector<std::vector<int32_t>> pi(pieces.size());
    int64_t steps = 0;
    for (size_t q = 0; q < pieces.size(); ++q) {
        mgc_info info;
        check(mgc_get_info(pieces[q].sim, &info), "mgc_get_info");
        steps = info.step - before;
        if (steps <= 0) return;
        int64_t first = 0, ns = 0, ni = 0;
        pc[q].resize(steps);
        const int64_t cap = (int64_t)pieces[q].count * 64 + (1 << 20);
        pi[q].resize(cap);
        const int st = mgc_read_raster(pieces[q].sim, &first, pc[q].data(), steps, pi[q].data(), cap, &ns, &ni);
        if (st == MGC_ERR_OVERFLOW) {
            // more spikes than the raster holds: keep simulating, stop recording
            if (raster_complete) std::cerr << "mgbrain_b200: raster buffer overflow, raster incomplete" << std::endl;
            raster_complete = false;
        } else {
            check(st, "mgc_read_raster");
        }
        pc[q].resize(ns);
        pi[q].resize(ni);
        steps = std::min<int64_t>(steps, ns);
    }
    if (pieces.size() == 1) {
        raster_counts.insert(raster_counts.end(), pc[0].begin(), pc[0].end());
        raster_ids.insert(raster_ids.end(), pi[0].begin(), pi[0].end());
        return;
    }
    // partitions: step by step, the union of their (whole-network) ids, ascending
    std::vector<size_t> pos(pieces.size(), 0);
    for (int64_t s = 0; s < steps; ++s) {
        const size_t at = raster_ids.size();
        for (size_t q = 0; q < pieces.size(); ++q) {
            const size_t c = (size_t)pc[q][s];
            raster_ids.insert(raster_ids.end(), pi[q].begin() + pos[q], pi[q].begin() + pos[q] + c);
            pos[q] += c;
        }
        std::sort(raster_ids.begin() + at, raster_ids.end());
        raster_counts.push_back((long long)(raster_ids.size() - at));
    }
}

mgc_tune_report MGSimulator::autotune(long long steps_per_trial)
{
    mgc_tune_report rep{};
    if (pieces.size() != 1) check(MGC_ERR_INVALID, "autotune: the network runs on one handle per partition");
    drain_raster();
    check(mgc_autotune_rewind(sim, steps_per_trial, &rep), "mgc_autotune_rewind");
    tuned = true;
    return rep;
}

void MGSimulator::simulate(real time)
{
    // mgsim.cpp:801-802: round(time/STEP) steps; when that is not a multiple
    // of the minimum delay the last partial cycle is not run.
    const long long steps = static_cast<int>(std::round(time / Config::STEP));
    const long long eff = mgc_effective_steps(steps, min_delay);
    if (Config::AUTOTUNE_STEPS > 0 && !tuned && pieces.size() == 1) autotune(Config::AUTOTUNE_STEPS);
    timer t;
    if (pieces.size() == 1) {
        for (long long left = eff; left > 0;) {
            const long long c = std::min(left, kChunkSteps);
            check(mgc_run(sim, c), "mgc_run");
            check(mgc_sync(sim), "mgc_sync");
            drain_raster();
            left -= c;
        }
    } else {
        // windows of at most min_delay - 1 steps, each followed by the exchange
        long long since_drain = 0;
        for (long long left = eff; left > 0;) {
            const int c = (int)std::min<long long>(left, min_delay - 1);
            for (Piece& p : pieces) check(mgc_run(p.sim, c), "mgc_run");
            exchange(c);
            left -= c;
            since_drain += c;
            if (since_drain >= kChunkSteps || left == 0) {
                drain_raster();
                since_drain = 0;
            }
        }
    }
    for (Piece& p : pieces) check(mgc_sync(p.sim), "mgc_sync");
    total_steps += eff;
    sim_time = t.stop();
    if (Config::FIRE_CHECK) get_firing_rate(time);
}

double MGSimulator::get_time() { return sim_time; }

// mgsim.cpp:596-615: fire counts per zone (partition), then over all neurons
real MGSimulator::get_firing_rate(real time)
{
    std::vector<int> fc = get_fire_cnt();
    std::vector<size_t> zone_cnt(npart, 0), zone_neu(npart, 0);
    for (int i = 0; i < n_neurons; ++i) {
        const int z = (part.size() == (size_t)n_neurons && part[i] >= 0 && part[i] < npart) ? part[i] : 0;
        zone_cnt[z] += (size_t)fc[i];
        zone_neu[z] += 1;
    }
    size_t all = 0, alln = 0;
    for (int z = 0; z < npart; ++z) {
        std::cout << "zone(" << z << ")'fire cnt:" << zone_cnt[z] << std::endl;
        std::cout << "zone(" << z << ")'fire rate:" << (float)zone_cnt[z] / zone_neu[z] / time << " hz" << std::endl;
        all += zone_cnt[z];
        alln += zone_neu[z];
    }
    const float r = (float)all / alln / time;
    std::cout << "fire rate:" << r << "hz" << std::endl;
    return r;
}

const std::vector<long long>& MGSimulator::spike_counts() { return raster_counts; }
const std::vector<int>& MGSimulator::spike_ids() { return raster_ids; }

std::vector<real> MGSimulator::get_v()
{
    std::vector<real> v(n_neurons);
    for (Piece& p : pieces)
        check(mgc_read_state(p.sim, v.data() + p.first, nullptr, nullptr, nullptr, nullptr, nullptr), "mgc_read_state");
    return v;
}

std::vector<int> MGSimulator::get_fire_cnt()
{
    std::vector<int> c(n_neurons);
    for (Piece& p : pieces)
        check(mgc_read_state(p.sim, nullptr, nullptr, nullptr, nullptr, nullptr, c.data() + p.first), "mgc_read_state");
    return c;
}

std::vector<real> MGSimulator::get_weights()
{
    if (pieces.size() == 1) {
        mgc_info info;
        check(mgc_get_info(sim, &info), "mgc_get_info");
        std::vector<real> w(info.n_synapses);
        if (!w.empty()) check(mgc_read_weights(sim, w.data()), "mgc_read_weights");
        return w;
    }
    // a partition holds the synapses that target its neurons, in synapse order
    std::vector<real> w(syn_tar.size());
    for (Piece& p : pieces) {
        mgc_info info;
        check(mgc_get_info(p.sim, &info), "mgc_get_info");
        if (info.n_synapses == 0) continue;
        std::vector<real> wp(info.n_synapses);
        check(mgc_read_weights(p.sim, wp.data()), "mgc_read_weights");
        size_t j = 0;
        for (size_t k = 0; k < syn_tar.size(); ++k)
            if (syn_tar[k] >= p.first && syn_tar[k] < p.first + p.count) w[k] = wp[j++];
    }
    return w;
}

void MGSimulator::set_rates(const std::vector<real>& rate)
{
    if (rate.size() != (size_t)n_neurons) check(MGC_ERR_INVALID, "set_rates: one rate per neuron");
    for (Piece& p : pieces) {
        check(mgc_set_rates(p.sim, rate.data() + p.first, p.count), "mgc_set_rates");
        check(mgc_sync(p.sim), "mgc_sync");
    }
}

long long MGSimulator::get_events()
{
    long long e = 0;
    for (Piece& p : pieces) {
        mgc_info info;
        check(mgc_get_info(p.sim, &info), "mgc_get_info");
        e += info.events;
    }
    return e;
}

}  // namespace MGBrain
