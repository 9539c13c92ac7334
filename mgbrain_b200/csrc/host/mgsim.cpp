// MGBrain C++ API: MGSimulator over the C ABI of the CUDA core.
#include "mgbrain/mgsim.h"

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

MGSimulator::MGSimulator(Network& net, std::vector<int>& part, int nparts)
{
    npart = nparts < 1 ? 1 : nparts;
    std::cout << (npart == 1 ? "run single-net on single-GPU" : "run multi-net on single-GPU") << std::endl;
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
    check(mgc_create(&d, &sim), "mgc_create");
    this->part = part;
}

MGSimulator::~MGSimulator()
{
    if (sim) mgc_destroy(sim);
}

void MGSimulator::drain_raster()
{
    int64_t first = 0, ns = 0, ni = 0;
    mgc_info info;
    check(mgc_get_info(sim, &info), "mgc_get_info");
    const int64_t steps = info.step - (int64_t)raster_counts.size();
    if (steps <= 0) return;
    std::vector<int64_t> counts(steps);
    int64_t total_cap = (int64_t)n_neurons * 64 + (1 << 20);
    std::vector<int32_t> ids(total_cap);
    const int st = mgc_read_raster(sim, &first, counts.data(), steps, ids.data(), total_cap, &ns, &ni);
    if (st == MGC_ERR_OVERFLOW) {
        // more spikes than the raster holds: keep simulating, stop recording
        if (!raster_complete) std::cerr << "mgbrain_b200: raster buffer overflow, raster incomplete" << std::endl;
        raster_complete = false;
    } else {
        check(st, "mgc_read_raster");
    }
    for (int64_t i = 0; i < ns; ++i) raster_counts.push_back(counts[i]);
    raster_ids.insert(raster_ids.end(), ids.begin(), ids.begin() + ni);
}

void MGSimulator::simulate(real time)
{
    // mgsim.cpp:801-802: round(time/STEP) steps; when that is not a multiple
    // of the minimum delay the last partial cycle is not run.
    const long long steps = static_cast<int>(std::round(time / Config::STEP));
    const long long eff = mgc_effective_steps(steps, min_delay);
    timer t;
    for (long long left = eff; left > 0;) {
        const long long c = std::min(left, kChunkSteps);
        check(mgc_run(sim, c), "mgc_run");
        check(mgc_sync(sim), "mgc_sync");
        drain_raster();
        left -= c;
    }
    check(mgc_sync(sim), "mgc_sync");
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
    check(mgc_read_state(sim, v.data(), nullptr, nullptr, nullptr, nullptr, nullptr), "mgc_read_state");
    return v;
}

std::vector<int> MGSimulator::get_fire_cnt()
{
    std::vector<int> c(n_neurons);
    check(mgc_read_state(sim, nullptr, nullptr, nullptr, nullptr, nullptr, c.data()), "mgc_read_state");
    return c;
}

std::vector<real> MGSimulator::get_weights()
{
    mgc_info info;
    check(mgc_get_info(sim, &info), "mgc_get_info");
    std::vector<real> w(info.n_synapses);
    check(mgc_read_weights(sim, w.data()), "mgc_read_weights");
    return w;
}

void MGSimulator::set_rates(const std::vector<real>& rate)
{
    check(mgc_set_rates(sim, rate.data(), (int32_t)rate.size()), "mgc_set_rates");
    check(mgc_sync(sim), "mgc_sync");
}

long long MGSimulator::get_events()
{
    mgc_info info;
    check(mgc_get_info(sim, &info), "mgc_get_info");
    return info.events;
}

}  // namespace MGBrain
