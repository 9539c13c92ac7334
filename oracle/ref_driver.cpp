/*
 * Test infrastructure: drives the reference MGBrain code itself, compiled
 * from its own sources (see oracle/Makefile, target `ref`), to produce
 * golden networks, rasters and end states.  Nothing of the reference is
 * copied: this file only calls the reference's public classes and its
 * step function the way MGSimulator::simulate_sparse does for npart=1
 * (src/simulator/mgsim/adj/mgsim.cpp:794-857), reading the fired flags
 * after each step because the reference records no raster.
 *
 * Two binaries come from this file: ref_gen (gen only, CPU, no CUDA
 * libraries) and ref_sim (all commands, needs a GPU).
 *
 *   ref_driver gen <spec> <out.net>
 *       env MGB_REF_MT_SEED (gen_net's mt19937), MGB_REF_RAND_SEED (srand)
 *   ref_driver steps <in.net> <out_prefix> <steps> <v0.f32|-> <stdp 0|1> [rates_off_step]
 *       runs exactly <steps> steps through mgsim_step_sparse
 *       (mgcore.cu:535-554); env MGB_REF_SEED seeds the Poisson draws;
 *       from step rates_off_step on, every POISSON rate is 0.
 *       Writes <out_prefix>.raster (int64 steps, int64 counts[steps],
 *       int32 ids) and <out_prefix>.state (see write_state).
 *   ref_driver simulate <in.net> <out_prefix> <seconds> <v0.f32|-> <stdp 0|1>
 *       calls MGSimulator::simulate(seconds) itself and writes the end
 *       state plus the wall time in <out_prefix>.time.
 */
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <queue>
#include <random>
#include <sstream>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#ifndef MGB_REF_GEN_ONLY
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <nvml.h>
#include <omp.h>
#endif

#include "macro.h"
#include "model/constgen.h"
#include "model/maker.h"
#include "model/model.h"
#include "model/netgen.h"
#include "model/network.h"
#ifndef MGB_REF_GEN_ONLY
#include "simulator/sim.h"
#endif

#include "mgb_netfile.h"
#include "mgb_spec.h"

using namespace MGBrain;

#ifndef MGB_REF_GEN_ONLY
// MGSimulator keeps its MultiNet private (mgsim.h:54-57).  The driver needs
// the device pointers to dump per-step fired flags, so it names the member
// through an explicit template instantiation, which C++ allows for private
// members ([temp.explicit]).
template <class Tag, typename Tag::type Member>
struct MemberAccess {
    friend typename Tag::type member_of(Tag) { return Member; }
};
struct MultiNetTag {
    typedef MultiNet MGSimulator::*type;
    friend type member_of(MultiNetTag);
};
template struct MemberAccess<MultiNetTag, &MGSimulator::multinet>;
static MultiNet& multinet_of(MGSimulator& sim) { return sim.*member_of(MultiNetTag()); }
#endif

static std::string slurp(const char* path)
{
    std::ifstream f(path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

static int cmd_gen(const char* spec, const char* out)
{
    const char* rs = getenv("MGB_REF_RAND_SEED");
    srand(rs ? (unsigned)strtoul(rs, nullptr, 10) : 1u);
    Model m;
    mgb_spec::Applied app = mgb_spec::apply(slurp(spec), m);
    Network net;
    NetGen::gen_net(net, m);
    for (auto& pr : app.rates)
        for (int id : net.pops.at(pr.first).neurons) net.neurons[id].rate = pr.second;
    mgb_netfile::write(out, net, Config::STEP, Config::DW);
    printf("neurons %zu synapses %zu\n", net.neurons.size(), net.synapses.size());
    return 0;
}

#ifndef MGB_REF_GEN_ONLY
static void load_network(const char* path, Network& net, bool stdp)
{
    mgb_netfile::Arrays a = mgb_netfile::read(path);
    Config::set_timestep(a.step);
    Config::set_dw(a.dw);
    Config::enable_single_gpu();
    if (stdp) Config::enable_stdp();
    int nid = 0;
    for (int p = 0; p < a.n_pops; ++p) {
        const int32_t* r = &a.pops[4 * p];
        net.pops.emplace_back(r[0], r[1], r[2] != 0, (NeuronType)r[3]);
        for (int j = 0; j < r[1]; ++j) net.pops.back().neurons[j] = nid++;
    }
    net.neurons.reserve(a.n);
    for (int i = 0; i < a.n; ++i) {
        net.neurons.emplace_back(i, false, (NeuronType)a.type[i]);
        net.neurons.back().rate = a.rate[i];
    }
    net.synapses.reserve(a.S);
    for (int64_t k = 0; k < a.S; ++k)
        net.synapses.emplace_back(a.src[k], a.tar[k], a.weight[k], a.delay[k]);
    net.nlifconst = a.nlifconst != 0;
    net.nstdpconst = a.nstdpconst != 0;
    for (int i = 0; i < 30; ++i) net.lifconst[i] = a.lifconst[i];
    for (int i = 0; i < 6; ++i) net.stdpconst[i] = a.stdpconst[i];
}

static void set_v0(MGSimulator& sim, const char* v0path, int n)
{
    if (!v0path || std::string(v0path) == "-") return;
    std::vector<float> v0(n);
    FILE* f = fopen(v0path, "rb");
    if (!f || fread(v0.data(), 4, n, f) != (size_t)n) {
        fprintf(stderr, "cannot read %s\n", v0path);
        exit(2);
    }
    fclose(f);
    GSubNet* tmp = toCPU(multinet_of(sim).gnets[0], 1);
    CUDACHECK(cudaMemcpy(tmp->neus.V_m, v0.data(), 4 * (size_t)n, cudaMemcpyHostToDevice));
    delete[] tmp;
}

template <class T>
static void dump(FILE* f, const T* dev, size_t n)
{
    std::vector<T> h(n);
    if (n) CUDACHECK(cudaMemcpy(h.data(), dev, sizeof(T) * n, cudaMemcpyDeviceToHost));
    fwrite(h.data(), sizeof(T), n, f);
}

/* <prefix>.state: float V[n], float I_exc[n], float I_inh[n], int32 refrac[n],
 * int32 last_fired[n], int32 fire_cnt[n], float weight[S] (synapse order). */
static void write_state(MGSimulator& sim, const std::string& prefix)
{
    GSubNet* tmp = toCPU(multinet_of(sim).gnets[0], 1);
    size_t n = tmp->neus.size, S = tmp->syns.size;
    FILE* f = fopen((prefix + ".state").c_str(), "wb");
    dump(f, tmp->neus.V_m, n);
    dump(f, tmp->neus.I_exc, n);
    dump(f, tmp->neus.I_inh, n);
    dump(f, tmp->neus.Refrac_state, n);
    dump(f, tmp->neus.last_fired, n);
    dump(f, tmp->neus.fire_cnt, n);
    dump(f, tmp->syns.weight, S);
    fclose(f);
    delete[] tmp;
}

static int cmd_steps(const char* netpath, const char* prefix, long steps, const char* v0, bool stdp,
                     long rates_off)
{
    Network net;
    load_network(netpath, net, stdp);
    int n = (int)net.neurons.size();
    std::vector<int> part(n, 0);
    MGSimulator sim(net, part, 1);
    set_v0(sim, v0, n);
    GSubNet* gnet = multinet_of(sim).gnets[0];
    GSubNet* cnet = multinet_of(sim).cnets[0];
    BufferManager& manager = multinet_of(sim).manager;
    cudaStream_t stream = manager.sim_streams[0];
    GSubNet* tmp = toCPU(gnet, 1);
    bool* dfired = tmp->neus.fired;
    delete[] tmp;
    std::vector<int64_t> counts(steps);
    std::vector<int32_t> ids;
    std::vector<unsigned char> fired(n);
    for (long i = 0; i < steps; ++i) {
        if (i == rates_off) {  // input schedule: every POISSON rate drops to 0 from this step
            GSubNet* t2 = toCPU(gnet, 1);
            CUDACHECK(cudaMemset(t2->neus.rate, 0, sizeof(real) * n));
            delete[] t2;
        }
        mgsim_step_sparse(gnet, cnet, (int)i, multinet_of(sim).blocksize, manager,
                          multinet_of(sim).gaddrs[0], 0, stream);
        CUDACHECK(cudaStreamSynchronize(stream));
        CUDACHECK(cudaMemcpy(fired.data(), dfired, n, cudaMemcpyDeviceToHost));
        int64_t c = 0;
        for (int j = 0; j < n; ++j)
            if (fired[j]) { ids.push_back(j); ++c; }
        counts[i] = c;
    }
    FILE* f = fopen((std::string(prefix) + ".raster").c_str(), "wb");
    int64_t st = steps;
    fwrite(&st, 8, 1, f);
    fwrite(counts.data(), 8, steps, f);
    fwrite(ids.data(), 4, ids.size(), f);
    fclose(f);
    write_state(sim, prefix);
    printf("steps %ld spikes %zu M %d min_delay %d\n", steps, ids.size(), multinet_of(sim).max_delay,
           multinet_of(sim).min_delay);
    return 0;
}

static int cmd_simulate(const char* netpath, const char* prefix, float secs, const char* v0, bool stdp)
{
    Network net;
    load_network(netpath, net, stdp);
    int n = (int)net.neurons.size();
    std::vector<int> part(n, 0);
    MGSimulator sim(net, part, 1);
    set_v0(sim, v0, n);
    sim.simulate(secs);
    CUDACHECK(cudaDeviceSynchronize());
    write_state(sim, prefix);
    FILE* f = fopen((std::string(prefix) + ".time").c_str(), "w");
    fprintf(f, "%.9f\n", sim.get_time());
    fclose(f);
    printf("simulate %.6f s wall %.6f s\n", secs, sim.get_time());
    return 0;
}

#endif

int main(int argc, char** argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: ref_driver gen|steps|simulate ...\n");
        return 2;
    }
    std::string cmd = argv[1];
    if (cmd == "gen" && argc == 4) return cmd_gen(argv[2], argv[3]);
#ifndef MGB_REF_GEN_ONLY
    if (cmd == "steps" && (argc == 7 || argc == 8))
        return cmd_steps(argv[2], argv[3], atol(argv[4]), argv[5], atoi(argv[6]) != 0,
                         argc == 8 ? atol(argv[7]) : -1);
    if (cmd == "simulate" && argc == 7)
        return cmd_simulate(argv[2], argv[3], (float)atof(argv[4]), argv[5], atoi(argv[6]) != 0);
#endif
    fprintf(stderr, "bad arguments\n");
    return 2;
}
