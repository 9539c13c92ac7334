// Test program for the MGBrain C++ API of mgbrain_b200, written the way the
// reference's own bench programs use the API (bench/single_brunel.cpp):
// model -> netgen::gen_net -> parter::part_network -> mgsim.simulate.
//
//   api_driver gen <spec> <out.net>              env MGB_MT_SEED, MGB_RAND_SEED
//   api_driver simulate <spec> <out_prefix> <seconds> <v0.f32|-> <stdp 0|1> [npart [single|multi]]
//                                                env MGB_MT_SEED, MGB_RAND_SEED, MGB_SEED
//   (npart > 1: SIMPLE partitions; "single" calls config::enable_single_gpu())
//   env MGB_DEVICE_NETGEN=1: config::enable_device_netgen() (the network is
//   generated on the device when the simulator is built)
//   env MGB_AUTOTUNE=k: config::enable_autotune(k) (trials of k steps before
//   the first step, undone)
// simulate writes <out_prefix>.state (V, fire_cnt, weights) and .raster.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "mgbrain.h"
#define MGB_SPEC_EXTENSIONS  // this Model has the fixed in-degree and all-but-self rules
#include "../../oracle/mgb_netfile.h"
#include "../../oracle/mgb_spec.h"

static std::string slurp(const char* p)
{
    std::ifstream f(p);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

static long long env(const char* k, long long d)
{
    const char* v = getenv(k);
    return v ? atoll(v) : d;
}

static void build(const char* spec, network& net)
{
    config::set_netgen_seed(env("MGB_MT_SEED", 5489));
    config::enable_device_netgen(env("MGB_DEVICE_NETGEN", 0) != 0);
    srand((unsigned)env("MGB_RAND_SEED", 1));
    model m;
    mgb_spec::Applied app = mgb_spec::apply(slurp(spec), m);
    netgen::gen_net(net, m);
    for (auto& pr : app.rates)
        for (int id : net.pops.at(pr.first).neurons) net.neurons[id].rate = pr.second;
}

int main(int argc, char** argv)
{
    if (argc >= 4 && std::string(argv[1]) == "gen") {
        network net;
        build(argv[2], net);
        mgb_netfile::write(argv[3], net, MGBrain::Config::STEP, MGBrain::Config::DW);
        printf("neurons %zu synapses %zu\n", net.neurons.size(), net.synapses.size());
        return 0;
    }
    if ((argc == 7 || argc == 9) && std::string(argv[1]) == "simulate") {
        network net;
        build(argv[2], net);
        if (std::string(argv[5]) != "-") {
            net.v_init.resize(net.neurons.size());
            FILE* f = fopen(argv[5], "rb");
            if (!f || fread(net.v_init.data(), 4, net.v_init.size(), f) != net.v_init.size()) return 2;
            fclose(f);
        }
        if (atoi(argv[6])) config::enable_stdp();
        config::set_seed(env("MGB_SEED", 1));
        config::enable_fire_check();
        if (env("MGB_AUTOTUNE", 0) > 0) config::enable_autotune(env("MGB_AUTOTUNE", 0));
        const int npart = argc == 9 ? atoi(argv[7]) : 1;
        if (argc == 9 && std::string(argv[8]) == "single") config::enable_single_gpu();
        std::vector<int> part = parter::part_network(net, npart, npart > 1 ? PartType::SIMPLE : PartType::MODEL);
        mgsim sim(net, part, npart);
        sim.simulate((real)atof(argv[4]));
        std::string pre = argv[3];
        FILE* f = fopen((pre + ".state").c_str(), "wb");
        std::vector<real> v = sim.get_v();
        std::vector<int> fc = sim.get_fire_cnt();
        std::vector<real> w = sim.get_weights();
        fwrite(v.data(), 4, v.size(), f);
        fwrite(fc.data(), 4, fc.size(), f);
        fwrite(w.data(), 4, w.size(), f);
        fclose(f);
        f = fopen((pre + ".raster").c_str(), "wb");
        const auto& c = sim.spike_counts();
        const auto& ids = sim.spike_ids();
        long long st = (long long)c.size();
        fwrite(&st, 8, 1, f);
        fwrite(c.data(), 8, c.size(), f);
        fwrite(ids.data(), 4, ids.size(), f);
        fclose(f);
        printf("steps %lld time %.6f handles %d\n", sim.get_steps(), sim.get_time(), sim.get_handles());
        return 0;
    }
    fprintf(stderr, "usage: api_driver gen|simulate ...\n");
    return 2;
}
