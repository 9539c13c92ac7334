// MGBrain C++ API: instantiated network.  Interface of
// src/model/network.h:9-68 plus one addition, Network::v_init.
#pragma once
#include "model.h"

namespace MGBrain {

struct Pop {
    int id;
    int num;
    bool source;
    NeuronType type;
    std::vector<int> neurons;   // neuron ids of this population
    Pop(int _id, int _num, bool _source, NeuronType _type) : id(_id), num(_num), source(_source), type(_type)
    {
        neurons.resize(_num);
    }
};

struct Neuron {
    int id;
    bool source;
    NeuronType type;
    real rate;                  // POISSON: firing probability per step
    int fire_cnt;
    std::vector<int> nxt;       // targets
    std::vector<int> pre;       // sources
    std::vector<size_t> syns;   // synapse indices + 1 (as the reference stores them)
    Neuron(int _id, bool _source, NeuronType _type) : id(_id), source(_source), type(_type)
    {
        rate = 0;
        fire_cnt = 0;
    }
};

struct Synapse {
    int src;
    int tar;
    real weight;
    real delay;                 // seconds
    Synapse(int _src, int _tar, real _weight, real _delay) : src(_src), tar(_tar), weight(_weight), delay(_delay) {}
};

class Network {
public:
    std::vector<Pop> pops;
    std::vector<Neuron> neurons;
    std::vector<Synapse> synapses;
    std::array<real, 30> lifconst{};
    std::array<real, 6> stdpconst{};
    bool nlifconst = false;
    bool nstdpconst = false;
    // addition: per-neuron initial membrane potential.  Empty means
    // lifconst[1] for every neuron, as the reference does (mgsim.cpp:97).
    std::vector<real> v_init;
    // addition: synapse-type of each synapse (STATIC/STDP) when the
    // projections should gate plasticity; empty means Config::STDP decides
    // for every synapse, as the reference does.
    std::vector<unsigned char> plastic;
    // addition: with Config::DEVICE_NETGEN, gen_net leaves `synapses` and the
    // neurons' nxt/pre/syns lists empty and records here what MGSimulator
    // generates on the device: the projections in gen_net's order, NetGen's
    // mt19937 before the first (its 624 words in logical order), and the
    // weights and delays (in steps) gen_net draws with rand() for ranged
    // projections, in synapse order.
    struct GenProjection {
        int src = 0, tar = 0;     // population indices
        int rule = 0;             // mgc_gen_proj rule (MGC_RULE_*)
        float prob = 0.0f;
        int k = 0;
        unsigned long long seed = 1;
        real weight = 0;
        int delay = 1, delay_max = 1;  // steps
        std::vector<real> weights;     // empty: every synapse has `weight`
        std::vector<int> delays;       // empty: every synapse has `delay`
        bool plastic = false;
    };
    struct GenRecipe {
        bool active = false;
        std::vector<GenProjection> projs;
        std::array<uint32_t, 624> mt{};
        long long synapses = 0;
    } recipe;
};

}  // namespace MGBrain
