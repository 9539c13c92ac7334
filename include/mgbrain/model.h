// MGBrain C++ API: model description (populations and projections).
// Interface of src/model/model.h:12-63.
#pragma once
#include "macro.h"

namespace MGBrain {

struct Population {
    int id;
    int num;
    bool source;
    NeuronType type;
    Population(int _id, int _num, bool _source, NeuronType _type)
        : id(_id), num(_num), source(_source), type(_type) {}
};

struct Projection {
    int src;                      // population ids
    int tar;
    std::array<real, 2> wrange;   // weight range
    std::array<real, 2> drange;   // delay range, seconds
    float ctype;                  // 0 one-to-one, 1 all-to-all, (0,1) fixed probability
    SynapseType stype;
    // Rules the reference's ctype cannot express (no reference counterpart):
    // 0 as ctype says; 1 fixed in-degree `k`; 2 all pairs but equal indices.
    int rule = 0;
    int k = 0;
    unsigned long long seed = 1;  // fixed in-degree draws
    Projection(int _src, int _tar, std::array<real, 2> _wrange, std::array<real, 2> _drange,
               float _ctype, SynapseType _stype)
        : src(_src), tar(_tar), wrange(_wrange), drange(_drange), ctype(_ctype), stype(_stype) {}
};

class Model {
public:
    std::vector<Population> pops;
    std::vector<Projection> pros;
    std::array<real, 30> lifconst{};
    bool nlifconst = false;
    std::array<real, 6> stdpconst{};
    bool nstdpconst = false;
    int indexer;

    Model();
    void set_lif_const(std::array<real, 30> lifconst);
    void set_stdp_const(std::array<real, 6> stdpconst);
    Population& create_pop(int num, NeuronType type, bool isSource = false);
    bool connect(Population& src, Population tar, std::array<real, 2> _wrange, std::array<real, 2> _drange,
                 float type, SynapseType _stype);
    bool connect(Population& src, Population tar, real weight, real delay, float type, SynapseType _stype);
    bool connect(Population& src, Population tar, std::array<real, 2> _wrange, std::array<real, 2> _drange,
                 float type);
    bool connect(Population& src, Population tar, real weight, real delay, float type);

    // Extensions, no reference counterpart.  Every neuron of `tar` gets
    // exactly `k` synapses whose sources are drawn uniformly, with
    // replacement, from `src`, weight `weight`, delay uniform in whole steps
    // of Config::STEP over drange: the draws of mgc_create_fixed_indegree
    // (Philox4x32-10 keyed by `seed`, counter (target id, draw, projection
    // index)), so the same projection built here or on the device is the
    // same set of synapses.
    bool connect_fixed_indegree(Population& src, Population tar, int k, real weight, std::array<real, 2> drange,
                                SynapseType stype = SynapseType::STATIC, unsigned long long seed = 1);
    // All pairs (i, j) of src x tar except i == j (local indices); weights
    // and delays drawn as for all-to-all.
    bool connect_all_but_self(Population& src, Population tar, std::array<real, 2> wrange,
                              std::array<real, 2> drange, SynapseType stype = SynapseType::STATIC);
};

}  // namespace MGBrain
