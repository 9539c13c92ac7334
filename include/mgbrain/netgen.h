// MGBrain C++ API: network generation.  Interface of src/model/netgen.h:9-16;
// the algorithm (including its random-number consumption) is that of
// src/model/netgen.cpp:2-229, so a given mt19937 seed and glibc rand()
// state give the reference's network synapse for synapse.
#pragma once
#include "network.h"

namespace MGBrain {

class NetGen {
public:
    static void rand_vector(std::vector<bool>& list, int gen_num, int max_num);
    static real rand_weight(real floor, real ceil);
    static real rand_delay(real floor, real ceil);
    // mt19937 seed: Config::NETGEN_SEED when >= 0, else the system clock
    // (netgen.cpp:47).  glibc rand() is used as the caller left it.
    static void gen_net(Network& net, Model& model);
};

}  // namespace MGBrain
