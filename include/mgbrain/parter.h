// MGBrain C++ API: partitioning.  Interface of src/partition/parter.h:10-36
// and src/partition/analysis.h:8-30.
//
// On one GPU a partition only orders work; npart <= 1 returns all zeros
// exactly as the reference (parter.cpp:103-104).  BSIM and SIMPLE follow
// parter.cpp:64-99.  METIS and MODEL need the METIS library, which this
// core does not link: they fall back to SIMPLE and say so on stderr.
#pragma once
#include <string>

#include "network.h"

namespace MGBrain {

class Partitioner {
public:
    static std::vector<int> part_network(Network& network, int nparts, PartType type);
};

// Cut and balance statistics of a partition (src/partition/analysis.cpp).
class PartitionAnalysis {
    std::string name;
    std::vector<int>& part;
    Network& net;
    int nparts;

public:
    PartitionAnalysis(std::string _name, std::vector<int>& _part, Network& _net, int _nparts)
        : name(_name), part(_part), net(_net), nparts(_nparts) {}
    PartitionAnalysis(std::vector<int>& _part, Network& _net, int _nparts, PartType type)
        : part(_part), net(_net), nparts(_nparts)
    {
        name = type == PartType::BSIM ? "bsim" : type == PartType::METIS ? "metis"
               : type == PartType::MODEL ? "model" : "simple";
    }
    int getCostNum(bool print = false);
    float getCostRatio(bool print = false);
    float getZoneNeu(bool print = false);
    float getZoneWgt(bool print = false);
    float getZoneSyn(bool print = false);
    float getZoneOut(bool print = false);
    float getZoneIn(bool print = false);
    void printAll();
};

}  // namespace MGBrain
