// MGBrain C++ API: partitioning, partition statistics, CLI parameters.
#include <cmath>
#include <iostream>

#include "mgbrain/parser.h"
#include "mgbrain/parter.h"

namespace MGBrain {

namespace {

// parter.cpp:64-81: consecutive neurons until a part holds ~S/nparts synapses
void part_bsim(Network& net, int nparts, std::vector<int>& part)
{
    const size_t cap = (size_t)std::ceil(net.synapses.size() / nparts);
    size_t cur = 0;
    int p = 0;
    for (size_t i = 0; i < net.neurons.size(); ++i) {
        cur += net.neurons[i].nxt.size();
        if (cur <= cap) {
            part[i] = p;
        } else {
            cur = 0;
            if (p < nparts - 1) ++p;
        }
    }
}

// parter.cpp:82-99: equal consecutive blocks after the remainder
void part_simple(Network& net, int nparts, std::vector<int>& part)
{
    const int n = (int)net.neurons.size();
    const int zone = n / nparts;
    for (int p = 0, i = n % nparts; p < nparts; ++p)
        for (int k = 0; k < zone; ++k, ++i) part[i] = p;
}

// neuron and synapse cost weights of src/partition/calculator.cpp:3-16
int neuron_weight(NeuronType t, float rate, float syn_weights)
{
    int w = 1;
    switch (t) {
    case LIF: w = 8; break;
    case POISSON: w = 2; break;
    case LIF0: w = 4; break;
    case RAW: w = 1; break;
    case LIFB: w = 4; break;
    case LIFE: w = 6; break;
    }
    return (int)std::round(1 + w * rate + syn_weights);
}

float sd_of(const std::vector<int>& zones, float avg)
{
    float sum = 0;
    for (int z : zones) sum += (z - avg) * (z - avg);
    return std::sqrt(sum / zones.size());
}

void print_zones(const std::string& what, const std::vector<int>& zones, float sd)
{
    std::cout << what;
    for (size_t i = 0; i < zones.size(); ++i) std::cout << "(" << i << ":" << zones[i] << ")";
    std::cout << "\t Standard Deviation:" << sd << std::endl;
}

}  // namespace

std::vector<int> Partitioner::part_network(Network& network, int nparts, PartType type)
{
    std::vector<int> part(network.neurons.size(), 0);
    if (nparts <= 1) return part;
    switch (type) {
    case PartType::BSIM:
        part_bsim(network, nparts, part);
        break;
    case PartType::SIMPLE:
        part_simple(network, nparts, part);
        break;
    default:
        std::cerr << "mgbrain_b200: METIS is not linked; partitioning with SIMPLE" << std::endl;
        part_simple(network, nparts, part);
        break;
    }
    return part;
}

int PartitionAnalysis::getCostNum(bool print)
{
    int cost = 0;
    for (const Synapse& s : net.synapses) cost += part[s.src] != part[s.tar];
    if (print) std::cout << name << " part cost:" << cost << std::endl;
    return cost;
}

float PartitionAnalysis::getCostRatio(bool print)
{
    const int cost = getCostNum();
    const float r = (float)cost / (float)net.synapses.size();
    if (print) std::cout << name << " cut-rate:" << r << "(" << cost << "/" << net.synapses.size() << ")" << std::endl;
    return r;
}

float PartitionAnalysis::getZoneNeu(bool print)
{
    std::vector<int> z(nparts, 0);
    for (size_t i = 0; i < net.neurons.size(); ++i) z[part[i]]++;
    const float sd = sd_of(z, (float)net.neurons.size() / nparts);
    if (print) print_zones(name + " part zone neu:", z, sd);
    return sd;
}

float PartitionAnalysis::getZoneWgt(bool print)
{
    std::vector<int> z(nparts, 0);
    int total = 0;
    for (size_t i = 0; i < net.neurons.size(); ++i) {
        float syn = 0;
        for (size_t j = 0; j < net.neurons[i].nxt.size(); ++j) syn += 2 * 0.01f;
        const int w = neuron_weight(net.neurons[i].type, 0.5f, syn);
        z[part[i]] += w;
        total += w;
    }
    const float sd = sd_of(z, (float)total / nparts);
    if (print) print_zones(name + " part zone wgt:", z, sd);
    return sd;
}

float PartitionAnalysis::getZoneSyn(bool print)
{
    std::vector<int> z(nparts, 0);
    for (const Synapse& s : net.synapses) z[part[s.src]]++;
    const float sd = sd_of(z, (float)net.synapses.size() / nparts);
    if (print) print_zones(name + " part zone syn:", z, sd);
    return sd;
}

float PartitionAnalysis::getZoneOut(bool print)
{
    std::vector<int> z(nparts, 0);
    int total = 0;
    for (const Synapse& s : net.synapses)
        if (part[s.src] != part[s.tar]) {
            z[part[s.src]]++;
            ++total;
        }
    const float sd = sd_of(z, (float)total / nparts);
    if (print) print_zones(name + " part zone outter:", z, sd);
    return sd;
}

float PartitionAnalysis::getZoneIn(bool print)
{
    std::vector<int> z(nparts, 0);
    int total = 0;
    for (const Synapse& s : net.synapses)
        if (part[s.src] != part[s.tar]) {
            z[part[s.tar]]++;
            ++total;
        }
    const float sd = sd_of(z, (float)total / nparts);
    if (print) print_zones(name + " part zone inner:", z, sd);
    return sd;
}

void PartitionAnalysis::printAll()
{
    getCostRatio(true);
    getZoneNeu(true);
    getZoneWgt(true);
    getZoneSyn(true);
    getZoneOut(true);
    getZoneIn(true);
}

// ---------------------------------------------------------------------------
std::string ParamsParser::NSYN = "--nsyn";
std::string ParamsParser::NPART = "--npart";
std::string ParamsParser::MODEL = "--model";
std::string ParamsParser::FILE = "--file";
std::string ParamsParser::PREFIX = "--prefix";
std::string ParamsParser::RATE = "--rate";

ParamsParser::ParamsParser(int args, char* argv[])
{
    params[NSYN] = "10000";
    params[NPART] = "1";
    params[MODEL] = "model";
    params[FILE] = "tmp.txt";
    params[PREFIX] = "../../benchdata/";
    params[RATE] = "0.002";
    for (int i = 1; i < args; ++i) {
        const std::string a = argv[i];
        const size_t eq = a.find('=');
        if (eq == std::string::npos)
            params[a] = "";
        else
            params[a.substr(0, eq)] = a.substr(eq + 1);
    }
}

std::string ParamsParser::getStr(std::string name) { return params.count(name) ? params[name] : ""; }

size_t ParamsParser::getNum(std::string name)
{
    if (!params.count(name)) return (size_t)-1;
    std::stringstream ss(params[name]);
    size_t v = 0;
    ss >> v;
    return v;
}

float ParamsParser::getFloat(std::string name)
{
    if (!params.count(name)) return -1;
    std::stringstream ss(params[name]);
    float v = 0;
    ss >> v;
    return v;
}

bool ParamsParser::getBool(std::string name) { return params.count(name) && params[name] == "y"; }

}  // namespace MGBrain
