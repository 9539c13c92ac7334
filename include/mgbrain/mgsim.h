// MGBrain C++ API: the simulator.  Interface of
// src/simulator/mgsim/adj/mgsim.h:53-58 (MGSimulator(Network&,
// std::vector<int>&, int), simulate(real seconds), get_time()), running on
// one GPU through the C ABI in mgc.h.
//
// Behaviour kept from the reference: delays quantised to round(d/STEP)
// steps, ring length max_delay+1, simulate(t) runs round(t/STEP) steps
// minus the remainder the reference drops when that count is not a
// multiple of the minimum delay, FIRE_CHECK prints the same fire-count
// lines, errors print "Error:..." and exit(1) unless
// Config::THROW_ON_ERROR.
// Deliberate differences: a second simulate() continues from where the
// first stopped (the reference restarts its step counter, mgsim.cpp:810);
// npart > 1 runs every partition on the one GPU; the destructor does not
// call cudaDeviceReset.
#pragma once
#include <stdexcept>

#include "network.h"

struct mgc_sim;

namespace MGBrain {

class Error : public std::runtime_error {
public:
    int status;
    Error(int st, const std::string& msg) : std::runtime_error(msg), status(st) {}
};

class MGSimulator {
    mgc_sim* sim = nullptr;
    double sim_time = 0.0;
    int npart = 1;
    int min_delay = 1;
    int max_delay = 0;
    int n_neurons = 0;
    long long total_steps = 0;
    std::vector<int> part;
    std::vector<long long> raster_counts;
    std::vector<int> raster_ids;
    bool raster_complete = true;
    void check(int status, const char* what);
    void drain_raster();
    real get_firing_rate(real time);

public:
    MGSimulator(Network& net, std::vector<int>& part, int nparts);
    ~MGSimulator();
    MGSimulator(const MGSimulator&) = delete;
    MGSimulator& operator=(const MGSimulator&) = delete;
    // Advances the network by `time` seconds of simulated time.
    void simulate(real time);
    // Wall seconds of the last simulate().
    double get_time();

    // additions ------------------------------------------------------------
    // Spikes recorded since construction: counts[i] spikes in step i, ids in
    // step order, ascending within a step.
    const std::vector<long long>& spike_counts();
    const std::vector<int>& spike_ids();
    // Neuron state and weights (synapse order of the Network).
    std::vector<real> get_v();
    std::vector<int> get_fire_cnt();
    std::vector<real> get_weights();
    void set_rates(const std::vector<real>& rate);
    long long get_steps() const { return total_steps; }
    long long get_events();
    int get_min_delay() const { return min_delay; }
    int get_ring_len() const { return max_delay + 1; }
    mgc_sim* handle() { return sim; }
};

}  // namespace MGBrain
