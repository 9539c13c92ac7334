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
// the destructor does not call cudaDeviceReset.
//
// npart > 1 (mgsim.cpp:337-363): with Config::enable_single_gpu() the
// reference maps every partition to device 0; here the network then runs
// as one handle on Config::DEVICE, which computes the same.  Otherwise the
// reference spreads the partitions over the GPUs; here each partition gets
// its own handle (mgc_create_partition) on device (DEVICE + p) % devices,
// and the partitions exchange spike ids every min_delay - 1 steps.  That
// needs the partition's neurons to be consecutive ids (SIMPLE and BSIM
// partitions are), static weights and a minimum delay >= 2; otherwise the
// network runs as one handle and a line on stderr says why.
//
// A Network that NetGen::gen_net recorded under Config::DEVICE_NETGEN (no
// host synapse list, Network::recipe) is generated on the device
// (mgc_create_generated) and runs as one handle.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "../mgc.h"
#include "network.h"

namespace MGBrain {

class Error : public std::runtime_error {
public:
    int status;
    Error(int st, const std::string& msg) : std::runtime_error(msg), status(st) {}
};

class MGSimulator {
    // One handle per partition (a single one covering every neuron unless
    // the partitions run separately).
    struct Piece {
        mgc_sim* sim = nullptr;
        int first = 0, count = 0, device = 0;
        int32_t* xout = nullptr;  // device: exported spike ids of a window
        int32_t* xin = nullptr;   // device: every partition's ids, imported
        long long xin_cap = 0;
    };
    std::vector<Piece> pieces;
    mgc_sim* sim = nullptr;       // pieces[0].sim
    std::vector<int32_t> syn_tar; // partitions: each synapse's target (weights in synapse order)
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
    bool tuned = false;
    void check(int status, const char* what);
    void build_generated(Network& net);
    void drain_raster();
    void exchange(int steps);
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
    // Times the launch configurations and keeps the fastest, with the trial
    // steps undone (mgc_autotune_rewind); one handle only.  Simulate() calls
    // it before the first step when Config::AUTOTUNE_STEPS > 0.
    mgc_tune_report autotune(long long steps_per_trial = 640);
    // The C ABI handle (of the first partition when they run separately).
    mgc_sim* handle() { return sim; }
    // Handles the network runs on: 1, or one per partition.
    int get_handles() const { return (int)pieces.size(); }
};

}  // namespace MGBrain
