// MGBrain C++ API: global configuration and shared types.
//
// Same names, values and meanings as the reference's src/macro.h:29-171 so
// that programs written against MGBrain compile unchanged; the additions
// (seeds, device, error mode) are marked.
#pragma once

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <iostream>
#include <random>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

namespace MGBrain {

const float CONN_TYPE_O2O = 0;   // Projection::ctype values (src/model/model.cpp:20-45)
const float CONN_TYPE_FULL = 1;

typedef float real;              // src/macro.h:37
typedef unsigned long sid;

enum NeuronType { RAW, LIF0, POISSON, LIF, LIFE, LIFB };   // src/macro.h:40-48
enum SynapseType { STATIC, STDP };                         // src/macro.h:49-53
enum PartType { METIS, MODEL, BSIM, SIMPLE };              // src/macro.h:54-60

struct LIFConsts {
    real P22, P11exc, P11inh, P21exc, P21inh, C_m, V_reset, V_rest, V_thresh, Tau_m, Tau_exc,
        Tau_inh, I_offset, Tau_refrac;
};
struct STDPConsts {
    real A_LTP, A_LTD, TAU_LTP, TAU_LTD, W_max, W_min;
};

// Static configuration, src/macro.h:89-157 (STEP/DT in seconds).
class Config {
public:
    static real STEP;
    static real DT;
    static real DW;
    static bool STDP;
    static bool SINGLE_GPU;
    static bool PEER_ACCESS;
    static bool SHUFFLE_GEN;
    static bool FIRE_CHECK;
    static bool DENSE_SPIKE;
    static bool STAGGERED;
    static float MIN_GPUMEM;
    static bool SEQUENCE;
    // additions: fixed seeds (negative = seeded from the clock, as the
    // reference always is), device ordinal, throw instead of exit(1)
    static long long SEED;
    static long long NETGEN_SEED;
    static int DEVICE;
    static bool THROW_ON_ERROR;
    static bool STDP_BY_TYPE;    // addition: only STDP-typed projections learn
    // additions: NetGen's fixed-probability rule draws its candidate pairs on
    // this many host threads (0: all hardware threads) once a projection has
    // at least NETGEN_PARALLEL_PAIRS pairs; the network is the same
    static int NETGEN_THREADS;
    static long long NETGEN_PARALLEL_PAIRS;
    // addition: NetGen::gen_net records the projections instead of listing
    // the synapses on the host, and MGSimulator generates them on the device
    // (mgc_create_generated): the same network, without the host synapse
    // list (Network::recipe)
    static bool DEVICE_NETGEN;
    // addition: steps per trial of the autotuner that MGSimulator runs, with
    // the trials undone (mgc_autotune_rewind), before the first step of a
    // network on one handle; 0: off
    static long long AUTOTUNE_STEPS;

    static void set_timestep(real time_step)
    {
        STEP = time_step;
        DT = time_step;
    }
    static int get_steps(real time) { return (int)std::round(time * 1000 / STEP); }
    static void set_dw(real dw) { DW = dw; }
    static void enable_stdp() { STDP = true; }
    static void enable_single_gpu()
    {
        SINGLE_GPU = true;
        PEER_ACCESS = false;
    }
    static void enable_shuffle_gen() { SHUFFLE_GEN = true; }
    static void enable_fire_check() { FIRE_CHECK = true; }
    static void enable_dense_spike() { DENSE_SPIKE = true; }
    static void disable_peer_access() { PEER_ACCESS = false; }
    static void enable_staggered() { STAGGERED = true; }
    static void set_min_gpumem(float mem) { MIN_GPUMEM = mem; }
    static void enable_sequence() { SEQUENCE = true; }
    // additions
    static void set_seed(long long seed) { SEED = seed; }
    static void set_netgen_seed(long long seed) { NETGEN_SEED = seed; }
    static void set_device(int device) { DEVICE = device; }
    static void enable_autotune(long long steps_per_trial = 640) { AUTOTUNE_STEPS = steps_per_trial; }
    static void set_netgen_threads(int threads, long long min_pairs = 1LL << 24)
    {
        NETGEN_THREADS = threads;
        NETGEN_PARALLEL_PAIRS = min_pairs;
    }
    static void throw_on_error(bool on) { THROW_ON_ERROR = on; }
    static void enable_device_netgen(bool on = true) { DEVICE_NETGEN = on; }
    // With STDP on, the reference updates every synapse (mgcore.cu:365-412)
    // whatever its projection's SynapseType; this restricts it to STDP ones.
    static void enable_stdp_by_type()
    {
        STDP = true;
        STDP_BY_TYPE = true;
    }
};

// Wall-clock timer, src/macro.h:161-171.
class timer {
    std::chrono::time_point<std::chrono::high_resolution_clock> s;

public:
    timer() { s = std::chrono::high_resolution_clock::now(); }
    double stop()
    {
        using namespace std::chrono;
        return duration_cast<microseconds>(high_resolution_clock::now() - s).count() * 1e-6;
    }
};

}  // namespace MGBrain
