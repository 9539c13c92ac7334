// MGBrain C++ API: Config storage, Model, NetGen.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <thread>

#include "mgbrain/constgen.h"
#include "mgbrain/mt19937.h"
#include "mgc.h"
#include "mgbrain/netgen.h"

#ifndef __CUDACC__  // the core's Philox header, here compiled for the host only
#define __host__
#define __device__
#define __forceinline__ inline
#endif
#include "../philox.cuh"

namespace MGBrain {

// Defaults of src/macro.cpp:3-14, plus the additions.
real Config::STEP = 0.001f;
real Config::DT = 0.001f;
real Config::DW = 0.01f;
bool Config::STDP = false;
bool Config::SINGLE_GPU = false;
bool Config::PEER_ACCESS = true;
bool Config::SHUFFLE_GEN = false;
bool Config::FIRE_CHECK = false;
bool Config::DENSE_SPIKE = false;
bool Config::STAGGERED = false;
float Config::MIN_GPUMEM = 3.0f;
bool Config::SEQUENCE = false;
long long Config::SEED = -1;
long long Config::NETGEN_SEED = -1;
int Config::DEVICE = 0;
bool Config::THROW_ON_ERROR = false;
bool Config::STDP_BY_TYPE = false;
int Config::NETGEN_THREADS = 0;
long long Config::NETGEN_PARALLEL_PAIRS = 1LL << 24;
bool Config::DEVICE_NETGEN = false;
long long Config::AUTOTUNE_STEPS = 0;

Model::Model() { indexer = 0; }

void Model::set_lif_const(std::array<real, 30> c)
{
    nlifconst = true;
    lifconst = c;
}

void Model::set_stdp_const(std::array<real, 6> c)
{
    nstdpconst = true;
    stdpconst = c;
}

Population& Model::create_pop(int num, NeuronType type, bool isSource)
{
    pops.emplace_back(indexer++, num, isSource, type);
    return pops.back();
}

// src/model/model.cpp:86-111: a one-to-one projection needs equal sizes; a
// repeated (src, tar) pair replaces the last matching projection only when
// that projection is not the first one (index > 0), else it is appended.
bool Model::connect(Population& src, Population tar, std::array<real, 2> w, std::array<real, 2> d, float ctype,
                    SynapseType stype)
{
    if (ctype == 0.0 && src.num != tar.num) return false;
    int last = -1;
    for (int i = 0; i < (int)pros.size(); ++i)
        if (pros[i].src == src.id && pros[i].tar == tar.id) last = i;
    if (last > 0) {
        pros[last].wrange = w;
        pros[last].drange = d;
        pros[last].ctype = ctype;
        pros[last].stype = stype;
    } else {
        pros.emplace_back(src.id, tar.id, w, d, ctype, stype);
    }
    return true;
}

bool Model::connect(Population& src, Population tar, real weight, real delay, float ctype, SynapseType stype)
{
    return connect(src, tar, {weight, weight}, {delay, delay}, ctype, stype);
}

bool Model::connect(Population& src, Population tar, std::array<real, 2> w, std::array<real, 2> d, float ctype)
{
    return connect(src, tar, w, d, ctype, SynapseType::STATIC);
}

bool Model::connect(Population& src, Population tar, real weight, real delay, float ctype)
{
    return connect(src, tar, {weight, weight}, {delay, delay}, ctype, SynapseType::STATIC);
}

bool Model::connect_fixed_indegree(Population& src, Population tar, int k, real weight, std::array<real, 2> d,
                                   SynapseType stype, unsigned long long seed)
{
    if (k < 0 || (k > 0 && src.num <= 0) || d[1] < d[0]) return false;
    pros.emplace_back(src.id, tar.id, std::array<real, 2>{weight, weight}, d, 1.0f, stype);
    pros.back().rule = 1;
    pros.back().k = k;
    pros.back().seed = seed;
    return true;
}

bool Model::connect_all_but_self(Population& src, Population tar, std::array<real, 2> w, std::array<real, 2> d,
                                 SynapseType stype)
{
    pros.emplace_back(src.id, tar.id, w, d, 1.0f, stype);
    pros.back().rule = 2;
    return true;
}

// ---------------------------------------------------------------------------
// NetGen: the reference's generation algorithm (src/model/netgen.cpp),
// consuming std::mt19937 and glibc rand() in the same order.
// ---------------------------------------------------------------------------
void NetGen::rand_vector(std::vector<bool>& list, int gen_num, int max_num)
{
    list.assign(max_num, false);
    for (int i = 0; i < max_num && i < gen_num; ++i) list[i] = true;
    for (int index = max_num - 1; index > 0; --index) {
        const int j = rand() % max_num;
        const bool t = list[index];
        list[index] = list[j];
        list[j] = t;
    }
}

// Weights come in steps of Config::DW; for a range whose floor is >= 0 the
// steps go downwards from the floor (netgen.cpp:26-29).
real NetGen::rand_weight(real floor, real ceil)
{
    if (ceil == floor) return floor;
    const int range = (int)((ceil - floor) / Config::DW) + 1;
    const real step = (rand() % range) * Config::DW;
    return floor < 0 ? floor + step : floor - step;
}

real NetGen::rand_delay(real floor, real ceil)
{
    if (ceil == floor) return floor;
    const int range = (int)((ceil - floor) / Config::DT) + 1;
    return floor + (rand() % range) * Config::DT;
}

namespace {

// draw % max_num for 32-bit draws: the draw itself when max_num exceeds
// every draw, else Lemire's remainder by multiplication ("Faster remainder by
// direct computation", 2019), exact for 32-bit operands.
struct DrawMod {
    explicit DrawMod(size_t max_num)
        : big(max_num > 0xffffffffull), d((uint32_t)max_num), M(big ? 0 : UINT64_MAX / (uint32_t)max_num + 1)
    {
    }
    uint64_t operator()(uint32_t a) const
    {
        if (big) return a;
        const uint64_t low = M * a;
        return (uint64_t)(((unsigned __int128)low * d) >> 64);
    }
    bool big;
    uint32_t d;
    uint64_t M;
};

// Pairs [lo, hi) of the fixed-probability rule, drawing from g: pair k is
// taken when its draw % max_num < limit, until out holds cap pairs.  Leaves g
// after the draws consumed (one per pair up to the cap-th taken).  Draws come
// in blocks; the block that reaches the cap is redrawn from its start up to
// the last pair it took.
void scan_pairs(Mt19937& g, size_t lo, size_t hi, size_t max_num, double limit, size_t cap,
                std::vector<size_t>& out)
{
    constexpr size_t kBlock = 4096;
    uint32_t buf[kBlock];
    const DrawMod mod(max_num);
    for (size_t k = lo; k < hi && out.size() < cap;) {
        const size_t n = std::min(kBlock, hi - k);
        const Mt19937 at_start = g;
        g.generate(buf, n);
        for (size_t j = 0; j < n; ++j)
            if ((double)mod(buf[j]) < limit) {
                out.push_back(k + j);
                if (out.size() == cap) {
                    g = at_start;
                    g.discard(j + 1);
                    return;
                }
            }
        k += n;
    }
}

// The fixed-probability rule's candidate pairs (netgen.cpp): pair k of the
// row-major order is taken, while fewer than gen_num are taken, when the
// k-th draw of rng satisfies draw % max_num < limit.  Returns the taken
// pairs (the first gen_num in order) and leaves rng after the draws the rule
// consumed (one per pair until the gen_num-th is taken).  With more than one
// thread the pairs are cut into equal stretches, each thread starts from the
// generator jumped ahead to its stretch (MtJump) and takes its pairs as if
// none had been taken before; the stretches' pairs are then joined in order
// and cut at gen_num, which is the sequential result.
std::vector<size_t> draw_pairs(Mt19937& rng, size_t max_num, size_t gen_num, double limit)
{
    std::vector<size_t> picked;
    picked.reserve(gen_num);
    unsigned threads = Config::NETGEN_THREADS > 0 ? (unsigned)Config::NETGEN_THREADS
                                                  : std::max(1u, std::thread::hardware_concurrency());
    if (threads <= 1 || gen_num == 0 || max_num == 0 || (long long)max_num < Config::NETGEN_PARALLEL_PAIRS) {
        scan_pairs(rng, 0, max_num, max_num, limit, gen_num, picked);
        return picked;
    }
    const size_t T = std::min<size_t>(threads, max_num);
    const size_t C = (max_num + T - 1) / T;
    std::vector<Mt19937> start(T, rng);
    const MtJump jump(C);
    for (size_t k = 1; k < T; ++k) {
        start[k] = start[k - 1];
        jump.apply(start[k]);
    }
    std::vector<std::vector<size_t>> local(T);
    std::vector<std::thread> pool;
    for (size_t k = 0; k < T; ++k)
        pool.emplace_back([&, k] {
            Mt19937 g = start[k];
            const size_t lo = k * C, hi = std::min(max_num, lo + C);
            if (lo < hi) scan_pairs(g, lo, hi, max_num, limit, gen_num, local[k]);
        });
    for (auto& th : pool) th.join();
    size_t consumed = max_num;  // draws the sequential rule makes
    for (size_t k = 0; k < T && picked.size() < gen_num; ++k)
        for (size_t idx : local[k]) {
            picked.push_back(idx);
            if (picked.size() == gen_num) {
                consumed = idx + 1;
                break;
            }
        }
    const size_t kc = (consumed - 1) / C;  // the stretch of the last draw consumed
    rng = start[kc];
    rng.discard(consumed - kc * C);
    return picked;
}

void add_synapse(Network& net, int src, int tar, real w, real d, SynapseType stype)
{
    net.synapses.emplace_back(src, tar, w, d);
    net.neurons[src].nxt.push_back(tar);
    net.neurons[tar].pre.push_back(src);
    net.neurons[src].syns.push_back(net.synapses.size());
    net.plastic.push_back(stype == SynapseType::STDP ? 1 : 0);
}

// add_synapse for the pairs (m, n) = (picked[t] / tn, picked[t] % tn) of
// populations sp -> tp, in order: the synapses and their weight and delay
// draws (glibc rand(), in the reference's order) one after the other; then
// the per-neuron lists, each reserved once, filled by threads that own the
// neurons by id, each neuron's entries in synapse order.  The same Network
// as calling add_synapse pair by pair.
void add_pairs(Network& net, const Pop& sp, const Pop& tp, const std::vector<size_t>& picked, real w0, real w1,
               real d0, real d1, SynapseType stype)
{
    const size_t G = picked.size(), base = net.synapses.size();
    const size_t tn = (size_t)tp.num;
    net.synapses.reserve(base + G);
    net.plastic.reserve(net.plastic.size() + G);
    for (size_t t = 0; t < G; ++t) {
        const real w = NetGen::rand_weight(w0, w1);
        const real d = NetGen::rand_delay(d0, d1);
        net.synapses.emplace_back(sp.neurons[picked[t] / tn], tp.neurons[picked[t] % tn], w, d);
        net.plastic.push_back(stype == SynapseType::STDP ? 1 : 0);
    }
    std::vector<uint32_t> out_n(net.neurons.size(), 0), in_n(net.neurons.size(), 0);
    for (size_t t = 0; t < G; ++t) {
        ++out_n[net.synapses[base + t].src];
        ++in_n[net.synapses[base + t].tar];
    }
    for (size_t i = 0; i < net.neurons.size(); ++i) {
        Neuron& nr = net.neurons[i];
        if (out_n[i]) {
            nr.nxt.reserve(nr.nxt.size() + out_n[i]);
            nr.syns.reserve(nr.syns.size() + out_n[i]);
        }
        if (in_n[i]) nr.pre.reserve(nr.pre.size() + in_n[i]);
    }
    unsigned T = Config::NETGEN_THREADS > 0 ? (unsigned)Config::NETGEN_THREADS
                                            : std::max(1u, std::thread::hardware_concurrency());
    if ((long long)G < Config::NETGEN_PARALLEL_PAIRS / 16) T = 1;
    auto fill = [&](unsigned part) {
        for (size_t t = 0; t < G; ++t) {
            const Synapse& s = net.synapses[base + t];
            if ((unsigned)s.src % T == part) {
                net.neurons[s.src].nxt.push_back(s.tar);
                net.neurons[s.src].syns.push_back(base + t + 1);
            }
            if ((unsigned)s.tar % T == part) net.neurons[s.tar].pre.push_back(s.src);
        }
    };
    if (T == 1) {
        fill(0);
        return;
    }
    std::vector<std::thread> pool;
    for (unsigned p = 0; p < T; ++p) pool.emplace_back(fill, p);
    for (auto& th : pool) th.join();
}

// Config::DEVICE_NETGEN: the projections as the device generator takes
// them (mgc_gen_proj), with the weights and delays gen_net draws with rand()
// for ranged projections drawn here, in the same order (one rand_weight and
// one rand_delay per synapse, projection after projection), so the rand()
// stream advances as gen_net's does; the mt19937 draws of the
// fixed-probability rule happen on the device, from the state recorded here.
void record_recipe(Network& net, const Model& model, const Mt19937& rng)
{
    Network::GenRecipe& rc = net.recipe;
    rc = Network::GenRecipe{};
    rc.active = true;
    rng.state_words(rc.mt.data());
    for (size_t pi = 0; pi < model.pros.size(); ++pi) {
        const Projection& pr = model.pros[pi];
        const size_t sn = (size_t)net.pops[pr.src].num, tn = (size_t)net.pops[pr.tar].num;
        const real w0 = pr.wrange[0], w1 = pr.wrange[1], d0 = pr.drange[0], d1 = pr.drange[1];
        Network::GenProjection g;
        g.src = pr.src;
        g.tar = pr.tar;
        g.plastic = pr.stype == SynapseType::STDP;
        g.weight = w0;
        g.delay = (int)std::round(d0 / Config::STEP);  // build_multinet's rounding (mgsim.cpp:49)
        size_t count = 0;
        if (pr.rule == 1) {
            g.rule = MGC_RULE_FIXED_INDEGREE;
            g.k = pr.k;
            g.seed = pr.seed;
            g.delay_max = (int)std::round(d1 / Config::STEP);
            count = tn * (size_t)pr.k;
        } else if (pr.rule == 2) {
            g.rule = MGC_RULE_ALL_BUT_SELF;
            count = sn * tn - std::min(sn, tn);
        } else if (pr.ctype == 1.0) {
            g.rule = MGC_RULE_ALL;
            count = sn * tn;
        } else if (pr.ctype == 0.0) {
            g.rule = MGC_RULE_ONE;
            count = sn;
        } else if (pr.ctype > 0.0 && pr.ctype < 1.0) {
            g.rule = MGC_RULE_PROB;
            g.prob = pr.ctype;
            const size_t max_num = sn * tn;
            count = static_cast<size_t>(std::round(max_num * pr.ctype));
        } else {
            continue;  // gen_net makes no synapses for it
        }
        g.delay_max = std::max(g.delay_max, g.delay);
        if (g.rule != MGC_RULE_FIXED_INDEGREE && (w1 != w0 || d1 != d0)) {
            if (w1 != w0) g.weights.reserve(count);
            if (d1 != d0) g.delays.reserve(count);
            for (size_t t = 0; t < count; ++t) {
                const real w = NetGen::rand_weight(w0, w1);
                const real d = NetGen::rand_delay(d0, d1);
                if (w1 != w0) g.weights.push_back(w);
                if (d1 != d0) g.delays.push_back((int)std::round(d / Config::STEP));
            }
        }
        rc.synapses += (long long)count;
        rc.projs.push_back(std::move(g));
    }
}

}  // namespace

void NetGen::gen_net(Network& net, Model& model)
{
    const unsigned long seed = Config::NETGEN_SEED >= 0
                                   ? (unsigned long)Config::NETGEN_SEED
                                   : (unsigned long)std::chrono::system_clock::now().time_since_epoch().count();
    Mt19937 rng((uint32_t)seed);  // std::mt19937's outputs for the same seed
    net.nlifconst = model.nlifconst;
    net.nstdpconst = model.nstdpconst;
    net.lifconst = model.lifconst;
    net.stdpconst = model.stdpconst;
    // neurons: population after population, ids in creation order
    net.pops.reserve(net.pops.size() + model.pops.size());
    int next_id = 0;
    for (const Population& p : model.pops) {
        net.pops.emplace_back(p.id, p.num, p.source, p.type);
        net.neurons.reserve(net.neurons.size() + p.num);
        for (int j = 0; j < p.num; ++j) {
            net.pops.back().neurons[j] = next_id;
            net.neurons.emplace_back(next_id, p.source, p.type);
            ++next_id;
        }
    }
    model.indexer = next_id;
    net.recipe = Network::GenRecipe{};
    if (Config::DEVICE_NETGEN) {
        if (!Config::SHUFFLE_GEN) {
            record_recipe(net, model, rng);
            return;
        }
        std::cerr << "mgbrain_b200: the shuffle placement is drawn on the host; NetGen lists the synapses"
                  << std::endl;
    }

    for (size_t pi = 0; pi < model.pros.size(); ++pi) {
        const Projection& pr = model.pros[pi];
        const Pop& sp = net.pops[pr.src];
        const Pop& tp = net.pops[pr.tar];
        const int sn = sp.num, tn = tp.num;
        const real w0 = pr.wrange[0], w1 = pr.wrange[1], d0 = pr.drange[0], d1 = pr.drange[1];
        if (pr.rule == 1) {
            // fixed in-degree, the device generator's draws (delays in steps)
            const int dmin = (int)std::round(d0 / Config::STEP), dmax = (int)std::round(d1 / Config::STEP);
            const uint32_t span = (uint32_t)(dmax - dmin + 1);
            net.synapses.reserve(net.synapses.size() + (size_t)tn * pr.k);
            for (int n = 0; n < tn; ++n) {
                const int t = tp.neurons[n];
                for (int j = 0; j < pr.k; ++j) {
                    const mgc::U32x4 r = mgc::conn_draw(pr.seed, (uint32_t)t, (uint32_t)j, (uint32_t)pi);
                    const int s = sp.neurons[mgc::scale_u32(r.x, (uint32_t)sn)];
                    const int steps = dmin + (int)mgc::scale_u32(r.y, span);
                    add_synapse(net, s, t, w0, (real)steps * Config::STEP, pr.stype);
                }
            }
            continue;
        }
        if (pr.rule == 2) {
            net.synapses.reserve(net.synapses.size() + (size_t)sn * tn);
            for (int m = 0; m < sn; ++m)
                for (int n = 0; n < tn; ++n) {
                    if (m == n) continue;
                    const real w = rand_weight(w0, w1);
                    const real d = rand_delay(d0, d1);
                    add_synapse(net, sp.neurons[m], tp.neurons[n], w, d, pr.stype);
                }
            continue;
        }
        if (pr.ctype == 1.0) {
            net.synapses.reserve(net.synapses.size() + (size_t)sn * tn);
            for (int m = 0; m < sn; ++m)
                for (int n = 0; n < tn; ++n) {
                    const real w = rand_weight(w0, w1);
                    const real d = rand_delay(d0, d1);
                    add_synapse(net, sp.neurons[m], tp.neurons[n], w, d, pr.stype);
                }
        } else if (pr.ctype == 0.0) {
            for (int k = 0; k < sn; ++k) {
                const real w = rand_weight(w0, w1);
                const real d = rand_delay(d0, d1);
                add_synapse(net, sp.neurons[k], tp.neurons[k], w, d, pr.stype);
            }
        } else if (pr.ctype > 0.0 && pr.ctype < 1.0) {
            if (Config::SHUFFLE_GEN) {
                // exactly round(sn*tn*p) pairs placed by a rand()-driven
                // shuffle (std::random_shuffle in libstdc++: position i swaps
                // with rand() % (i+1))
                const size_t len = (size_t)(int)(sn * tn);
                const size_t gen_num = (size_t)std::round(len * pr.ctype);
                std::vector<bool> chosen(len);
                for (size_t k = 0; k < len; ++k) chosen[k] = k < gen_num;
                for (size_t k = 1; k < len; ++k) {
                    const size_t j = (size_t)((long)rand() % (long)(k + 1));
                    if (j != k) {
                        const bool t = chosen[k];
                        chosen[k] = chosen[j];
                        chosen[j] = t;
                    }
                }
                for (int m = 0; m < sn; ++m)
                    for (int n = 0; n < tn; ++n)
                        if (chosen[(size_t)m * tn + n]) {
                            const real w = rand_weight(w0, w1);
                            const real d = rand_delay(d0, d1);
                            add_synapse(net, sp.neurons[m], tp.neurons[n], w, d, pr.stype);
                        }
            } else {
                // Each pair in row-major order is taken with probability
                // 1.1 p while fewer than round(sn*tn*p) are taken; the
                // remaining slots of the list stay pair (0, 0).
                const size_t max_num = (size_t)sn * (size_t)tn;
                const size_t gen_num = static_cast<size_t>(std::round(max_num * pr.ctype));
                const double limit = gen_num * 1.1;
                std::vector<size_t> picked = draw_pairs(rng, max_num, gen_num, limit);
                picked.resize(gen_num, 0);
                add_pairs(net, sp, tp, picked, w0, w1, d0, d1, pr.stype);
            }
        }
    }
}

}  // namespace MGBrain
