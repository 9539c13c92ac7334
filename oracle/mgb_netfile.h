/*
 * Test infrastructure: binary network file shared by the reference driver,
 * the C++ test programs and the Python tests (tests/mgb_testlib.py reads it).
 * Templated over the Network type so it serialises either the reference's
 * MGBrain::Network (src/model/network.h:50-68) or mgbrain_b200's.
 *
 * Layout, little endian:
 *   char[8] "MGBNET02"
 *   int32 n_pops, int32 n_neurons, int64 n_syn
 *   float step, float dw, int32 nlifconst, int32 nstdpconst
 *   float lifconst[30], float stdpconst[6]
 *   n_pops x int32 {id, num, source, type}
 *   int8 type[n_neurons], float rate[n_neurons]
 *   int32 src[n_syn], int32 tar[n_syn], float weight[n_syn], float delay[n_syn]
 */
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace mgb_netfile {

template <class T>
static void put(FILE* f, const T* p, size_t n)
{
    if (n && fwrite(p, sizeof(T), n, f) != n) throw std::runtime_error("netfile write failed");
}

template <class NetT>
void write(const std::string& path, const NetT& net, float step, float dw)
{
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open " + path);
    put(f, "MGBNET02", 8);
    int32_t np = (int32_t)net.pops.size(), nn = (int32_t)net.neurons.size();
    int64_t ns = (int64_t)net.synapses.size();
    put(f, &np, 1); put(f, &nn, 1); put(f, &ns, 1);
    put(f, &step, 1); put(f, &dw, 1);
    int32_t nl = net.nlifconst ? 1 : 0, nsd = net.nstdpconst ? 1 : 0;
    put(f, &nl, 1); put(f, &nsd, 1);
    float lc[30], sc[6];
    for (int i = 0; i < 30; ++i) lc[i] = nl ? (float)net.lifconst[i] : 0.0f;
    for (int i = 0; i < 6; ++i) sc[i] = nsd ? (float)net.stdpconst[i] : 0.0f;
    put(f, lc, 30); put(f, sc, 6);
    for (const auto& p : net.pops) {
        int32_t rec[4] = {p.id, p.num, p.source ? 1 : 0, (int32_t)p.type};
        put(f, rec, 4);
    }
    std::vector<int8_t> ty(nn);
    std::vector<float> rate(nn);
    for (int32_t i = 0; i < nn; ++i) {
        ty[i] = (int8_t)net.neurons[i].type;
        rate[i] = (float)net.neurons[i].rate;
    }
    put(f, ty.data(), nn); put(f, rate.data(), nn);
    std::vector<int32_t> a(ns);
    std::vector<float> b(ns);
    for (int64_t k = 0; k < ns; ++k) a[k] = net.synapses[k].src;
    put(f, a.data(), ns);
    for (int64_t k = 0; k < ns; ++k) a[k] = net.synapses[k].tar;
    put(f, a.data(), ns);
    for (int64_t k = 0; k < ns; ++k) b[k] = (float)net.synapses[k].weight;
    put(f, b.data(), ns);
    for (int64_t k = 0; k < ns; ++k) b[k] = (float)net.synapses[k].delay;
    put(f, b.data(), ns);
    fclose(f);
}

/* Plain arrays read back from a file (used by the reference driver). */
struct Arrays {
    int32_t n_pops = 0, n = 0;
    int64_t S = 0;
    float step = 0, dw = 0;
    int32_t nlifconst = 0, nstdpconst = 0;
    float lifconst[30] = {}, stdpconst[6] = {};
    std::vector<int32_t> pops;  // 4 per pop
    std::vector<int8_t> type;
    std::vector<float> rate;
    std::vector<int32_t> src, tar;
    std::vector<float> weight, delay;
};

template <class T>
static void get(FILE* f, T* p, size_t n)
{
    if (n && fread(p, sizeof(T), n, f) != n) throw std::runtime_error("netfile truncated");
}

inline Arrays read(const std::string& path)
{
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    Arrays a;
    char magic[8];
    get(f, magic, 8);
    if (memcmp(magic, "MGBNET02", 8) != 0) throw std::runtime_error("bad netfile magic");
    get(f, &a.n_pops, 1); get(f, &a.n, 1); get(f, &a.S, 1);
    get(f, &a.step, 1); get(f, &a.dw, 1);
    get(f, &a.nlifconst, 1); get(f, &a.nstdpconst, 1);
    get(f, a.lifconst, 30); get(f, a.stdpconst, 6);
    a.pops.resize(4 * (size_t)a.n_pops);
    get(f, a.pops.data(), a.pops.size());
    a.type.resize(a.n); a.rate.resize(a.n);
    get(f, a.type.data(), a.n); get(f, a.rate.data(), a.n);
    a.src.resize(a.S); a.tar.resize(a.S); a.weight.resize(a.S); a.delay.resize(a.S);
    get(f, a.src.data(), a.S); get(f, a.tar.data(), a.S);
    get(f, a.weight.data(), a.S); get(f, a.delay.data(), a.S);
    fclose(f);
    return a;
}

}  // namespace mgb_netfile
