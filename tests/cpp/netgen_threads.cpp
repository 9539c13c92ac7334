// NetGen's fixed-probability rule on several host threads gives the network
// of one thread, synapse for synapse, and MGBrain::Mt19937 (with its
// jump-ahead) gives std::mt19937's outputs.
//   netgen_threads <spec> <threads> <min_pairs>
// prints "ok <synapses>" or the first difference.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <random>
#include <sstream>

#include "mgbrain.h"
#include "mgbrain/mt19937.h"
#define MGB_SPEC_EXTENSIONS
#include "../../oracle/mgb_spec.h"

static std::string slurp(const char* p)
{
    std::ifstream f(p);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

static void gen(const std::string& spec, network& net, int threads, long long min_pairs)
{
    config::set_netgen_seed(4242);
    config::set_netgen_threads(threads, min_pairs);
    srand(17);
    model m;
    mgb_spec::apply(spec, m);
    netgen::gen_net(net, m);
}

static int check_mt()
{
    MGBrain::Mt19937 a(12345u);
    std::mt19937 b(12345u);
    for (int i = 0; i < 200000; ++i)
        if (a() != (uint32_t)b()) {
            printf("Mt19937 differs from std::mt19937 at output %d\n", i);
            return 1;
        }
    MGBrain::Mt19937 c;
    for (int i = 0; i < 9999; ++i) c();
    if (c() != 4123659995u) {  // the C++ standard's value for the 10,000th output
        printf("Mt19937: 10,000th output wrong\n");
        return 1;
    }
    const unsigned long long jumps[] = {0, 1, 2, 396, 397, 623, 624, 625, 1247, 19936, 19937, 19938, 1000003, 7777777};
    for (unsigned long long J : jumps) {
        MGBrain::Mt19937 g(99u), h(99u);
        for (int i = 0; i < 311; ++i) g(), h();  // a ring position that is not 0
        MGBrain::MtJump(J).apply(g);
        h.discard(J);
        for (int i = 0; i < 2000; ++i)
            if (g() != h()) {
                printf("jump by %llu differs from sequential at output %d\n", J, i);
                return 1;
            }
    }
    // composition: two jumps make one
    MGBrain::Mt19937 p(7u), q(7u);
    MGBrain::MtJump(123456789).apply(p);
    MGBrain::MtJump(23456789).apply(p);
    MGBrain::MtJump(123456789ull + 23456789ull).apply(q);
    for (int i = 0; i < 2000; ++i)
        if (p() != q()) {
            printf("jump composition differs\n");
            return 1;
        }
    return 0;
}

int main(int argc, char** argv)
{
    if (argc != 4) {
        fprintf(stderr, "usage: netgen_threads <spec> <threads> <min_pairs>\n");
        return 2;
    }
    if (check_mt()) return 1;
    const std::string spec = slurp(argv[1]);
    network a, b;
    gen(spec, a, 1, 0);
    gen(spec, b, atoi(argv[2]), atoll(argv[3]));
    if (a.synapses.size() != b.synapses.size()) {
        printf("synapse counts differ: %zu vs %zu\n", a.synapses.size(), b.synapses.size());
        return 1;
    }
    for (size_t k = 0; k < a.synapses.size(); ++k) {
        const auto &x = a.synapses[k], &y = b.synapses[k];
        if (x.src != y.src || x.tar != y.tar || x.weight != y.weight || x.delay != y.delay) {
            printf("synapse %zu differs\n", k);
            return 1;
        }
    }
    // the per-neuron lists, filled by threads that own neurons by id, in
    // the order add_synapse would have appended them
    if (a.neurons.size() != b.neurons.size()) {
        printf("neuron counts differ: %zu vs %zu\n", a.neurons.size(), b.neurons.size());
        return 1;
    }
    for (size_t i = 0; i < a.neurons.size(); ++i) {
        const auto &x = a.neurons[i], &y = b.neurons[i];
        if (x.nxt != y.nxt || x.pre != y.pre || x.syns != y.syns) {
            printf("neuron %zu: nxt/pre/syns lists differ\n", i);
            return 1;
        }
    }
    printf("ok %zu\n", a.synapses.size());
    return 0;
}
