/*
 * Test infrastructure: a line-based model description applied through the
 * MGBrain Model API.  The same text drives the reference's Model
 * (src/model/model.h:45-63) in the reference driver and mgbrain_b200's Model
 * in the C++ test programs, so both generate their networks from identical
 * API calls.  Names resolve in namespace MGBrain, whichever implementation
 * was included first.
 *
 *   timestep <seconds>                 Config::set_timestep
 *   dw <value>                         Config::set_dw
 *   shuffle 1                          Config::enable_shuffle_gen
 *   lifconst <30 floats>               Model::set_lif_const
 *   life_const <10 floats>             Model::set_lif_const(ConstGen::gen_life_const(...))
 *   stdpconst <6 floats>               Model::set_stdp_const
 *   pop <num> <TYPE> <source 0|1>      Model::create_pop
 *   conn <src> <tar> <wmin> <wmax> <dmin> <dmax> <ctype> <STATIC|STDP>
 *                                      Model::connect (wrange, drange form)
 *   maker brunel|vogel <nsyn>          ModelMaker::make_brunel / make_vogel
 *   rate <pop> <per-step probability>  (applied to the Network after gen_net)
 * With MGB_SPEC_EXTENSIONS defined (mgbrain_b200's Model only):
 *   fixed_indegree <src> <tar> <k> <w> <dmin> <dmax> <seed> <STATIC|STDP>
 *                                      Model::connect_fixed_indegree
 *   all_but_self <src> <tar> <wmin> <wmax> <dmin> <dmax> <STATIC|STDP>
 *                                      Model::connect_all_but_self
 */
#pragma once
#include <array>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace mgb_spec {

inline MGBrain::NeuronType parse_type(const std::string& s)
{
    if (s == "RAW") return MGBrain::NeuronType::RAW;
    if (s == "LIF0") return MGBrain::NeuronType::LIF0;
    if (s == "POISSON") return MGBrain::NeuronType::POISSON;
    if (s == "LIF") return MGBrain::NeuronType::LIF;
    if (s == "LIFE") return MGBrain::NeuronType::LIFE;
    if (s == "LIFB") return MGBrain::NeuronType::LIFB;
    throw std::runtime_error("unknown neuron type " + s);
}

struct Applied {
    std::vector<std::pair<int, float>> rates;  // (pop id, per-step probability)
};

template <class ModelT>
Applied apply(const std::string& text, ModelT& m)
{
    Applied out;
    std::vector<MGBrain::Population> pops;
    std::istringstream in(text);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string kw;
        if (!(ls >> kw) || kw[0] == '#') continue;
        if (kw == "timestep") {
            float dt; ls >> dt;
            MGBrain::Config::set_timestep(dt);
        } else if (kw == "dw") {
            float dw; ls >> dw;
            MGBrain::Config::set_dw(dw);
        } else if (kw == "shuffle") {
            int on; ls >> on;
            if (on) MGBrain::Config::enable_shuffle_gen();
        } else if (kw == "lifconst") {
            std::array<MGBrain::real, 30> c{};
            for (auto& x : c) ls >> x;
            m.set_lif_const(c);
        } else if (kw == "life_const") {
            float a[10];
            for (auto& x : a) ls >> x;
            m.set_lif_const(MGBrain::ConstGen::gen_life_const(a[0], a[1], a[2], a[3], a[4], a[5],
                                                              a[6], a[7], a[8], a[9]));
        } else if (kw == "stdpconst") {
            std::array<MGBrain::real, 6> c{};
            for (auto& x : c) ls >> x;
            m.set_stdp_const(c);
        } else if (kw == "pop") {
            int num, src; std::string t;
            ls >> num >> t >> src;
            pops.push_back(m.create_pop(num, parse_type(t), src != 0));
        } else if (kw == "conn") {
            int s, t; float wmin, wmax, dmin, dmax, ctype; std::string st;
            ls >> s >> t >> wmin >> wmax >> dmin >> dmax >> ctype >> st;
            MGBrain::SynapseType stype =
                st == "STDP" ? MGBrain::SynapseType::STDP : MGBrain::SynapseType::STATIC;
            m.connect(pops.at(s), pops.at(t), std::array<MGBrain::real, 2>{wmin, wmax},
                      std::array<MGBrain::real, 2>{dmin, dmax}, ctype, stype);
        } else if (kw == "maker") {
            std::string which; long long nsyn;
            ls >> which >> nsyn;
            if (which == "brunel") MGBrain::ModelMaker::make_brunel(m, (int)nsyn);
            else if (which == "vogel") MGBrain::ModelMaker::make_vogel(m, (int)nsyn);
            else throw std::runtime_error("unknown maker " + which);
#ifdef MGB_SPEC_EXTENSIONS
        } else if (kw == "fixed_indegree") {
            int s, t, k; float w, dmin, dmax; unsigned long long seed; std::string st;
            ls >> s >> t >> k >> w >> dmin >> dmax >> seed >> st;
            m.connect_fixed_indegree(pops.at(s), pops.at(t), k, w, std::array<MGBrain::real, 2>{dmin, dmax},
                                     st == "STDP" ? MGBrain::SynapseType::STDP : MGBrain::SynapseType::STATIC,
                                     seed);
        } else if (kw == "all_but_self") {
            int s, t; float wmin, wmax, dmin, dmax; std::string st;
            ls >> s >> t >> wmin >> wmax >> dmin >> dmax >> st;
            m.connect_all_but_self(pops.at(s), pops.at(t), std::array<MGBrain::real, 2>{wmin, wmax},
                                   std::array<MGBrain::real, 2>{dmin, dmax},
                                   st == "STDP" ? MGBrain::SynapseType::STDP : MGBrain::SynapseType::STATIC);
#endif
        } else if (kw == "rate") {
            int p; float r;
            ls >> p >> r;
            out.rates.emplace_back(p, r);
        } else {
            throw std::runtime_error("unknown spec keyword " + kw);
        }
    }
    return out;
}

}  // namespace mgb_spec
