// MGBrain C++ API: the reference's canned models (src/model/maker.h:10-43):
// make_brunel = 50 % POISSON / 40 % exc / 10 % inh LIFB, p = 0.1 for six
// projections, weights scaled by 20000/pop_size, 1.6 ms delays;
// make_vogel = 80/20 LIFE, p = 0.02, 0.8 ms delays.  Same arithmetic
// (including its float/double mix) so the same sizes and weights result.
#pragma once
#include "constgen.h"
#include "model.h"

namespace MGBrain {

class ModelMaker {
public:
    static void make_brunel(Model& m, int nsyn)
    {
        const float con_prob = 0.1f;
        const int pop_size = static_cast<int>(std::sqrt((float)nsyn / (con_prob * 0.5)));
        Population p = m.create_pop(pop_size * 5 / 10, NeuronType::POISSON, true);
        Population e = m.create_pop(pop_size * 4 / 10, NeuronType::LIFB, false);
        Population i = m.create_pop(pop_size * 1 / 10, NeuronType::LIFB, false);
        const real w_exc = 0.0001 * 20000 / pop_size;
        const real w_inh = -0.0005 * 20000 / pop_size;
        const real delay = 0.0016f;
        m.set_lif_const(ConstGen::gen_life_const2());
        m.connect(p, e, w_exc, delay, con_prob);
        m.connect(p, i, w_exc, delay, con_prob);
        m.connect(e, e, w_exc, delay, con_prob);
        m.connect(e, i, w_exc, delay, con_prob);
        m.connect(i, i, w_inh, delay, con_prob);
        m.connect(i, e, w_inh, delay, con_prob);
    }
    static void make_vogel(Model& m, int nsyn)
    {
        const float con_prob = 0.02f;
        const int pop_size = static_cast<int>(std::sqrt((float)nsyn / (con_prob)));
        Population pe = m.create_pop(pop_size * 8 / 10, NeuronType::LIFE, false);
        Population pi = m.create_pop(pop_size * 2 / 10, NeuronType::LIFE, false);
        const real w_exc = 0.4 * 16000000 / pop_size / pop_size;
        const real w_inh = -5.1 * 16000000 / pop_size / pop_size;
        const real delay = 0.0008f;
        m.set_lif_const(ConstGen::gen_life_const1());
        m.connect(pe, pe, w_exc, delay, con_prob);
        m.connect(pe, pi, w_exc, delay, con_prob);
        m.connect(pi, pe, w_inh, delay, con_prob);
        m.connect(pi, pi, w_inh, delay, con_prob);
    }
};

}  // namespace MGBrain
