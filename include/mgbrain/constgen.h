// MGBrain C++ API: neuron and STDP constant sets.  Same functions, index
// map and fp32 arithmetic as src/model/constgen.h:9-160.
//
// LIFECONSTS index map: 0 DT, 1 V_INIT, 2 V_REST, 3 V_RESET, 4 V_THRESH,
// 5 C_M, 6 TAU_M, 7 I_OFFSET, 8 TAU_REFRAC, 9 (LIFB leak override, see
// mgc.h), 10 TAU_SYN_EXC, 11 TAU_SYN_INH, 12 P_EXC, 13 P_INH, 14 V_TMP,
// 15 C_EXC, 16 C_INH, 17 CM, 21 P11EXC, 22 P11INH, 23 P21EXC, 24 P21INH,
// 25 P22.  STDP set: A_LTP, A_LTD, TAU_LTP, TAU_LTD (steps), W_MAX, W_MIN.
#pragma once
#include <cmath>
#include <iostream>

#include "macro.h"

namespace MGBrain {

class ConstGen {
public:
    static std::array<real, 30> gen_life_const(real v_init, real v_rest, real v_reset, real cm, real tau_m,
                                               real tau_refrac, real tau_syn_E, real tau_syn_I, real v_thresh,
                                               real i_offset)
    {
        const real dt = Config::DT;
        real rm = 1.0f;
        if (std::fabs(cm) > 0.00001) {
            std::cout << "cm" << std::endl;
            rm = tau_m / cm;
        }
        const real cm_decay = tau_m > 0 ? std::exp(-dt / tau_m) : 0.0f;
        const real ce_decay = tau_syn_E > 0 ? std::exp(-dt / tau_syn_E) : 0.0f;
        const real ci_decay = tau_syn_I > 0 ? std::exp(-dt / tau_syn_I) : 0.0f;
        // The reference scales an offset local that it never assigns; the
        // compiled reference yields 0 there, which is used here.
        real v_tmp = 0.0f * rm + v_rest;
        v_tmp *= (1 - cm_decay);
        real c_e = rm * tau_syn_E / (tau_syn_E - tau_m);
        real c_i = rm * tau_syn_I / (tau_syn_I - tau_m);
        c_e = c_e * (ce_decay - cm_decay);
        c_i = c_i * (ci_decay - cm_decay);
        std::array<real, 30> c{};
        c[0] = dt;
        c[1] = v_init;
        c[2] = v_rest;
        c[3] = v_reset;
        c[4] = v_thresh;
        c[5] = cm;
        c[6] = tau_m;
        c[7] = i_offset;
        c[8] = tau_refrac;
        c[10] = tau_syn_E;
        c[11] = tau_syn_I;
        c[12] = c_e;
        c[13] = c_i;
        c[14] = v_tmp;
        c[15] = ce_decay;
        c[16] = ci_decay;
        c[17] = cm_decay;
        c[21] = 0.951229453f;
        c[22] = 0.967216074f;
        c[23] = 0.0799999982f;
        c[24] = 0.0599999987f;
        c[25] = 0.90483743f;
        return c;
    }
    static std::array<real, 30> gen_lif0_const(real v_init, real v_rest, real v_reset, real cm, real tau_m,
                                               real tau_refrac, real tau_syn_E, real tau_syn_I, real v_thresh,
                                               real i_offset)
    {
        std::array<real, 30> c{};
        c[0] = Config::DT;
        c[1] = v_init;
        c[2] = v_rest;
        c[3] = v_reset;
        c[4] = v_thresh;
        c[5] = cm;
        c[6] = tau_m;
        c[7] = i_offset;
        c[8] = tau_refrac;
        c[10] = tau_syn_E;
        c[11] = tau_syn_I;
        c[12] = 0.9999f;
        c[13] = 0.9999f;
        c[15] = 0.9999f;
        c[16] = 0.9999f;
        c[21] = 0.951229453f;
        c[22] = 0.967216074f;
        c[23] = 0.0799999982f;
        c[24] = 0.0599999987f;
        c[25] = 0.90483743f;
        return c;
    }
    // Vogels-Abbott LIFE set
    static std::array<real, 30> gen_life_const1()
    {
        return gen_life_const(-0.06f, -0.06f, -0.06f, 0, 0, 0.005f, 1, 1, -0.05f, 0);
    }
    // Brunel LIFB set: threshold 20 mV, refractory 2 ms
    static std::array<real, 30> gen_life_const2()
    {
        return gen_life_const(0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.002f, 1.0f, 1.0f, 0.02f, 0.0f);
    }
    static std::array<real, 30> gen_life_const3()
    {
        return gen_life_const(0.0f, 0.0f, 0.0f, 0.25f, 10.0f, 0.0004f, 1.0f, 1.0f, 15.0f, 0.0f);
    }
    static std::array<real, 6> gen_stdp_const(real a_ltp, real a_ltd, real tau_ltp, real tau_ltd, real w_max,
                                              real w_min)
    {
        return {a_ltp, a_ltd, tau_ltp, tau_ltd, w_max, w_min};
    }
    static std::array<real, 6> gen_stdp_const1() { return {0.1f, -0.01f, 17, 34, 40, 0}; }
    static std::array<real, 6> gen_stdp_const2() { return {}; }
};

}  // namespace MGBrain
