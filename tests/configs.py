"""The benchmark configurations at their stated sizes, as model descriptions
for NetGen (the reference's generator, restated by the oracle and pinned to
the reference's own gen_net).

C0  Brunel balanced network: 8,000 exc + 2,000 inh LIFB (V_th 20 mV, V_reset
    10 mV, t_ref 2 ms, leak 0.005 = dt/tau_m), V0 ~ U[0, 20 mV), 1,000 POISSON
    inputs at 20 Hz (0.002 per step); every projection fixed-probability
    p = 0.1, J = +0.1 mV (exc and input), -0.5 mV (inh, g = 5), delay 1.5 ms;
    dt 0.1 ms, 1 s.  The reference's LIFB kernel is the LIF of this config
    (its LIF0 has no update branch), weights and thresholds in volts.
C1  Vogels-Abbott-style network: 3,200 exc + 800 inh LIF with V shifted by
    +60 mV (V_rest -60 -> 0, V_th -50 -> 10 mV, V_reset -60 -> 0, t_ref 5 ms),
    p = 0.02, +0.27 mV / -4.5 mV, delay 0.1 ms (one step); 5 % of the neurons
    (200 exc) each get a POISSON input at 100 Hz (0.01 per step, 20 mV, one
    to one) for the first 50 ms; V0 ~ U[0, 10 mV); dt 0.1 ms, 10 s.
C0R a C0-shaped network (2,000 LIFB + 200 POISSON, p = 0.1) whose weights
    and delays are drawn from ranges by NetGen's rand_weight / rand_delay
    (exc ranges 0.4-0.6 mV, inh -3 to -2 mV, in steps of DW = 0.05 mV;
    delays 1.0-2.0 ms): unequal weights of one sign, the case whose fp32 sums
    depend on the order of arrival.  (rand_weight draws downwards from a
    positive floor, netgen.cpp:19-31, so the exc weights are 0.2-0.4 mV.)
C3  lives in stdp_net.py (explicit synapse lists: all-to-all, one-to-one and
    all-but-self, per-projection plasticity).
"""
import numpy as np

import mgb_testlib as T


def lif_line(dt, v_init, v_reset, v_th, t_ref):
    c = [0.0] * 30
    c[0], c[1], c[3], c[4], c[8] = dt, v_init, v_reset, v_th, t_ref
    return "lifconst " + " ".join(repr(float(np.float32(x))) for x in c)


def lifconst(dt, v_init, v_reset, v_th, t_ref):
    c = np.zeros(30, np.float32)
    c[0], c[1], c[3], c[4], c[8] = dt, v_init, v_reset, v_th, t_ref
    return c


C0_LIF = (0.0001, 0.0, 0.01, 0.02, 0.002)
C1_LIF = (0.0001, 0.0, 0.0, 0.01, 0.005)


def c0_spec(rate=0.002):
    J, G, D = 0.0001, 5.0, 0.0015
    lines = ["timestep 0.0001", lif_line(*C0_LIF),
             "pop 8000 LIFB 0", "pop 2000 LIFB 0", "pop 1000 POISSON 1"]
    for s, w in ((2, J), (0, J), (1, -G * J)):
        for t in (0, 1):
            lines.append(f"conn {s} {t} {w!r} {w!r} {D} {D} 0.1 STATIC")
    lines.append(f"rate 2 {rate!r}")
    return "\n".join(lines) + "\n"


def c1_spec():
    we, wi, d, p = 0.00027, -0.0045, 0.0001, 0.02
    lines = ["timestep 0.0001", lif_line(*C1_LIF),
             "pop 200 LIFB 0", "pop 3000 LIFB 0", "pop 800 LIFB 0", "pop 200 POISSON 1",
             f"conn 3 0 0.02 0.02 {d} {d} 0 STATIC"]   # the kick: one to one
    for s, w in ((0, we), (1, we), (2, wi)):
        for t in (0, 1, 2):
            lines.append(f"conn {s} {t} {w!r} {w!r} {d} {d} {p} STATIC")
    lines.append("rate 3 0.01")
    return "\n".join(lines) + "\n"


def c0r_spec():
    lines = ["timestep 0.0001", "dw 0.00005", lif_line(*C0_LIF),
             "pop 1600 LIFB 0", "pop 400 LIFB 0", "pop 200 POISSON 1"]
    for src, (lo, hi) in ((2, (0.0004, 0.0006)), (0, (0.0004, 0.0006)), (1, (-0.003, -0.002))):
        for t in (0, 1):
            lines.append(f"conn {src} {t} {lo!r} {hi!r} 0.001 0.002 0.1 STATIC")
    lines.append("rate 2 0.02")
    return "\n".join(lines) + "\n"


C0 = dict(spec=c0_spec(), mt=1, rnd=1, seed=1, v0=(0.0, 0.02, 11), lif=C0_LIF, seconds=1.0)
C0_DRIVEN = dict(spec=c0_spec(rate=0.01), mt=2, rnd=2, seed=2, v0=(0.0, 0.02, 12), lif=C0_LIF, seconds=0.3)
C0R = dict(spec=c0r_spec(), mt=4, rnd=4, seed=4, v0=(0.0, 0.02, 14), lif=C0_LIF, seconds=0.2)
C1 = dict(spec=c1_spec(), mt=3, rnd=3, seed=3, v0=(0.0, 0.01, 13), lif=C1_LIF, seconds=10.0, rates_off=500)


def build(cfg):
    """(network dict as NetGen fills it, with its constants; V0; steps that
    simulate(seconds) runs for it)."""
    spec = T.parse_spec(cfg["spec"])
    net = T.oracle_netgen(spec, cfg["mt"], cfg["rnd"])
    net["lifconst"] = lifconst(*cfg["lif"])
    net["nlifconst"] = 1
    net["stdpconst"] = np.zeros(6, np.float32)
    net["nstdpconst"] = 0
    lo, hi, s = cfg["v0"]
    v0 = np.random.default_rng(s).uniform(lo, hi, net["n"]).astype(np.float32)
    _, dmin, _ = T.quantize_delays(net["delay"], net["step"])
    steps = T.oracle().mgbo_effective_steps(T.oracle().mgbo_steps_for_time(cfg["seconds"], net["step"]), dmin)
    return net, v0, int(steps)
