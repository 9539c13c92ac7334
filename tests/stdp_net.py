"""The STDP network (784 Poisson inputs -> 1600 exc LIFB, 1:1 exc->inh,
all-but-self inh->exc) as explicit synapse arrays, at any scale.

Units follow the reference's LIFB kernel (V in the weight units): threshold
20, reset 0, leak dt/tau_m = 0.5 ms / 20 ms = 0.025 (lifconst[9]),
refractory 5 ms; inputs are POISSON neurons whose per-step probability is
intensity * 63.75 Hz * dt with intensities U[0,1] redrawn every 350 ms.
Input->exc weights start U[0, 0.3] and are the only plastic synapses
(pair-based nearest-spike STDP of the reference, A+ 0.01, A- -0.0105,
tau 40 steps = 20 ms, clipped to [0, 1]).  Delays are one step.
"""
import numpy as np

DT = 0.0005
REDRAW_STEPS = 700          # 350 ms


def build(n_in=784, n_exc=1600, seed=0):
    rng = np.random.default_rng(seed)
    n = n_in + 2 * n_exc
    P, E, I = 0, n_in, n_in + n_exc
    types = np.array([2] * n_in + [5] * (2 * n_exc), np.int8)
    # inputs -> exc, all to all, plastic
    s1 = np.repeat(np.arange(P, P + n_in), n_exc)
    t1 = np.tile(np.arange(E, E + n_exc), n_in)
    w1 = rng.uniform(0.0, 0.3, len(s1)).astype(np.float32)
    # exc -> inh one to one
    s2 = np.arange(E, E + n_exc)
    t2 = np.arange(I, I + n_exc)
    w2 = np.full(n_exc, 25.0, np.float32)
    # inh -> exc all but own partner
    ii, ee = np.meshgrid(np.arange(n_exc), np.arange(n_exc), indexing="ij")
    keep = ii != ee
    s3 = (I + ii[keep]).astype(np.int64)
    t3 = (E + ee[keep]).astype(np.int64)
    w3 = np.full(len(s3), -17.0, np.float32)
    src = np.concatenate([s1, s2, s3]).astype(np.int32)
    tar = np.concatenate([t1, t2, t3]).astype(np.int32)
    w = np.concatenate([w1, w2, w3])
    plastic = np.concatenate([np.ones(len(s1), np.uint8), np.zeros(len(s2) + len(s3), np.uint8)])
    delay = np.ones(len(src), np.int32)
    lif = np.zeros(30, np.float32)
    lif[0], lif[3], lif[4], lif[8], lif[9] = DT, 0.0, 20.0, 0.005, 0.025
    stdp = np.array([0.01, -0.0105, 40.0, 40.0, 1.0, 0.0], np.float32)
    return dict(n=n, n_in=n_in, n_exc=n_exc, type=types, src=src, tar=tar, weight=w,
                delay=delay, plastic=plastic, lifconst=lif, stdpconst=stdp)


def rates(net, epoch, seed=1):
    """Per-step input probabilities for input epoch `epoch`."""
    r = np.zeros(net["n"], np.float32)
    inten = np.random.default_rng((seed, epoch)).uniform(0.0, 1.0, net["n_in"])
    r[:net["n_in"]] = (inten * 63.75 * DT).astype(np.float32)
    return r
