"""Golden cases shared by the CPU and GPU parity tests."""
import json
import os

import numpy as np

import mgb_testlib as T

GOLD = T.GOLDEN
CASES = json.load(open(os.path.join(GOLD, "cases.json")))
NAMES = sorted(CASES)


def load(name):
    c = CASES[name]
    net = T.read_netfile(os.path.join(GOLD, name + ".net"))
    v0p = os.path.join(GOLD, name + ".v0")
    v0 = np.fromfile(v0p, np.float32) if os.path.exists(v0p) else None
    return c, net, v0


def ref_outputs(name):
    """Raster and end state the reference kernels produced, or None."""
    rp = os.path.join(GOLD, name + ".ref.raster")
    sp = os.path.join(GOLD, name + ".ref.state")
    if not (os.path.exists(rp) and os.path.exists(sp)):
        return None
    c, net, _ = load(name)
    counts, ids = T.read_raster(rp)
    st = T.read_state(sp, net["n"], len(net["src"]))
    return counts, ids, st


def run_oracle(name, precision=T.F32, fx=None):
    """The oracle on a golden case; fx: fixed-point accumulation with this
    shift (the CUDA core's MGC_ACC_FIXED arithmetic)."""
    c, net, v0 = load(name)
    sim = T.OracleSim(net, c["seed"], v0=v0, stdp=c["stdp"], precision=precision)
    if fx is not None:
        sim.set_fx(fx)
    off = c.get("rates_off")
    if off:
        c1, i1 = sim.run(off)
        sim.set_rates(np.zeros(net["n"], np.float32))
        c2, i2 = sim.run(c["steps"] - off)
        counts, ids = np.concatenate([c1, c2]), np.concatenate([i1, i2])
    else:
        counts, ids = sim.run(c["steps"])
    return counts, ids, sim.state(), sim
