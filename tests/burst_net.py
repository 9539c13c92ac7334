"""The bursting network of mgbrain_b200.brunel.burst_network with the
fields the oracle reads (delays in seconds, the timestep)."""
import numpy as np

from mgbrain_b200 import brunel

DT = 1e-4


def build(**kw):
    net = brunel.burst_network(**kw)
    net["delay"] = (net["dsteps"] * DT).astype(np.float32)
    net["step"] = np.float32(DT)
    net["nlifconst"] = 1
    net["dw"] = np.float32(0.01)
    return net


def simulator(net, seed=3, **kw):
    return brunel.burst_simulator(net, seed=seed, **kw)
