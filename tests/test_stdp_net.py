"""The STDP network (per-projection plasticity, input rates redrawn every
350 ms, LIFB leak override) through the CUDA core against the oracle, and
the oracle's fp32 path against its fp64 twin."""
import numpy as np
import pytest

import mgb_testlib as T
import mgbrain_b200 as mgb
import stdp_net

RTOL = 1e-5


def oracle_net(net):
    return dict(n=net["n"], type=net["type"], rate=np.zeros(net["n"], np.float32),
                src=net["src"], tar=net["tar"], weight=net["weight"],
                delay=np.full(len(net["src"]), stdp_net.DT, np.float32), step=np.float32(stdp_net.DT),
                nlifconst=1, lifconst=net["lifconst"], nstdpconst=1, stdpconst=net["stdpconst"])


def run_oracle(net, epochs, precision=T.F32):
    o = T.OracleSim(oracle_net(net), 11, stdp=1, plastic=net["plastic"], precision=precision)
    cs, ids = [], []
    for ep in range(epochs):
        o.set_rates(stdp_net.rates(net, ep))
        c, i = o.run(stdp_net.REDRAW_STEPS)
        cs.append(c)
        ids.append(i)
    return np.concatenate(cs), np.concatenate(ids), o.state()


def test_stdp_net_fp32_vs_fp64():
    net = stdp_net.build(n_in=196, n_exc=100)
    c32, i32, s32 = run_oracle(net, 2, T.F32)
    c64, i64, s64 = run_oracle(net, 2, T.F64)
    assert c32.sum() > 50
    # population spike count within 1 % and, while rasters agree, weights
    # within fp32 rounding of the fp64 run
    assert abs(int(c32.sum()) - int(c64.sum())) <= max(1, 0.01 * c64.sum())
    if np.array_equal(c32, c64) and np.array_equal(i32, i64):
        w = s32["weight"]
        np.testing.assert_allclose(w, s64["weight"], rtol=1e-4, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["push", "pull"])
def test_stdp_net_cuda_matches_oracle(mode):
    net = stdp_net.build(n_in=784, n_exc=400)
    oc, oi, ost = run_oracle(net, 2)
    m = {"push": mgb.MODE_PUSH, "pull": mgb.MODE_PULL}[mode]
    g = mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"],
                                  net["delay"], net["lifconst"], net["stdpconst"], stdp=True,
                                  plastic=net["plastic"], seed=11, mode=m)
    assert g.info()["mode"] == m
    for ep in range(2):
        g.set_rates(stdp_net.rates(net, ep))
        g.run(stdp_net.REDRAW_STEPS)
    _, gc, gi = g.read_raster()
    assert oc.sum() > 100
    assert np.array_equal(gc, oc) and np.array_equal(gi, oi)
    w = g.weights()
    np.testing.assert_allclose(w, ost["weight32"], rtol=RTOL, atol=1e-7)
    # static synapses never change
    st = net["plastic"] == 0
    assert np.array_equal(w[st], net["weight"][st])
    np.testing.assert_allclose(g.state()["V"], ost["V32"], rtol=RTOL, atol=1e-5)
