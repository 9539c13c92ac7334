"""Checkpoints: a handle that loads another's state continues exactly as the
original does (raster, V, weights), for the pipelined deferred method, the
ring method with STDP and the pull method with STDP; a checkpoint of another
network is refused."""
import numpy as np
import pytest

import mgbrain_b200 as mgb

import bench
import stdp_net


def brunel(mode):
    w = bench.workload(scale=0.03, nu=0.01)
    return mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], rate=w["rate"], v_init=w["v0"],
                                        conn_seed=4, seed=6, mode=mode)


def stdp(mode):
    net = stdp_net.build(n_in=196, n_exc=100)
    g = mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], net["delay"],
                                  net["lifconst"], net["stdpconst"], stdp=True, plastic=net["plastic"], seed=11,
                                  mode=mode)
    g.set_rates(stdp_net.rates(net, 0))
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("wide_first", [True, False])
def test_resume_across_accumulator_cycles(wide_first):
    """A checkpoint taken while windows of 8 steps run (8-buffer cycle) loads
    into a fresh handle (4-buffer cycle) and continues under the pipelined
    group, and the other way round, exactly as the uninterrupted run."""
    def form(sim, wide):
        sim.set_persistent(3 if wide else 2)
        if wide:
            sim.set_window(8)
    a = brunel(mgb.MODE_AUTO)
    form(a, wide_first)
    a.run(1203)
    a.read_raster()
    blob = a.checkpoint()
    b = brunel(mgb.MODE_AUTO)
    b.restore(blob)
    form(a, not wide_first)
    form(b, not wide_first)
    a.run(1501)
    b.run(1501)
    fa, ca, ia = a.read_raster()
    fb, cb, ib = b.read_raster()
    assert fa == fb == 1203 and ca.sum() > 0
    assert np.array_equal(ca, cb) and np.array_equal(ia, ib)
    assert np.array_equal(a.state()["V"], b.state()["V"])


@pytest.mark.gpu
@pytest.mark.parametrize("make,mode", [(brunel, mgb.MODE_AUTO), (brunel, mgb.MODE_PUSH),
                                       (stdp, mgb.MODE_PUSH), (stdp, mgb.MODE_PULL)])
def test_resume_equals_uninterrupted(make, mode):
    a = make(mode)
    a.run(1203)
    a.read_raster()
    blob = a.checkpoint()
    b = make(mode)
    b.restore(blob)
    assert b.info()["step"] == 1203
    a.run(1500)
    b.run(1500)
    fa, ca, ia = a.read_raster()
    fb, cb, ib = b.read_raster()
    assert fa == fb == 1203
    assert ca.sum() > 0
    assert np.array_equal(ca, cb) and np.array_equal(ia, ib)
    sa, sb = a.state(), b.state()
    for k in ("refrac", "last_fired", "fire_cnt"):
        assert np.array_equal(sa[k], sb[k]), k
    if make is stdp and mode == mgb.MODE_PUSH:
        # unequal (plastic) weights summed by atomics: the order, and so the
        # last bits of V, differ between any two runs, resumed or not
        np.testing.assert_allclose(sa["V"], sb["V"], rtol=1e-5, atol=1e-8)
    else:
        assert np.array_equal(sa["V"], sb["V"])
    if make is stdp:
        assert np.array_equal(a.weights(), b.weights())
    assert a.info()["events"] == b.info()["events"]


@pytest.mark.gpu
def test_checkpoint_of_another_network_is_refused():
    a = brunel(mgb.MODE_AUTO)
    blob = a.checkpoint()
    b = stdp(mgb.MODE_PUSH)
    with pytest.raises(mgb.MgcError):
        b.restore(blob)
    with pytest.raises(mgb.MgcError):
        a.restore(blob[:100])
