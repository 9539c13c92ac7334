"""Edge cases of network shape and activity, each against the oracle bit for
bit: no synapses at all, a single neuron, neurons with no synapses in or out,
delays spanning more values than the delay-bucketed method takes (the ring
method runs them), every POISSON neuron firing every step, and the packing
limit of a CSR word (target bits + delay bits) refused at creation."""
import numpy as np
import pytest

import mgb_testlib as T
import mgbrain_b200 as mgb

LIF = np.zeros(30, np.float32)
LIF[0], LIF[3], LIF[4], LIF[8] = 1e-4, 0.01, 0.02, 0.002   # DT, V_reset, V_th, t_ref (LIFB)


def make_net(types, src, tar, w, delay_steps, rate=None):
    n = len(types)
    return dict(n=n, type=np.asarray(types, np.int8),
                rate=np.zeros(n, np.float32) if rate is None else np.asarray(rate, np.float32),
                src=np.asarray(src, np.int32), tar=np.asarray(tar, np.int32),
                weight=np.asarray(w, np.float32),
                delay=(np.asarray(delay_steps, np.float32) * np.float32(1e-4)).astype(np.float32),
                step=np.float32(1e-4), dw=np.float32(0.01), nlifconst=1, lifconst=LIF)


def run_both(net, steps, v0, seed=3, mode=mgb.MODE_AUTO):
    dsteps, _, _ = T.quantize_delays(net["delay"], net["step"])
    g = mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], dsteps, LIF,
                                  rate=net["rate"], v_init=v0, seed=seed, mode=mode)
    g.run(steps)
    g.sync()
    _, gc, gi = g.read_raster(max_steps=steps, max_ids=net["n"] * steps)
    gs = g.state()
    o = T.OracleSim(net, seed, v0=v0)
    oc, oi = o.run(steps)
    os_ = o.state()
    assert np.array_equal(gc, oc), "spike counts per step differ"
    assert np.array_equal(gi, oi), "spike ids differ"
    assert np.array_equal(gs["V"].view(np.int32), os_["V32"].view(np.int32)), "V not bit-exact"
    assert np.array_equal(gs["fire_cnt"], os_["fire_cnt"])
    return g, gc


@pytest.mark.gpu
def test_no_synapses():
    types = [mgb.POISSON] * 4 + [mgb.LIFB] * 7
    net = make_net(types, [], [], [], [], rate=[0.3] * 4 + [0.0] * 7)
    v0 = np.linspace(0.0, 0.025, len(types)).astype(np.float32)
    g, counts = run_both(net, 400, v0)
    assert counts.sum() > 0 and g.S == 0


@pytest.mark.gpu
def test_single_neuron():
    net = make_net([mgb.LIFB], [], [], [], [])
    g, counts = run_both(net, 200, np.array([0.03], np.float32))   # above threshold: fires once, then leaks
    assert counts.sum() == 1


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [mgb.MODE_AUTO, mgb.MODE_PUSH])
def test_isolated_neurons_and_sparse_rows(mode):
    rng = np.random.default_rng(5)
    n = 203                                   # not a multiple of 4
    types = np.full(n, mgb.LIFB, np.int8)
    types[-40:] = mgb.POISSON
    rate = np.where(types == mgb.POISSON, 0.05, 0.0).astype(np.float32)
    # only half the LIFB neurons receive, only a third of the neurons send
    senders = rng.choice(n, n // 3, replace=False)
    receivers = rng.choice(n - 40, (n - 40) // 2, replace=False)
    src = rng.choice(senders, 1500)
    tar = rng.choice(receivers, 1500)
    w = np.where(src < n - 80, 6e-4, -1.5e-3).astype(np.float32)
    d = rng.integers(2, 9, 1500)
    net = make_net(types, src, tar, w, d, rate)
    v0 = rng.uniform(0, 0.02, n).astype(np.float32)
    run_both(net, 1500, v0, mode=mode)


@pytest.mark.gpu
def test_delays_beyond_the_bucketed_method():
    """3,000 delay values: more than the delay-bucketed method holds (2,048),
    so the ring method runs them, with a ring of 3,001 slots."""
    rng = np.random.default_rng(9)
    n = 120
    types = np.full(n, mgb.LIFB, np.int8)
    types[:20] = mgb.POISSON
    rate = np.where(types == mgb.POISSON, 0.1, 0.0).astype(np.float32)
    src = rng.integers(0, n, 2000)
    tar = rng.integers(20, n, 2000)
    d = np.where(rng.random(2000) < 0.5, rng.integers(1, 40, 2000), rng.integers(2900, 3001, 2000))
    w = np.full(2000, 4e-3, np.float32)
    net = make_net(types, src, tar, w, d, rate)
    v0 = rng.uniform(0, 0.02, n).astype(np.float32)
    g, counts = run_both(net, 3300, v0)
    info = g.info()
    assert info["mode"] == mgb.MODE_PUSH and info["ring_len"] == 3001
    assert info["max_delay"] == 3000


@pytest.mark.gpu
def test_every_poisson_neuron_fires_every_step():
    rng = np.random.default_rng(2)
    n = 600
    types = np.full(n, mgb.POISSON, np.int8)
    types[:100] = mgb.LIFB
    rate = np.where(types == mgb.POISSON, 1.0, 0.0).astype(np.float32)   # probability 1: always fires
    src = rng.integers(100, n, 20000)
    tar = rng.integers(0, 100, 20000)
    w = np.full(20000, 1e-5, np.float32)
    d = rng.integers(3, 12, 20000)
    net = make_net(types, src, tar, w, d, rate)
    g, counts = run_both(net, 120, np.zeros(n, np.float32))
    assert (counts >= 500).all()


@pytest.mark.gpu
def test_csr_word_limit_is_refused():
    """Target ids and delays share one 32-bit word: 2^24 neurons leave 8 bits,
    so a delay of 300 steps cannot be stored and the build says so."""
    n = 1 << 24
    pops = [(0, n - 16, mgb.LIFB), (n - 16, 16, mgb.POISSON)]
    projs = [(1, 0, 1, 1e-4, 290, 300)]
    with pytest.raises(mgb.MgcError) as e:
        mgb.Simulator.fixed_indegree(pops, projs, LIF, conn_seed=1)
    assert e.value.status == mgb.capi.MGC_ERR_INVALID
