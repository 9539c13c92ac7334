"""Pull steps of the windowed step group (mgc_set_pull): a step whose
arrivals come from many (spike, delay) pairs is delivered by one pass over
every target's incoming row instead of the scattered push.  The results
are the push's bit for bit, on a bursting network (fp32 sums, one weight per
sign) and on a network with unequal weights (fixed-point sums), also when
the forms are mixed and after a checkpoint; the raster agrees with the
oracle."""
import numpy as np
import pytest

import burst_net
import configs
import mgb_testlib as T
import mgbrain_b200 as mgb

STEPS = 3000


@pytest.fixture(scope="module")
def burst():
    return burst_net.build()


def end_state(sim):
    sim.sync()
    _, c, i = sim.read_raster()
    st = sim.state()
    return c, i, st, sim.info()["events"]


def assert_same(a, b, label):
    ca, ia, sa, ea = a
    cb, ib, sb, eb = b
    assert np.array_equal(ca, cb) and np.array_equal(ia, ib), label + ": raster"
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), f"{label}: {k}"
    assert ea == eb, label + ": events"


@pytest.fixture(scope="module")
def pushed(burst):
    sim = burst_net.simulator(burst)
    sim.set_persistent(3)
    sim.set_window(8)
    sim.run(STEPS)
    out = end_state(sim)
    sim.close()
    return out


@pytest.mark.gpu
def test_burst_network_bursts(burst, pushed):
    counts = pushed[0]
    assert counts.max() > 0.3 * 10_000          # volleys of more than 30 % of the neurons
    assert (counts > 1000).sum() >= 20


@pytest.mark.gpu
def test_burst_raster_matches_oracle(burst, pushed):
    o = T.OracleSim(burst, 3, v0=burst["v0"], nthreads=8)
    oc, oi = o.run(400)
    n = int(oc.sum())
    assert n > 0
    assert np.array_equal(pushed[0][:400], oc) and np.array_equal(pushed[1][:n], oi)


@pytest.mark.gpu
@pytest.mark.parametrize("min_pairs", [1, 1500, 10**9])
@pytest.mark.parametrize("window", [8, 3])
def test_pull_steps_equal_push(burst, pushed, min_pairs, window):
    sim = burst_net.simulator(burst)
    sim.set_persistent(3)
    sim.set_window(window)
    sim.set_pull(min_pairs)
    sim.run(STEPS)
    assert_same(end_state(sim), pushed, f"pull >= {min_pairs}, window {window}")
    sim.close()


@pytest.mark.gpu
def test_pull_steps_mixed_with_other_forms(burst, pushed):
    """Runs of the other forms in between (which write no bitmaps) restart
    the span the pull may read; checkpoints drop it."""
    sim = burst_net.simulator(burst)
    sim.set_pull(1)
    plan = [(3, 8, 701), (0, None, 64), (3, 8, 300), (2, None, 37), (3, 5, 201), (1, None, 3), (3, 8, 555)]
    done = 0
    for mode, window, steps in plan:
        sim.set_persistent(mode)
        if window:
            sim.set_window(window)
        sim.run(steps)
        done += steps
    blob = sim.checkpoint()
    fresh = burst_net.simulator(burst)
    fresh.set_pull(1)
    fresh.restore(blob)
    fresh.set_persistent(3)
    fresh.set_window(8)
    fresh.run(STEPS - done)
    sim.set_persistent(3)
    sim.run(STEPS - done)
    a = end_state(sim)
    assert_same(a, pushed, "mixed")
    b = end_state(fresh)
    n_done = int(pushed[0][:done].sum())
    assert np.array_equal(b[0], pushed[0][done:]) and np.array_equal(b[1], pushed[1][n_done:])
    assert np.array_equal(b[2]["V"], pushed[2]["V"])
    sim.close()
    fresh.close()


@pytest.mark.gpu
def test_pull_steps_fixed_point():
    """Unequal weights of one sign (C0R): fixed-point sums, pull and push
    give the same bits."""
    net, v0, steps = configs.build(configs.C0R)
    dsteps, _, _ = T.quantize_delays(net["delay"], net["step"])

    def mk():
        return mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], dsteps,
                                         T.default_lifconst(net), rate=net["rate"], v_init=v0, seed=4)
    out = []
    for pull in (0, 1):
        sim = mk()
        assert sim.info()["accumulation"] == mgb.ACC_FIXED
        sim.set_persistent(3)
        sim.set_window(sim.info()["min_delay"] if sim.info()["min_delay"] <= 8 else 8)
        sim.set_pull(pull)
        sim.run(steps)
        out.append(end_state(sim))
        sim.close()
    assert out[0][0].sum() > 100
    assert_same(out[1], out[0], "fixed point")


@pytest.mark.gpu
def test_pull_steps_refused():
    net, v0, steps = configs.build(configs.C0R)
    dsteps, _, _ = T.quantize_delays(net["delay"], net["step"])
    sim = mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], dsteps,
                                    T.default_lifconst(net), rate=net["rate"], v_init=v0, seed=4)
    sim.set_accumulation(mgb.ACC_FLOAT)   # unequal weights summed in fp32: no exact pull
    with pytest.raises(mgb.MgcError):
        sim.set_pull(10)
    with pytest.raises(mgb.MgcError):
        sim.set_pull(-1)
    sim.set_pull(0)                       # off is always allowed
    sim.close()
    c, netc, v0c = configs_c1()
    one = mgb.Simulator.from_arrays(netc["n"], netc["type"], netc["src"], netc["tar"], netc["weight"],
                                    T.quantize_delays(netc["delay"], netc["step"])[0], T.default_lifconst(netc),
                                    rate=netc["rate"], v_init=v0c, seed=3)
    with pytest.raises(mgb.MgcError):     # minimum delay 1: no windowed group
        one.set_pull(10)
    one.close()


def configs_c1():
    from cases import load
    return load("c1s")


@pytest.mark.gpu
def test_autotune_tries_pull_steps(burst):
    """The autotuner times pull thresholds on this network (it is small
    enough for a copy of its incoming rows); whatever it keeps, the end
    state is the push's."""
    sim = burst_net.simulator(burst, raster_ids=-1)
    rep = sim.autotune(steps_per_trial=640)
    assert rep["pull_min"] in (0, 11_000 // 3, 11_000 // 8, 11_000 // 20)
    assert rep["persistent"] == 3 or rep["pull_min"] == 0
    t = sim.info()["step"]
    sim.run(500)
    sim.sync()
    got = sim.state()
    sim.close()
    ref = burst_net.simulator(burst, raster_ids=-1)
    ref.set_persistent(3)
    ref.set_window(8)
    ref.run(t + 500)
    ref.sync()
    want = ref.state()
    ref.close()
    for k in want:
        assert np.array_equal(got[k], want[k]), k


@pytest.mark.gpu
def test_autotune_rewind_keeps_the_push_state(burst):
    """The autotuner with its trials undone on the bursting network (whose
    pull trials build incoming rows and spike bitmaps): the step clock and
    the end state are those of a run that never tuned (a handle that
    records no raster)."""
    sim = burst_net.simulator(burst, raster_ids=-1)
    sim.run(200)
    rep = sim.autotune(steps_per_trial=640, rewind=True)
    assert rep["trials"] >= 1 and sim.info()["step"] == 200
    sim.run(500)
    sim.sync()
    got = sim.state()
    sim.close()
    ref = burst_net.simulator(burst, raster_ids=-1)
    ref.set_persistent(3)
    ref.set_window(8)
    ref.run(700)
    ref.sync()
    want = ref.state()
    ref.close()
    for k in want:
        assert np.array_equal(got[k], want[k]), k
