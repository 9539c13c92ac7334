"""mgc_autotune: the trials are real steps and the chosen launch
configuration changes no result (one weight value per sign, so every order
of the fp32 input sums gives the same bits); mgc_autotune_rewind undoes the
trials."""
import numpy as np
import pytest

import mgbrain_b200 as mgb
from mgbrain_b200 import brunel

import stdp_net


def make(n, delays, mode=mgb.MODE_AUTO):
    p = brunel.sweep_instances(count=1, n_min=n, n_max=n, seed=3)[0]
    b = brunel.sweep_block(p)
    projs = [(s, t, k, w, delays[0], delays[1]) for (s, t, k, w, _, _) in b["projs"]]
    return mgb.Simulator.fixed_indegree(b["pops"], projs, brunel.brunel_lifconst(), rate=b["rate"],
                                        v_init=b["v_init"], conn_seed=b["conn_seed"], seed=9, mode=mode)


@pytest.mark.gpu
@pytest.mark.parametrize("n,delays,mode", [(20_000, (15, 15), mgb.MODE_AUTO),
                                           (20_000, (10, 50), mgb.MODE_AUTO),
                                           (8_000, (1, 5), mgb.MODE_AUTO),
                                           (8_000, (10, 20), mgb.MODE_PUSH)])
def test_autotune_keeps_results(n, delays, mode):
    sim = make(n, delays, mode)
    rep = sim.autotune(steps_per_trial=64)
    assert rep["trials"] >= 1 and rep["ms_per_step"] > 0 and rep["default_ms_per_step"] > 0
    assert rep["ms_per_step"] <= rep["default_ms_per_step"]
    # 0: the ring method's push on a grid of fewer blocks than SMs
    assert rep["blocks_per_sm"] >= (0 if sim.info()["mode"] == mgb.MODE_PUSH else 1)
    sim.run(500)
    total = rep["steps"] + 500
    assert sim.info()["step"] == total
    _, c, i = sim.read_raster()
    ref = make(n, delays, mode)
    ref.run(total)
    _, cr, ir = ref.read_raster()
    assert np.array_equal(c, cr) and np.array_equal(i, ir)
    assert np.array_equal(sim.state()["V"], ref.state()["V"])
    assert c.sum() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("n,delays", [(20_000, (15, 15)), (20_000, (10, 50)), (8_000, (1, 5))])
def test_autotune_rewind_undoes_the_trials(n, delays):
    """mgc_autotune_rewind in the middle of a run: the step clock, raster and
    V continue as in a run that never tuned."""
    sim = make(n, delays)
    sim.run(300)
    sim.read_raster()
    rep = sim.autotune(steps_per_trial=64, rewind=True)
    assert rep["trials"] >= 1 and rep["steps"] > 0
    assert sim.info()["step"] == 300
    sim.run(500)
    f, c, i = sim.read_raster()
    ref = make(n, delays)
    ref.run(800)
    _, cr, ir = ref.read_raster()
    assert f == 300 and c.sum() > 0
    assert np.array_equal(c, cr[300:]) and np.array_equal(i, ir[cr[:300].sum():])
    assert np.array_equal(sim.state()["V"], ref.state()["V"])


@pytest.mark.gpu
def test_autotune_rewind_restores_stdp_weights():
    """With STDP the trials change the weights; the rewind puts back the
    weights and neuron state the call found."""
    net = stdp_net.build(n_in=196, n_exc=100)
    sim = mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], net["delay"],
                                    net["lifconst"], net["stdpconst"], stdp=True, plastic=net["plastic"], seed=11,
                                    mode=mgb.MODE_PUSH)
    sim.set_rates(stdp_net.rates(net, 0))
    sim.run(200)
    sim.read_raster()
    w0, s0 = sim.weights(), sim.state()
    sim.autotune(steps_per_trial=64, rewind=True)
    assert sim.info()["step"] == 200
    assert np.array_equal(sim.weights(), w0)
    for k in s0:
        assert np.array_equal(sim.state()[k], s0[k]), k
    sim.run(100)
    f, c, _ = sim.read_raster()
    assert f == 200 and len(c) == 100


@pytest.mark.gpu
def test_autotune_rewind_refuses_an_unread_raster():
    sim = make(8_000, (10, 20))
    sim.run(10)
    with pytest.raises(mgb.MgcError, match="read the raster"):
        sim.autotune(steps_per_trial=64, rewind=True)
    sim.read_raster()
    sim.autotune(steps_per_trial=64, rewind=True)
    assert sim.info()["step"] == 10
