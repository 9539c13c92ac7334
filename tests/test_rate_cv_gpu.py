"""Population rate and CV of the inter-spike intervals over a full run agree
within 1 % between the CUDA core and the oracle where rasters may drift apart:
the STDP network (weights follow CUDA expf vs libm expf, so the two runs can
separate after many updates), for both delivery methods."""
import numpy as np
import pytest

import mgb_testlib as T
import mgbrain_b200 as mgb
import stdp_net

EPOCHS = 8


rate_and_cv = T.rate_and_cv


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [mgb.MODE_PUSH, mgb.MODE_PULL])
def test_rate_and_cv_over_full_run(mode):
    net = stdp_net.build(n_in=784, n_exc=400)
    o = T.OracleSim(dict(n=net["n"], type=net["type"], rate=np.zeros(net["n"], np.float32),
                         src=net["src"], tar=net["tar"], weight=net["weight"],
                         delay=np.full(len(net["src"]), stdp_net.DT, np.float32), step=np.float32(stdp_net.DT),
                         nlifconst=1, lifconst=net["lifconst"], nstdpconst=1, stdpconst=net["stdpconst"]),
                    11, stdp=1, plastic=net["plastic"], nthreads=8)
    g = mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], net["delay"],
                                  net["lifconst"], net["stdpconst"], stdp=True, plastic=net["plastic"], seed=11,
                                  mode=mode, raster_steps=EPOCHS * stdp_net.REDRAW_STEPS + 1)
    oc, oi = [], []
    for ep in range(EPOCHS):
        r = stdp_net.rates(net, ep)
        o.set_rates(r)
        c, i = o.run(stdp_net.REDRAW_STEPS)
        oc.append(c)
        oi.append(i)
        g.set_rates(r)
        g.run(stdp_net.REDRAW_STEPS)
    _, gc, gi = g.read_raster(max_ids=net["n"] * EPOCHS * stdp_net.REDRAW_STEPS // 4)
    oc, oi = np.concatenate(oc), np.concatenate(oi)
    steps = EPOCHS * stdp_net.REDRAW_STEPS
    r_o, cv_o, k_o = rate_and_cv(oc, oi, net["n"], steps, stdp_net.DT)
    r_g, cv_g, k_g = rate_and_cv(gc, gi, net["n"], steps, stdp_net.DT)
    assert k_o > 100 and r_o > 0
    assert abs(r_g - r_o) <= 0.01 * r_o, (r_g, r_o)
    assert abs(cv_g - cv_o) <= 0.01 * cv_o, (cv_g, cv_o)
