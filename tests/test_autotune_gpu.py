"""mgc_autotune: the trials are real steps and the chosen launch
configuration changes no result (one weight value per sign, so every order
of the fp32 input sums gives the same bits)."""
import numpy as np
import pytest

import mgbrain_b200 as mgb
from mgbrain_b200 import brunel


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
