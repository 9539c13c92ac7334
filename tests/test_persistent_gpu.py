"""Persistent step groups (one cooperative launch per group, grid barrier
between steps) give the rasters and state of the graph path, also when the
two are mixed and the step count is no multiple of anything."""
import numpy as np
import pytest

import mgbrain_b200 as mgb

import bench


def make(nu):
    w = bench.workload(scale=0.03, nu=nu)
    return mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], rate=w["rate"], v_init=w["v0"],
                                        conn_seed=4, seed=6)


@pytest.mark.gpu
@pytest.mark.parametrize("nu", [0.002, 0.02])
def test_persistent_equals_graphs(nu):
    ref = make(nu)
    ref.run(3001)
    _, cr, ir = ref.read_raster()
    vr = ref.state()["V"]
    ev = ref.info()["events"]
    ref.close()

    sim = make(nu)
    sim.set_persistent(True)
    sim.run(1000)
    assert sim.info()["persistent"] == 1
    sim.set_persistent(False)
    sim.run(37)
    sim.set_persistent(True)
    sim.run(1964)
    sim.sync()
    _, c, i = sim.read_raster()
    assert sim.info()["step"] == 3001
    assert np.array_equal(c, cr) and np.array_equal(i, ir)
    assert np.array_equal(sim.state()["V"], vr)
    assert sim.info()["events"] == ev
    assert c.sum() > 0
    sim.close()
