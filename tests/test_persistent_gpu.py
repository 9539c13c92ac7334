"""Step groups (one cooperative launch per group: a grid barrier between
steps, or the pipelined arrive/wait two steps apart) give the rasters and
state of the graph path, also when the modes are mixed and the step counts
are no multiple of anything."""
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
@pytest.mark.parametrize("mode", [1, 2])
def test_step_groups_equal_graphs(nu, mode):
    ref = make(nu)
    ref.run(3001)
    _, cr, ir = ref.read_raster()
    vr = ref.state()["V"]
    ev = ref.info()["events"]
    ref.close()

    sim = make(nu)
    sim.set_persistent(mode)
    sim.run(1000)
    assert sim.info()["persistent"] == mode
    sim.set_persistent(0)
    sim.run(37)
    sim.set_persistent(mode)
    sim.run(1)
    sim.run(2)
    sim.set_persistent(3 - mode)
    sim.run(5)
    sim.set_persistent(mode)
    sim.run(1956)
    sim.sync()
    _, c, i = sim.read_raster()
    assert sim.info()["step"] == 3001
    assert np.array_equal(c, cr) and np.array_equal(i, ir)
    assert np.array_equal(sim.state()["V"], vr)
    assert sim.info()["events"] == ev
    assert c.sum() > 0
    sim.close()


@pytest.mark.gpu
def test_pipelined_needs_min_delay_four():
    w = bench.workload(scale=0.03)
    projs = [(s, t, k, wt, 2, 5) for (s, t, k, wt, _, _) in w["projs"]]
    sim = mgb.Simulator.fixed_indegree(w["pops"], projs, w["lif"], rate=w["rate"], v_init=w["v0"], conn_seed=4)
    sim.set_persistent(1)
    with pytest.raises(mgb.MgcError):
        sim.set_persistent(2)
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("nu", [0.002, 0.02])
def test_one_step_delay_group_equals_graphs(nu):
    """A minimum delay of one step (the arrivals of step s include step s-1's
    spikes): the step group with a barrier after the delivery and after the
    update gives the rasters and state of the single-step kernels, also when
    the two forms alternate."""
    w = bench.workload(scale=0.03, nu=nu)
    projs = [(s, t, k, wt, 1, 6) for (s, t, k, wt, _, _) in w["projs"]]

    def mk():
        return mgb.Simulator.fixed_indegree(w["pops"], projs, w["lif"], rate=w["rate"], v_init=w["v0"],
                                            conn_seed=8, seed=9)
    ref = mk()
    ref.set_persistent(0)
    ref.run(2500)
    _, cr, ir = ref.read_raster()
    vr = ref.state()["V"]
    ev = ref.info()["events"]
    ref.close()
    sim = mk()
    assert sim.info()["persistent"] == 1          # the default for this method
    sim.run(1000)
    sim.set_persistent(0)
    sim.run(77)
    sim.set_persistent(1)
    sim.run(1)
    sim.run(1422)
    sim.sync()
    _, c, i = sim.read_raster()
    assert np.array_equal(c, cr) and np.array_equal(i, ir)
    assert np.array_equal(sim.state()["V"], vr)
    assert sim.info()["events"] == ev
    assert c.sum() > 0
    with pytest.raises(mgb.MgcError):
        sim.set_persistent(2)
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("nu", [0.002, 0.02])
@pytest.mark.parametrize("window", [1, 2, 3, 4, 5, 8])
def test_windowed_group_equals_graphs(nu, window):
    """The windowed step group (arrivals of W steps delivered before the
    window, then W updates with the state in registers) gives the rasters,
    state and event count of the graph path, also when group lengths are no
    multiple of the window and the modes are mixed."""
    ref = make(nu)
    ref.set_persistent(0)
    ref.run(3001)
    _, cr, ir = ref.read_raster()
    vr = ref.state()["V"]
    st = ref.state()
    ev = ref.info()["events"]
    ref.close()

    sim = make(nu)
    sim.set_persistent(3)
    sim.set_window(window)
    info = sim.info()
    assert info["persistent"] == 3 and info["window"] == window
    sim.run(1001)
    sim.set_persistent(0)
    sim.run(37)
    sim.set_persistent(3)
    sim.run(1)
    sim.run(2)
    sim.run(3)
    sim.set_persistent(2)
    sim.run(5)
    sim.set_persistent(3)
    sim.run(1952)
    sim.sync()
    _, c, i = sim.read_raster()
    assert sim.info()["step"] == 3001
    assert np.array_equal(c, cr) and np.array_equal(i, ir)
    s2 = sim.state()
    assert np.array_equal(s2["V"], vr)
    for k in st:
        assert np.array_equal(s2[k], st[k]), k
    assert sim.info()["events"] == ev
    assert c.sum() > 0
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dmin", [2, 5, 9])
def test_windowed_group_short_min_delay(dmin):
    """Minimum delays 2, 5 and 9: every window up to min(8, dmin) steps
    (those of 5 or more in the 8-buffer cycle) gives the rasters and state of
    the graph path; a longer window is refused."""
    w = bench.workload(scale=0.03, nu=0.02)
    projs = [(s, t, k, wt, dmin, dmin + 5) for (s, t, k, wt, _, _) in w["projs"]]

    def mk():
        return mgb.Simulator.fixed_indegree(w["pops"], projs, w["lif"], rate=w["rate"], v_init=w["v0"],
                                            conn_seed=5, seed=3)
    ref = mk()
    ref.set_persistent(0)
    ref.run(1500)
    _, cr, ir = ref.read_raster()
    vr = ref.state()["V"]
    ref.close()
    for window in range(1, min(8, dmin) + 1):
        sim = mk()
        sim.set_persistent(3)
        sim.set_window(window)
        sim.run(777)
        sim.run(723)
        sim.sync()
        _, c, i = sim.read_raster()
        assert np.array_equal(c, cr) and np.array_equal(i, ir)
        assert np.array_equal(sim.state()["V"], vr)
        assert c.sum() > 0
        with pytest.raises(mgb.MgcError):
            sim.set_window(min(8, dmin) + 1)
        with pytest.raises(mgb.MgcError):
            sim.set_window(0)
        sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("nu", [0.002, 0.02])
def test_accumulator_cycle_switches(nu):
    """Runs that alternate between windows of more than 4 steps (8-buffer
    cycle) and every other form (4-buffer cycle), at odd step counts, give
    the rasters, state and event count of the graph path."""
    ref = make(nu)
    ref.set_persistent(0)
    ref.run(2400)
    _, cr, ir = ref.read_raster()
    vr, ev = ref.state()["V"], ref.info()["events"]
    ref.close()
    sim = make(nu)
    assert sim.info()["min_delay"] >= 8
    plan = [(3, 8, 301), (2, None, 211), (3, 5, 157), (0, None, 130), (3, 4, 99), (3, 7, 64), (1, None, 3),
            (3, 6, 1), (3, 8, 2), (2, None, 5)]
    done = 0
    for mode, window, steps in plan:
        sim.set_persistent(mode)
        if window:
            sim.set_window(window)
        sim.run(steps)
        done += steps
    sim.set_persistent(3)
    sim.set_window(8)
    sim.run(2400 - done)
    sim.sync()
    _, c, i = sim.read_raster()
    assert c.sum() > 0
    assert np.array_equal(c, cr) and np.array_equal(i, ir)
    assert np.array_equal(sim.state()["V"], vr)
    assert sim.info()["events"] == ev
    sim.close()


@pytest.mark.gpu
def test_windowed_group_refused_for_min_delay_one():
    w = bench.workload(scale=0.03)
    projs = [(s, t, k, wt, 1, 5) for (s, t, k, wt, _, _) in w["projs"]]
    sim = mgb.Simulator.fixed_indegree(w["pops"], projs, w["lif"], rate=w["rate"], v_init=w["v0"], conn_seed=4)
    with pytest.raises(mgb.MgcError):
        sim.set_persistent(3)
    with pytest.raises(mgb.MgcError):
        sim.set_window(1)
    assert sim.info()["window"] == 0
    sim.close()
