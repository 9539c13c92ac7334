"""Step scheduler: the MLP's forward/backward kernel against the fp64 CPU
oracle, unchanged rasters under every schedule mode, and what the trained
network gains over the threshold rule on a drive that changes with a period
the history reveals."""
import os
import sys

import numpy as np
import pytest

import mgbrain_b200 as mgb

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), ".."))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
import bench  # noqa: E402
import mlp_oracle as M  # noqa: E402

GROUP = 64
LOW, HIGH = 0.002, 0.02


@pytest.mark.gpu
def test_mlp_gradient_matches_oracle():
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.3, M.NPARAM).astype(np.float32)
    x = rng.normal(0, 1, (100, M.IN)).astype(np.float32)
    t = rng.normal(0, 1, (100, M.OUT)).astype(np.float32)
    loss, g = mgb.mlp_gradient(p, x, t)
    loss64, g64 = M.loss_and_grad(p, x, t)
    # fp32 kernel against the fp64 oracle of the same formula
    assert abs(loss - loss64) <= 1e-5 * abs(loss64)
    err = np.max(np.abs(g - g64)) / np.max(np.abs(g64))
    assert err < 1e-5, err


def rates_for(w, g):
    r = w["rate"].copy()
    r[w["n_lif"]:] = HIGH if (g // 3) % 2 == 0 else LOW   # 3 groups high, 3 low
    return r


def make(w):
    return mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], rate=w["rate"], v_init=w["v0"],
                                        conn_seed=3, seed=5)


def run_groups(sim, w, g0, groups):
    """Runs whole step groups under the periodic drive; events per step of each."""
    loads = []
    for g in range(g0, g0 + groups):
        sim.set_rates(rates_for(w, g))
        e0 = sim.info()["events"]
        sim.run(GROUP)
        loads.append((sim.info()["events"] - e0) / GROUP)
    return np.array(loads)


@pytest.mark.gpu
def test_schedules_keep_rasters_and_learned_beats_threshold():
    w = bench.workload(scale=0.02)
    sims = {m: make(w) for m in ("static", "threshold", "learned")}
    for sim in sims.values():
        sim.run(GROUP)                      # leaves the fused method's catch-up step behind
        sim.sched_collect(True, reset=True)
    g_train, g_eval = 150, 60
    loads = {m: run_groups(sim, w, 0, g_train) for m, sim in sims.items()}
    assert np.array_equal(loads["static"], loads["learned"])
    hi = np.median(loads["static"][[g for g in range(g_train) if (g // 3) % 2 == 0]])
    lo = np.median(loads["static"][[g for g in range(g_train) if (g // 3) % 2 == 1]])
    assert hi > 3 * lo
    thr = float(np.sqrt(hi * lo))
    for sim in sims.values():
        sim.sched_collect(False)
        sim.sched_threshold(thr, hi_variant=1)
    loss = sims["learned"].sched_train(epochs=400, lr=3e-3, seed=7)
    assert np.isfinite(loss) and loss < 0.5
    sims["threshold"].sched_mode(mgb.SCHED_THRESHOLD)
    sims["learned"].sched_mode(mgb.SCHED_LEARNED)
    for sim in sims.values():
        sim.sched_report(reset=True)
        run_groups(sim, w, g_train, g_eval)
    rep = {m: sim.sched_report() for m, sim in sims.items()}
    rasters = {m: sim.read_raster() for m, sim in sims.items()}
    states = {m: sim.state()["V"] for m, sim in sims.items()}
    for m in ("threshold", "learned"):
        assert np.array_equal(rasters[m][1], rasters["static"][1]), m
        assert np.array_equal(rasters[m][2], rasters["static"][2]), m
        assert np.array_equal(states[m], states["static"]), m
    # both variants ran under the adaptive modes
    assert min(rep["threshold"]["variant_groups"]) > 0
    assert rep["threshold"]["groups"] >= g_eval - 2 and rep["learned"]["groups"] >= g_eval - 2
    # the persistence rule misses at every change of the drive; the network
    # has seen the period in its four groups of history
    assert rep["threshold"]["misses"] >= g_eval // 6
    assert rep["learned"]["misses"] < rep["threshold"]["misses"] / 2, rep
    for sim in sims.values():
        sim.close()


@pytest.mark.gpu
def test_calibration_sets_a_rule():
    w = bench.workload(scale=0.02)
    sim = make(w)
    sim.run(GROUP)
    thr = sim.sched_calibrate(groups=8)
    rep = sim.sched_report()
    assert thr > 0 and rep["hi_variant"] in (0, 1)
    assert rep["threshold"] == pytest.approx(thr, rel=1e-6)
    assert sim.info()["step"] == GROUP + GROUP + 9 * GROUP
    sim.close()
