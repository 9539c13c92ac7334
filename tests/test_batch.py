"""Many independent Brunel instances of uneven size in one handle (the
parameter sweep): each instance's raster and end state equal those of the
same instance simulated alone, and instance 0 equals the oracle."""
import ctypes as C

import numpy as np
import pytest

import mgb_testlib as T
import mgbrain_b200 as mgb
from mgbrain_b200 import brunel

STEPS = 1200


def instances():
    return brunel.sweep_instances(count=6, n_min=300, n_max=3000, seed=7)


def test_sweep_parameters_follow_the_definition():
    ps = brunel.sweep_instances(count=256)
    N = np.array([p["N"] for p in ps])
    assert N.min() >= 1000 and N.max() <= 100_000
    assert all(3.0 <= p["g"] <= 7.0 and 10.0 <= p["nu"] <= 30.0 for p in ps)
    b = brunel.sweep_block(ps[0])
    K = min(ps[0]["N"] // 10, 1000)
    assert b["projs"][0][2] + b["projs"][1][2] == K


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [mgb.MODE_AUTO, mgb.MODE_PUSH])
def test_batch_equals_instances_alone(mode):
    ps = instances()
    sim, starts = brunel.sweep_batch(ps, seed=3, mode=mode)
    sim.run(STEPS)
    _, counts, ids = sim.read_raster()
    v = sim.state()["V"]
    offs = np.concatenate([[0], np.cumsum(counts)])
    assert counts.sum() > 100
    for i in range(len(ps)):
        alone = brunel.sweep_alone(ps, i, seed=3, mode=mode)
        alone.run(STEPS)
        _, ca, ia = alone.read_raster()
        lo, hi = starts[i], starts[i + 1]
        per_step = [ids[offs[k]:offs[k + 1]] for k in range(STEPS)]
        mine = [x[(x >= lo) & (x < hi)] - lo for x in per_step]
        assert np.array_equal(np.array([len(x) for x in mine]), ca), i
        assert np.array_equal(np.concatenate(mine), ia), i
        assert np.array_equal(alone.state()["V"], v[lo:hi]), i
        alone.close()


@pytest.mark.gpu
def test_batch_instance_matches_oracle():
    ps = instances()
    sim, starts = brunel.sweep_batch(ps, seed=3)
    sim.run(STEPS)
    _, counts, ids = sim.read_raster()
    b = brunel.sweep_block(ps[0])
    n = b["n"]
    L = T.oracle()
    P = np.array(b["pops"], np.int32)
    R = b["projs"]
    arr = lambda x, dt: np.ascontiguousarray(x, dt)  # noqa: E731
    keep = [arr(P[:, 0], np.int32), arr(P[:, 1], np.int32), arr(P[:, 2], np.int32),
            arr([r[0] for r in R], np.int32), arr([r[1] for r in R], np.int32),
            arr([r[2] for r in R], np.int32), arr([r[3] for r in R], np.float32),
            arr([r[4] for r in R], np.int32), arr([r[5] for r in R], np.int32)]
    h = L.mgbo_create_fixed_indegree(*[T._p(k) for k in keep[:3]], len(P),
                                     *[T._p(k) for k in keep[3:]], len(R), T._p(b["rate"]),
                                     T._p(b["v_init"]), T._p(brunel.brunel_lifconst()),
                                     b["conn_seed"], 3, 1, 0, 0)
    try:
        oc = np.zeros(STEPS, np.int64)
        oi = np.zeros(n * 100, np.int32)
        nid = C.c_int64()
        assert L.mgbo_run(h, STEPS, T._p(oc), T._p(oi), len(oi), C.byref(nid)) == 0
        offs = np.concatenate([[0], np.cumsum(counts)])
        mine = [ids[offs[k]:offs[k + 1]] for k in range(STEPS)]
        mine = [x[x < starts[1]] for x in mine]
        assert np.array_equal(np.array([len(x) for x in mine]), oc)
        assert np.array_equal(np.concatenate(mine), oi[:nid.value])
        ov = np.zeros(n, np.float32)
        L.mgbo_read_state_f32(h, T._p(ov), None)
        assert np.array_equal(sim.state()["V"][:n], ov)
    finally:
        L.mgbo_destroy(h)
