"""The staged raster readout (a device copy enqueued on the handle's stream,
collected while later steps run) returns exactly what the synchronous
readout returns, chunk by chunk; the two-stage limit and the ordering
against mgc_read_raster are enforced; the state of the run is untouched."""
import numpy as np
import pytest

import mgbrain_b200 as mgb

import bench


def make():
    w = bench.workload(scale=0.02, nu=0.02)
    return mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], rate=w["rate"], v_init=w["v0"],
                                        conn_seed=13, seed=14)


@pytest.mark.gpu
@pytest.mark.parametrize("persistent", [0, 2])
def test_staged_equals_synchronous(persistent):
    a, b = make(), make()
    a.set_persistent(persistent)
    b.set_persistent(persistent)
    sync_chunks, staged_chunks = [], []
    for i in range(5):
        a.run(777)
        sync_chunks.append(a.read_raster())
        b.run(777)
        b.stage_raster()
        if i >= 1:          # one chunk behind: the collect overlaps the next chunk's steps
            staged_chunks.append(b.collect_raster())
    staged_chunks.append(b.collect_raster())
    assert len(staged_chunks) == len(sync_chunks)
    for (f1, c1, i1), (f2, c2, i2) in zip(sync_chunks, staged_chunks):
        assert f1 == f2
        assert np.array_equal(c1, c2) and np.array_equal(i1, i2)
    assert sum(c.sum() for _, c, _ in sync_chunks) > 0
    assert np.array_equal(a.state()["V"], b.state()["V"])


@pytest.mark.gpu
def test_stage_limits():
    s = make()
    s.run(100)
    s.stage_raster()
    with pytest.raises(mgb.MgcError):
        s.read_raster()           # a stage is outstanding
    s.run(100)
    s.stage_raster()
    with pytest.raises(mgb.MgcError):
        s.stage_raster()          # two outstanding already
    f1, c1, _ = s.collect_raster()
    f2, c2, _ = s.collect_raster()
    assert (f1, len(c1), f2, len(c2)) == (0, 100, 100, 100)
    with pytest.raises(mgb.MgcError):
        s.collect_raster()        # nothing staged
    s.run(50)
    f3, c3, _ = s.read_raster()
    assert (f3, len(c3)) == (200, 50)
