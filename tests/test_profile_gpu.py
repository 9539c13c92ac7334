"""mgc_profile_steps times the kernels of real steps: profiled steps advance
the network exactly as mgc_run's steps do, every kernel class that runs gets
a positive time, and the handle (and the next one) stays usable."""
import numpy as np
import pytest

import mgbrain_b200 as mgb
from mgbrain_b200 import brunel


def make_explicit(mode):
    """Random LIFB network fed by POISSON inputs, delays 1..5 steps (min delay
    1: the deferred method runs delivery and update as two kernels)."""
    rng = np.random.default_rng(3)
    n_lif, n_in, S = 2000, 500, 120_000
    n = n_lif + n_in
    types = np.full(n, mgb.LIFB, np.int8)
    types[n_lif:] = mgb.POISSON
    rate = np.zeros(n, np.float32)
    rate[n_lif:] = 0.01
    src = rng.integers(0, n, S).astype(np.int32)
    tar = rng.integers(0, n_lif, S).astype(np.int32)
    w = np.where(src < 1600, 4e-4, -1.6e-3).astype(np.float32)
    w[src >= n_lif] = 4e-4   # one value per sign: sums independent of order
    d = rng.integers(1, 6, S).astype(np.int32)
    v0 = rng.uniform(0, 0.02, n).astype(np.float32)
    return mgb.Simulator.from_arrays(n, types, src, tar, w, d, brunel.brunel_lifconst(), rate=rate,
                                     v_init=v0, seed=5, mode=mode)


def make_fixed(mode):
    p = brunel.sweep_instances(count=1, n_min=4000, n_max=4000, seed=11)[0]
    b = brunel.sweep_block(p)
    return mgb.Simulator.fixed_indegree(b["pops"], b["projs"], brunel.brunel_lifconst(), rate=b["rate"],
                                        v_init=b["v_init"], conn_seed=b["conn_seed"], seed=5, mode=mode)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [mgb.MODE_AUTO, mgb.MODE_PUSH, mgb.MODE_DEFERRED])
@pytest.mark.parametrize("make", [make_fixed, make_explicit])
def test_profiled_steps_equal_run_steps(make, mode):
    ref = make(mode)
    ref.run(900)
    _, c_ref, i_ref = ref.read_raster()
    v_ref = ref.state()["V"]
    ref.close()

    sim = make(mode)
    sim.run(300)
    ms = sim.profile(300)          # 300 steps, timed, in four graph batches
    sim.run(300)
    _, c, i = sim.read_raster()
    assert sim.info()["step"] == 900
    assert np.array_equal(c, c_ref) and np.array_equal(i, i_ref)
    assert np.array_equal(sim.state()["V"], v_ref)
    assert ms[0] > 0 and ms[1] > 0 and ms[2] == 0
    sim.close()
    # a handle created after profiling builds and runs normally
    again = make(mode)
    again.run(10)
    again.sync()
    again.close()
