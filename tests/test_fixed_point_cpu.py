"""Fixed-point accumulation in the oracle (the arithmetic of the CUDA core's
MGC_ACC_FIXED): order-independent, so every thread count gives the same bits;
close to the fp32 path that restates the reference (rasters equal, V within
1e-5) and closer to the fp64 twin than it."""
import numpy as np
import pytest

import mgb_testlib as T
from cases import load


@pytest.mark.parametrize("name", ["lif_mixed", "c1s"])
def test_fixed_point_independent_of_order(name):
    c, net, v0 = load(name)
    hetero, shift = T.fx_plan(net)
    assert hetero
    runs = []
    for threads in (1, 8):
        o = T.OracleSim(net, c["seed"], v0=v0, nthreads=threads)
        o.set_fx(shift)
        counts, ids = o.run(c["steps"])
        runs.append((counts, ids, o.state()["V32"]))
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
    assert np.array_equal(runs[0][2].view(np.int32), runs[1][2].view(np.int32))


@pytest.mark.parametrize("name", ["lif_mixed", "c1s"])
def test_fixed_point_against_fp32_and_fp64(name):
    c, net, v0 = load(name)
    _, shift = T.fx_plan(net)
    steps = c["steps"] if not c.get("rates_off") else c["rates_off"]   # no rate change inside the window
    fx = T.OracleSim(net, c["seed"], v0=v0)
    fx.set_fx(shift)
    f32 = T.OracleSim(net, c["seed"], v0=v0)
    f64 = T.OracleSim(net, c["seed"], v0=v0, precision=T.F64)
    rs = [o.run(steps) for o in (fx, f32, f64)]
    assert np.array_equal(rs[0][0], rs[1][0]) and np.array_equal(rs[0][1], rs[1][1])
    v_fx, v_32, v_64 = fx.state()["V32"], f32.state()["V32"], f64.state()["V"]
    np.testing.assert_allclose(v_fx, v_32, rtol=1e-5, atol=1e-9)
    if np.array_equal(rs[2][0], rs[0][0]) and np.array_equal(rs[2][1], rs[0][1]):
        e_fx = np.abs(v_fx - v_64).max()
        e_32 = np.abs(v_32 - v_64).max()
        assert e_fx <= e_32 * 1.01 + 1e-12, (e_fx, e_32)


def test_fx_shift_makes_weights_exact():
    _, net, _ = load("lif_mixed")
    hetero, shift = T.fx_plan(net)
    w = net["weight"].astype(np.float64)
    q = w * 2.0 ** shift
    assert np.array_equal(q, np.rint(q))           # every weight an exact multiple of 2^-shift
    bound = np.bincount(net["tar"], weights=np.abs(w), minlength=net["n"]).max()
    assert bound * 2.0 ** shift < 2.0 ** 62         # any one step's sum fits the integer
