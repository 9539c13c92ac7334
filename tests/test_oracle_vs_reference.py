"""The oracle pinned against the reference itself: rasters and end states
that the reference's own kernels (mgcore.cu built for sm_100a with
--fmad=false and counter-based Poisson draws, oracle/_ref/ref_sim) produced
on a B200 for each golden network (tests/golden/*.ref.*, made by
tests/golden/make_golden.py sim)."""
import numpy as np
import pytest

import mgb_testlib as T
from cases import CASES, NAMES, load, ref_outputs, run_oracle

# fp32 STDP: the reference evaluates exp with CUDA's expf and the oracle with
# the host libm expf; the two differ in the last bits, so weights (and the
# membrane potentials they feed) agree to a relative 1e-5, rasters exactly.
STDP_RTOL = 1e-5


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_kernels(name):
    ref = ref_outputs(name)
    assert ref is not None, "golden reference outputs missing for " + name
    rc, ri, rst = ref
    c, net, _ = load(name)
    oc, oi, ost, _ = run_oracle(name)
    assert np.array_equal(oc, rc), "spike counts per step"
    assert np.array_equal(oi, ri), "spike ids"
    for k in ("fire_cnt", "last_fired", "refrac"):
        assert np.array_equal(ost[k], rst[k]), k
    if c["stdp"]:
        np.testing.assert_allclose(ost["V32"], rst["V"], rtol=STDP_RTOL, atol=1e-8)
        np.testing.assert_allclose(ost["weight32"], rst["weight"], rtol=STDP_RTOL, atol=1e-9)
    else:
        assert np.array_equal(ost["V32"].view(np.int32), rst["V"].view(np.int32))
        assert np.array_equal(ost["weight32"], rst["weight"])
        if net["type"].max() in (T.TYPES["LIF"], T.TYPES["LIFE"]):
            assert np.array_equal(ost["Iexc"].astype(np.float32), rst["Iexc"])


@pytest.mark.parametrize("name", [n for n in NAMES if CASES[n].get("simulate")])
def test_oracle_matches_reference_simulate(name):
    """MGSimulator::simulate(t) itself: its step-count rule and end state."""
    import os
    c, net, v0 = load(name)
    rs = T.read_state(os.path.join(T.GOLDEN, name + ".sim.state"), net["n"], len(net["src"]))
    o = T.OracleSim(net, c["seed"], v0=v0, stdp=c["stdp"])
    L = T.oracle()
    steps = L.mgbo_steps_for_time(np.float32(c["simulate"]), np.float32(net["step"]))
    eff = L.mgbo_effective_steps(steps, o.dmin)
    o.run(eff, record=False)
    st = o.state()
    assert np.array_equal(st["fire_cnt"], rs["fire_cnt"])
    assert np.array_equal(st["V32"].view(np.int32), rs["V"].view(np.int32))
    assert np.array_equal(st["last_fired"], rs["last_fired"])


def test_fp64_error_of_fp32_path():
    """fp32 path against the fp64 twin of the same algorithm on the
    reference's own Brunel maker: the raster is stated, and where rasters
    agree the membrane-potential error stays at fp32 rounding level."""
    name = "brunel_maker"
    oc, oi, o32, _ = run_oracle(name, T.F32)
    dc, di, o64, _ = run_oracle(name, T.F64)
    same_raster = np.array_equal(oc, dc) and np.array_equal(oi, di)
    if same_raster:
        err = np.abs(o32["V"] - o64["V"]).max()
        assert err < 1e-6, err
    # population rate within 1 %
    assert abs(oc.sum() - dc.sum()) <= 0.01 * dc.sum()
