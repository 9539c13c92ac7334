"""CUDA core against the oracle (and the reference kernels' golden outputs)
on the golden networks, through the C ABI.

Bar: rasters (step and neuron id of every spike) and every fp32 state array
bit-exact against the oracle's fp32 path, or against the oracle's
fixed-point path where the core sums inputs in fixed point (networks in which
some neuron receives unequal weights of one sign); STDP weights within 1e-5
relative (CUDA expf vs the host libm expf)."""
import numpy as np
import pytest

import mgb_testlib as T
import mgbrain_b200 as mgb
from cases import NAMES, load, ref_outputs, run_oracle

W_RTOL = 1e-5


def run_cuda(name, mode=mgb.MODE_AUTO, persistent=None):
    c, net, v0 = load(name)
    dsteps, dmin, dmax = T.quantize_delays(net["delay"], net["step"])
    sim = mgb.Simulator.from_arrays(
        net["n"], net["type"], net["src"], net["tar"], net["weight"], dsteps,
        T.default_lifconst(net), T.default_stdpconst(net), rate=net["rate"], v_init=v0,
        stdp=bool(c["stdp"]), seed=c["seed"], mode=mode)
    if persistent is not None:
        sim.set_persistent(persistent)
    off = c.get("rates_off")
    if off:
        sim.run(off)
        sim.set_rates(np.zeros(net["n"], np.float32))
        sim.run(c["steps"] - off)
    else:
        sim.run(c["steps"])
    sim.sync()
    first, counts, ids = sim.read_raster()
    assert first == 0
    return counts, ids, sim.state(), sim


MODES = {"push": mgb.MODE_PUSH, "auto": mgb.MODE_AUTO, "pull": mgb.MODE_PULL}


@pytest.mark.gpu
@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("name", NAMES)
def test_cuda_matches_oracle(name, mode):
    c, net, _ = load(name)
    gc, gi, gst, gsim = run_cuda(name, MODES[mode])
    info = gsim.info()
    fixed = info["accumulation"] == mgb.ACC_FIXED
    hetero, shift = T.fx_plan(net, stdp=bool(c["stdp"]), wlim=max(abs(T.default_stdpconst(net)[4]),
                                                                   abs(T.default_stdpconst(net)[5])))
    # fixed point exactly where some neuron gets unequal weights of one sign
    # (or weights are plastic), except for the pull method
    assert fixed == (hetero and info["mode"] != mgb.MODE_PULL)
    if fixed:
        assert info["fx_shift"] == shift
    oc, oi, ost, osim = run_oracle(name, fx=info["fx_shift"] if fixed else None)
    if mode == "auto":
        expect_mode = mgb.MODE_PUSH if c["stdp"] else mgb.MODE_DEFERRED
    else:
        expect_mode = MODES[mode]
    assert gsim.info()["mode"] == expect_mode
    assert np.array_equal(gc, oc), "spike counts per step differ"
    assert np.array_equal(gi, oi), "spike ids differ"
    for k in ("refrac", "last_fired", "fire_cnt"):
        assert np.array_equal(gst[k], ost[k]), k
    w = gsim.weights()
    if c["stdp"]:
        # CUDA expf vs host libm expf: last-bit differences in the weights
        np.testing.assert_allclose(w, ost["weight32"], rtol=W_RTOL, atol=1e-9)
        np.testing.assert_allclose(gst["V"], ost["V32"], rtol=W_RTOL, atol=1e-8)
    else:
        # one weight per sign: every order of the fp32 input sums gives the
        # same bits; unequal weights: the order-independent fixed-point sums
        # of the oracle's fixed-point path, bit for bit
        assert np.array_equal(gst["V"].view(np.int32), ost["V32"].view(np.int32)), "V not bit-exact"
        assert np.array_equal(w, net["weight"])
    if gsim.info()["mode"] in (mgb.MODE_PUSH, mgb.MODE_PULL):
        assert gsim.info()["events"] == osim.events  # counted at emission
    else:
        assert gsim.info()["events"] <= osim.events  # counted at arrival


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_matches_reference_kernels(name):
    ref = ref_outputs(name)
    if ref is None:
        pytest.skip("no golden reference outputs for " + name)
    rc, ri, rst = ref
    c, net, _ = load(name)
    gc, gi, gst, gsim = run_cuda(name)
    assert np.array_equal(gc, rc)
    assert np.array_equal(gi, ri)
    if c["stdp"]:
        np.testing.assert_allclose(gst["V"], rst["V"], rtol=1e-5, atol=1e-9)
        np.testing.assert_allclose(gsim.weights(), rst["weight"], rtol=W_RTOL, atol=1e-9)
    elif T.equal_per_sign(net["weight"]):
        assert np.array_equal(gst["V"].view(np.int32), rst["V"].view(np.int32))
    else:
        # unequal weights of one sign: the reference's fp32 atomics add them in
        # an order its scheduling decides, the core in fixed point exactly
        assert gsim.info()["accumulation"] == mgb.ACC_FIXED
        np.testing.assert_allclose(gst["V"], rst["V"], rtol=W_RTOL, atol=1e-8)
    for k in ("fire_cnt", "last_fired", "refrac"):
        assert np.array_equal(gst[k], rst[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_windowed_group_matches_reference_kernels(name):
    """The windowed step group (mgc_set_persistent mode 3, windows of up to 8
    steps) against the reference kernels' outputs: rasters and integer state
    bit-exact; V bit-exact with one weight per sign, else within 1e-5
    relative of the reference (whose fp32 atomics leave the order of unequal
    additions open) and bit-exact against the pipelined group (both sum
    such inputs in fixed point)."""
    ref = ref_outputs(name)
    if ref is None:
        pytest.skip("no golden reference outputs for " + name)
    c, net, _ = load(name)
    if c["stdp"]:
        pytest.skip("STDP networks run the pull method (no step groups)")
    dsteps, dmin, _ = T.quantize_delays(net["delay"], net["step"])
    if dmin < 2:
        pytest.skip("a minimum delay of one step has one step-group form")
    rc, ri, rst = ref
    gc, gi, gst, gsim = run_cuda(name, persistent=3)
    assert gsim.info()["persistent"] == 3 and gsim.info()["window"] == min(8, dmin)
    assert np.array_equal(gc, rc)
    assert np.array_equal(gi, ri)
    for k in ("fire_cnt", "last_fired", "refrac"):
        assert np.array_equal(gst[k], rst[k]), k
    if T.equal_per_sign(net["weight"]):
        assert np.array_equal(gst["V"].view(np.int32), rst["V"].view(np.int32))
    else:
        np.testing.assert_allclose(gst["V"], rst["V"], rtol=W_RTOL, atol=1e-8)
        # the pipelined group gives the same bits (fixed-point sums do not
        # depend on which warp adds which input)
        pc, pi, pst, _ = run_cuda(name)
        assert np.array_equal(pc, gc) and np.array_equal(pi, gi)
        assert np.array_equal(pst["V"].view(np.int32), gst["V"].view(np.int32))


@pytest.mark.gpu
def test_run_split_equals_straight():
    """Steps continue across calls: 700 + 1300 steps == 2000 steps."""
    name = "c0s"
    c, net, v0 = load(name)
    dsteps, _, _ = T.quantize_delays(net["delay"], net["step"])
    args = (net["n"], net["type"], net["src"], net["tar"], net["weight"], dsteps,
            T.default_lifconst(net))
    a = mgb.Simulator.from_arrays(*args, rate=net["rate"], v_init=v0, seed=c["seed"])
    a.run(2000)
    b = mgb.Simulator.from_arrays(*args, rate=net["rate"], v_init=v0, seed=c["seed"])
    b.run(700)
    b.run(1300)
    _, ca, ia = a.read_raster()
    _, cb, ib = b.read_raster()
    assert np.array_equal(ca, cb) and np.array_equal(ia, ib)
    assert np.array_equal(a.state()["V"], b.state()["V"])


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["auto", "push"])
def test_fixed_indegree_matches_oracle(mode):
    """Device-generated fixed in-degree network (the large-Brunel generator)
    at 5k neurons: CSR, raster and V bit-exact against the oracle."""
    import ctypes as C
    NE, NI, NP = 4000, 1000, 500
    pops = [(0, NE, mgb.LIFB), (NE, NI, mgb.LIFB), (NE + NI, NP, mgb.POISSON)]
    J = 0.0005
    projs = [(0, 0, 80, J, 10, 50), (0, 1, 80, J, 10, 50), (1, 0, 20, -5 * J, 10, 50),
             (1, 1, 20, -5 * J, 10, 50), (2, 0, 10, J, 10, 50), (2, 1, 10, J, 10, 50)]
    n = NE + NI + NP
    lif = np.zeros(30, np.float32)
    lif[0], lif[3], lif[4], lif[8] = 1e-4, 0.01, 0.02, 0.002
    rate = np.zeros(n, np.float32)
    rate[NE + NI:] = 0.02
    v0 = np.random.default_rng(3).uniform(0, 0.02, n).astype(np.float32)
    g = mgb.Simulator.fixed_indegree(pops, projs, lif, rate=rate, v_init=v0, conn_seed=77, seed=5,
                                     mode=MODES[mode])
    L = T.oracle()
    P = np.array(pops, np.int32)
    R = projs
    arr = lambda x, dt: np.ascontiguousarray(x, dt)
    keep = [arr(P[:, 0], np.int32), arr(P[:, 1], np.int32), arr(P[:, 2], np.int32),
            arr([r[0] for r in R], np.int32), arr([r[1] for r in R], np.int32),
            arr([r[2] for r in R], np.int32), arr([r[3] for r in R], np.float32),
            arr([r[4] for r in R], np.int32), arr([r[5] for r in R], np.int32)]
    h = L.mgbo_create_fixed_indegree(*[T._p(k) for k in keep[:3]], len(P),
                                     *[T._p(k) for k in keep[3:]], len(R), T._p(rate), T._p(v0),
                                     T._p(lif), 77, 5, 1, 0, 0)
    try:
        S = L.mgbo_n_syn(h)
        orp = np.zeros(n + 1, np.int64)
        ot = np.zeros(S, np.int32)
        od = np.zeros(S, np.int32)
        L.mgbo_export_csr(h, T._p(orp), T._p(ot), None, T._p(od))
        grp, gt, gw, gd = g.export_csr()
        assert np.array_equal(grp, orp)
        if g.info()["mode"] == mgb.MODE_PUSH:
            assert np.array_equal(gt, ot) and np.array_equal(gd, od)
        else:
            # rows are bucketed by delay: same multiset per row, ordered by
            # (delay, synapse-list order)
            for i in np.random.default_rng(0).choice(n, 200, replace=False):
                a, b = orp[i], orp[i + 1]
                key_o = np.lexsort((np.arange(b - a), od[a:b]))
                assert np.array_equal(gt[a:b], ot[a:b][key_o]) and np.array_equal(gd[a:b], od[a:b][key_o])
        steps = 1500
        counts = np.zeros(steps, np.int64)
        ids = np.zeros(n * 50, np.int32)
        nid = C.c_int64()
        assert L.mgbo_run(h, steps, T._p(counts), T._p(ids), len(ids), C.byref(nid)) == 0
        g.run(steps)
        _, gc, gi = g.read_raster()
        assert np.array_equal(gc, counts)
        assert np.array_equal(gi, ids[:nid.value])
        ov = np.zeros(n, np.float32)
        L.mgbo_read_state_f32(h, T._p(ov), None)
        assert np.array_equal(g.state()["V"], ov)
        assert counts.sum() > 100
    finally:
        L.mgbo_destroy(h)
