"""Order-independent (fixed-point) accumulation on the GPU: networks in which
some neuron receives unequal weights of one sign sum their inputs in 64-bit
fixed point (include/mgc.h, MGC_ACC_FIXED), so every delivery form (graphs of
single-step kernels, the step groups with a barrier per step, pipelined and
windowed with every window, the ring push) gives the same bits as the
oracle's fixed-point path, and every run repeats them.  Against the
reference's arithmetic (fp32 sums in an order the atomics decide) rasters are
equal and V agrees within 1e-5."""
import numpy as np
import pytest

import configs
import mgb_testlib as T
import mgbrain_b200 as mgb
from cases import load

STEPS = 2000


def network(name):
    if name == "c0r":
        net, v0, steps = configs.build(configs.C0R)
        return net, v0, configs.C0R["seed"], steps, None
    c, net, v0 = load(name)
    return net, v0, c["seed"], c["steps"], c.get("rates_off")


def make(net, v0, seed, mode=mgb.MODE_AUTO, **kw):
    dsteps, _, _ = T.quantize_delays(net["delay"], net["step"])
    return mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], dsteps,
                                     T.default_lifconst(net), rate=net["rate"], v_init=v0, seed=seed, mode=mode,
                                     **kw)


def run(sim, net, steps, rates_off):
    if rates_off:
        sim.run(rates_off)
        sim.set_rates(np.zeros(net["n"], np.float32))
        sim.run(steps - rates_off)
    else:
        sim.run(steps)
    sim.sync()
    _, counts, ids = sim.read_raster()
    return counts, ids, sim.state()


def oracle(net, v0, seed, steps, rates_off, fx):
    o = T.OracleSim(net, seed, v0=v0)
    if fx is not None:
        o.set_fx(fx)
    if rates_off:
        c1, i1 = o.run(rates_off)
        o.set_rates(np.zeros(net["n"], np.float32))
        c2, i2 = o.run(steps - rates_off)
        counts, ids = np.concatenate([c1, c2]), np.concatenate([i1, i2])
    else:
        counts, ids = o.run(steps)
    return counts, ids, o.state()


def forms(dmin):
    """(label, mode, persistent, window) of every delivery form the network allows."""
    out = [("push", mgb.MODE_PUSH, None, None), ("graphs", mgb.MODE_AUTO, 0, None)]
    if dmin >= 2:
        out.append(("barrier-per-step", mgb.MODE_AUTO, 1, None))
        out += [(f"windowed-{w}", mgb.MODE_AUTO, 3, w) for w in range(1, min(8, dmin) + 1)]
    else:
        out.append(("step-group-delay-1", mgb.MODE_AUTO, 1, None))
    if dmin >= 4:
        out.append(("pipelined", mgb.MODE_AUTO, 2, None))
    return out


NAMES = ["lif_mixed", "c1s", "c0r"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_every_form_gives_the_oracle_fixed_point_bits(name):
    net, v0, seed, steps, off = network(name)
    hetero, shift = T.fx_plan(net)
    assert hetero and not T.equal_per_sign(net["weight"])
    _, dmin, _ = T.quantize_delays(net["delay"], net["step"])
    oc, oi, ost = oracle(net, v0, seed, steps, off, shift)
    assert oc.sum() > 100
    for label, mode, pers, window in forms(dmin):
        g = make(net, v0, seed, mode=mode)
        info = g.info()
        assert info["accumulation"] == mgb.ACC_FIXED and info["fx_shift"] == shift, label
        if pers is not None:
            g.set_persistent(pers)
        if window is not None:
            g.set_window(window)
        gc, gi, gst = run(g, net, steps, off)
        assert np.array_equal(gc, oc) and np.array_equal(gi, oi), label + ": raster"
        for k in ("V", "Iexc", "Iinh"):
            assert np.array_equal(gst[k].view(np.int32), ost[k].astype(np.float32).view(np.int32)), f"{label}: {k}"
        for k in ("refrac", "last_fired", "fire_cnt"):
            assert np.array_equal(gst[k], ost[k]), f"{label}: {k}"
        g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["graphs", "pipelined", "windowed-4", "push"])
@pytest.mark.parametrize("name", ["lif_mixed", "c0r"])
def test_run_twice_is_bitwise_identical(name, form):
    net, v0, seed, steps, off = network(name)
    _, dmin, _ = T.quantize_delays(net["delay"], net["step"])
    label, mode, pers, window = [f for f in forms(dmin) if f[0] == form][0]
    out = []
    for _ in range(2):
        g = make(net, v0, seed, mode=mode)
        if pers is not None:
            g.set_persistent(pers)
        if window is not None:
            g.set_window(window)
        gc, gi, gst = run(g, net, steps, off)
        out.append((gc, gi, gst["V"].view(np.int32), gst["Iexc"].view(np.int32)))
        g.close()
    for x, y in zip(out[0], out[1]):
        assert np.array_equal(x, y)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_fixed_point_against_the_reference_arithmetic(name):
    """Against the oracle's fp32 path (the reference's arithmetic, inputs added
    in synapse order): rasters equal, V within 1e-5; and with the fp32 sums
    requested (ACC_FLOAT) the same bound."""
    net, v0, seed, steps, off = network(name)
    oc, oi, ost = oracle(net, v0, seed, steps, off, None)
    for acc in (mgb.ACC_FIXED, mgb.ACC_FLOAT):
        g = make(net, v0, seed)
        g.set_accumulation(acc)
        assert g.info()["accumulation"] == acc
        gc, gi, gst = run(g, net, steps, off)
        assert np.array_equal(gc, oc) and np.array_equal(gi, oi)
        np.testing.assert_allclose(gst["V"], ost["V32"], rtol=1e-5, atol=1e-9)
        g.close()


@pytest.mark.gpu
def test_accumulation_is_chosen_before_the_first_step():
    net, v0, seed, steps, off = network("lif_mixed")
    g = make(net, v0, seed)
    g.run(10)
    with pytest.raises(mgb.MgcError) as e:
        g.set_accumulation(mgb.ACC_FLOAT)
    assert e.value.status == mgb.capi.MGC_ERR_INVALID
    p = make(net, v0, seed, mode=mgb.MODE_PULL)
    assert p.info()["accumulation"] == mgb.ACC_FLOAT   # the pull method sums in a fixed order
    with pytest.raises(mgb.MgcError):
        p.set_accumulation(mgb.ACC_FIXED)
    c, netc, v0c = load("c0s")   # one weight per sign: fp32, bit-exact with the reference
    assert make(netc, v0c, c["seed"]).info()["accumulation"] == mgb.ACC_FLOAT


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [mgb.MODE_AUTO, mgb.MODE_PUSH])
def test_fixed_point_checkpoint_resumes_exactly(mode):
    net, v0, seed, steps, off = network("c0r")
    a = make(net, v0, seed, mode=mode)
    ac, ai, ast = run(a, net, steps, None)
    b = make(net, v0, seed, mode=mode)
    b.run(700)
    blob = b.checkpoint()
    c = make(net, v0, seed, mode=mode)
    c.restore(blob)
    c.run(steps - 700)
    c.sync()
    _, cc, ci = c.read_raster()
    n700 = int(ac[:700].sum())
    assert np.array_equal(cc, ac[700:]) and np.array_equal(ci, ai[n700:])
    assert np.array_equal(c.state()["V"].view(np.int32), ast["V"].view(np.int32))
    f = make(net, v0, seed, mode=mode)
    f.set_accumulation(mgb.ACC_FLOAT)
    with pytest.raises(mgb.MgcError):      # another accumulation: another state layout
        f.restore(blob)
