"""The benchmark configurations at their stated sizes through the CUDA core,
checked against
  - the oracle's fp32 path (the reference's kernels restated in C): spike
    rasters bit-exact for the first 100 ms and, where the arithmetic allows,
    the whole run; neuron state bit-exact with one weight per sign, else
    within 1e-5 relative; population rate and mean CV-ISI within 1 % over
    the whole run;
  - the reference's own kernels (its sm_100a build) run on the same network
    from the same seed, where the reference can express the network (C0, C1);
  - the oracle's fp64 twin: the error of the fp32 arithmetic, printed and
    bounded (1e-5 of the threshold while the rasters agree).
Run with -s to see the printed error lines (FP64ERR ...)."""
import numpy as np
import pytest

import configs
import mgb_testlib as T
import mgbrain_b200 as mgb
import stdp_net

RTOL = 1e-5
STEPS_100MS = 1000          # dt 0.1 ms


def equal_per_sign(w):
    return len(np.unique(w[w > 0])) <= 1 and len(np.unique(w[w <= 0])) <= 1


def run_oracle(net, v0, seed, steps, precision, rates_off=None, at=None, nthreads=1):
    """(counts, ids, end state, state after `at` steps)."""
    o = T.OracleSim(net, seed, v0=v0, precision=precision, nthreads=nthreads)
    cs, ids, mid = [], [], None
    marks = sorted({m for m in (rates_off, at) if m is not None and 0 < m < steps})
    done = 0
    for m in marks + [steps]:
        c, i = o.run(m - done)
        cs.append(c)
        ids.append(i)
        done = m
        if m == rates_off:
            o.set_rates(np.zeros(net["n"], np.float32))
        if m == at:
            mid = o.state()
    return np.concatenate(cs), np.concatenate(ids), o.state(), mid


def run_cuda(net, v0, seed, steps, mode=mgb.MODE_AUTO, persistent=None, rates_off=None, at=None):
    dsteps, _, _ = T.quantize_delays(net["delay"], net["step"])
    g = mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], dsteps,
                                  net["lifconst"], rate=net["rate"], v_init=v0, seed=seed, mode=mode,
                                  raster_steps=steps + 1, raster_ids=max(1 << 22, steps * 64))
    if persistent is not None:
        g.set_persistent(persistent)
    marks = sorted({m for m in (rates_off, at) if m is not None and 0 < m < steps})
    done, mid = 0, None
    for m in marks + [steps]:
        g.run(m - done)
        done = m
        if m == rates_off:
            g.set_rates(np.zeros(net["n"], np.float32))
        if m == at:
            g.sync()
            mid = g.state()
    g.sync()
    first, counts, ids = g.read_raster(max_steps=steps + 1, max_ids=max(1 << 22, steps * 64))
    assert first == 0 and len(counts) == steps
    return counts, ids, g.state(), mid, g


def fp64_error(v32, v64, vth, label):
    """Max |V_fp32 - V_fp64| (volts) and that over the threshold; printed."""
    err = float(np.max(np.abs(v32.astype(np.float64) - v64)))
    print(f"FP64ERR {label}: max |V - V_fp64| = {err:.3e} V = {err / vth:.3e} of V_th")
    return err / vth


@pytest.fixture(scope="module")
def c0():
    net, v0, steps = configs.build(configs.C0)
    seed = configs.C0["seed"]
    o32 = run_oracle(net, v0, seed, steps, T.F32, at=STEPS_100MS)
    o64 = run_oracle(net, v0, seed, steps, T.F64, at=STEPS_100MS)
    return net, v0, steps, seed, o32, o64


def check_against_oracle(label, net, steps, g, o32, o64, vth, exact_raster=True):
    gc, gi, gst, gmid = g
    oc, oi, ost, omid = o32
    # the first 100 ms bit-exact
    n100 = int(oc[:STEPS_100MS].sum())
    assert np.array_equal(gc[:STEPS_100MS], oc[:STEPS_100MS]), label + ": counts differ in the first 100 ms"
    assert np.array_equal(gi[:n100], oi[:n100]), label + ": ids differ in the first 100 ms"
    # population rate and CV-ISI over the whole run
    r_o, cv_o, k_o = T.rate_and_cv(oc, oi, net["n"], steps, net["step"])
    r_g, cv_g, k_g = T.rate_and_cv(gc, gi, net["n"], steps, net["step"])
    print(f"RATECV {label}: rate {r_g:.4f} Hz (oracle {r_o:.4f}), CV-ISI {cv_g:.4f} (oracle {cv_o:.4f}, "
          f"{k_o} neurons)")
    assert abs(r_g - r_o) <= 0.01 * r_o, (r_g, r_o)
    assert abs(cv_g - cv_o) <= 0.01 * cv_o, (cv_g, cv_o)
    same = np.array_equal(gc, oc) and np.array_equal(gi, oi)
    if exact_raster:
        assert same, label + ": rasters differ after the first 100 ms"
    w = net["weight"]
    for st_g, st_o, when in ((gmid, omid, "100 ms"), (gst, ost, "end")):
        if when == "end" and not same:
            continue
        for k in ("refrac", "last_fired", "fire_cnt"):
            assert np.array_equal(st_g[k], st_o[k]), f"{label} {when}: {k}"
        if equal_per_sign(w):
            assert np.array_equal(st_g["V"].view(np.int32), st_o["V32"].view(np.int32)), \
                f"{label} {when}: V not bit-exact"
        else:
            np.testing.assert_allclose(st_g["V"], st_o["V32"], rtol=RTOL, atol=RTOL * vth)
    # the fp32 arithmetic against the fp64 twin, while the rasters agree
    c64, i64, st64, mid64 = o64
    n100_64 = int(c64[:STEPS_100MS].sum())
    if np.array_equal(c64[:STEPS_100MS], gc[:STEPS_100MS]) and np.array_equal(i64[:n100_64], gi[:n100]):
        assert fp64_error(gmid["V"], mid64["V"], vth, label + " @100ms") <= RTOL
    else:
        print(f"FP64ERR {label} @100ms: the fp64 raster differs from the fp32 raster within 100 ms")
    if np.array_equal(c64, gc) and np.array_equal(i64, gi):
        assert fp64_error(gst["V"], st64["V"], vth, label + " @end") <= RTOL


C0_MODES = {"deferred-pipelined": (mgb.MODE_AUTO, None), "deferred-windowed": (mgb.MODE_AUTO, 3),
            "deferred-graphs": (mgb.MODE_AUTO, 0), "push": (mgb.MODE_PUSH, None)}


@pytest.mark.gpu
@pytest.mark.parametrize("form", sorted(C0_MODES))
def test_c0_as_specified(c0, form):
    """C0 (10k LIFB + 1k POISSON, p = 0.1, 1.1e7 synapses, 1 s = 9,990 steps
    as simulate(1.0) runs them with a 15-step delay)."""
    net, v0, steps, seed, o32, o64 = c0
    mode, pers = C0_MODES[form]
    g = run_cuda(net, v0, seed, steps, mode=mode, persistent=pers, at=STEPS_100MS)
    assert len(net["src"]) == 11_000_000 and steps == 9990
    check_against_oracle("c0 " + form, net, steps, g[:4], o32, o64, vth=0.02)
    assert o32[0].sum() > 10_000


@pytest.mark.gpu
def test_c0_matches_reference_kernels(c0, tmp_path):
    """The reference's own kernels on the same C0 network and seed: raster,
    V and integer state bit-exact over the whole second."""
    net, v0, steps, seed, o32, _ = c0
    ref = T.ref_steps(net, v0, seed, steps, str(tmp_path))
    if ref is None:
        pytest.skip("the reference build (oracle/_ref) is absent")
    rc, ri, rst = ref
    gc, gi, gst, _, _ = run_cuda(net, v0, seed, steps)
    assert np.array_equal(gc, rc) and np.array_equal(gi, ri)
    assert np.array_equal(gst["V"].view(np.int32), rst["V"].view(np.int32))
    for k in ("refrac", "last_fired", "fire_cnt"):
        assert np.array_equal(gst[k], rst[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["deferred-pipelined", "deferred-windowed"])
def test_c0_driven(form):
    """C0 with its inputs at 100 Hz (17 Hz network rate, 5.6e7 events in
    300 ms): recurrent delivery at full size, the reference's kernels beside."""
    net, v0, steps = configs.build(configs.C0_DRIVEN)
    seed = configs.C0_DRIVEN["seed"]
    o32 = run_oracle(net, v0, seed, steps, T.F32, at=STEPS_100MS, nthreads=8)
    o64 = run_oracle(net, v0, seed, steps, T.F64, at=STEPS_100MS, nthreads=8)
    mode, pers = C0_MODES[form]
    g = run_cuda(net, v0, seed, steps, mode=mode, persistent=pers, at=STEPS_100MS)
    check_against_oracle("c0-driven " + form, net, steps, g[:4], o32, o64, vth=0.02)
    assert o32[0].sum() > 50_000


@pytest.fixture(scope="module")
def c1():
    net, v0, steps = configs.build(configs.C1)
    seed, off = configs.C1["seed"], configs.C1["rates_off"]
    o32 = run_oracle(net, v0, seed, steps, T.F32, rates_off=off, at=STEPS_100MS)
    o64 = run_oracle(net, v0, seed, steps, T.F64, rates_off=off, at=STEPS_100MS)
    return net, v0, steps, seed, off, o32, o64


C1_MODES = {"deferred-group": (mgb.MODE_AUTO, None), "deferred-graphs": (mgb.MODE_AUTO, 0),
            "push": (mgb.MODE_PUSH, None)}


@pytest.mark.gpu
@pytest.mark.parametrize("form", sorted(C1_MODES))
def test_c1_as_specified(c1, form):
    """C1 (4,000 shifted LIFB, p = 0.02, one-step delays, a 50 ms kick of 5 %
    of the neurons, 10 s = 100,000 steps)."""
    net, v0, steps, seed, off, o32, o64 = c1
    mode, pers = C1_MODES[form]
    g = run_cuda(net, v0, seed, steps, mode=mode, persistent=pers, rates_off=off, at=STEPS_100MS)
    assert steps == 100_000
    check_against_oracle("c1 " + form, net, steps, g[:4], o32, o64, vth=0.01)


@pytest.mark.gpu
def test_c1_matches_reference_kernels(c1, tmp_path):
    net, v0, steps, seed, off, _, _ = c1
    ref = T.ref_steps(net, v0, seed, steps, str(tmp_path), rates_off=off)
    if ref is None:
        pytest.skip("the reference build (oracle/_ref) is absent")
    rc, ri, rst = ref
    gc, gi, gst, _, _ = run_cuda(net, v0, seed, steps, rates_off=off)
    assert np.array_equal(gc, rc) and np.array_equal(gi, ri)
    for k in ("refrac", "last_fired", "fire_cnt"):
        assert np.array_equal(gst[k], rst[k]), k
    # the kicked neurons add a 20 mV and a 0.27 mV weight in one step, an
    # order-dependent fp32 sum in the reference's atomics
    np.testing.assert_allclose(gst["V"], rst["V"], rtol=RTOL, atol=RTOL * 0.01)


C3_EPOCHS = 10              # 3.5 s of the 100 s run: ten input epochs of 350 ms
C3_100MS = 200              # dt 0.5 ms


def c3_oracle(net, epochs, precision):
    o = T.OracleSim(dict(n=net["n"], type=net["type"], rate=np.zeros(net["n"], np.float32), src=net["src"],
                         tar=net["tar"], weight=net["weight"],
                         delay=np.full(len(net["src"]), stdp_net.DT, np.float32), step=np.float32(stdp_net.DT),
                         nlifconst=1, lifconst=net["lifconst"], nstdpconst=1, stdpconst=net["stdpconst"]),
                    11, stdp=1, plastic=net["plastic"], precision=precision)
    cs, ids, mid = [], [], None
    for ep in range(epochs):
        o.set_rates(stdp_net.rates(net, ep))
        if ep == 0:
            c, i = o.run(C3_100MS)
            mid = o.state()
            cs.append(c)
            ids.append(i)
            c, i = o.run(stdp_net.REDRAW_STEPS - C3_100MS)
        else:
            c, i = o.run(stdp_net.REDRAW_STEPS)
        cs.append(c)
        ids.append(i)
    return np.concatenate(cs), np.concatenate(ids), o.state(), mid


@pytest.fixture(scope="module")
def c3():
    net = stdp_net.build(n_in=784, n_exc=1600)
    return net, c3_oracle(net, C3_EPOCHS, T.F32), c3_oracle(net, C3_EPOCHS, T.F64)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["pull", "push"])
def test_c3_stdp_network(c3, mode):
    """C3 at its stated size (784 inputs -> 1,600 exc all to all, plastic;
    1:1 exc -> inh; all-but-self inh -> exc at -17 mV; 3.8e6 synapses),
    ten 350 ms input epochs: raster bit-exact for the first 100 ms, weights
    and V within 1e-5, rate and CV-ISI within 1 % over the run, and the error
    of the fp32 weights against the fp64 twin."""
    net, o32, o64 = c3
    m = {"push": mgb.MODE_PUSH, "pull": mgb.MODE_PULL}[mode]
    steps = C3_EPOCHS * stdp_net.REDRAW_STEPS
    g = mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], net["delay"],
                                  net["lifconst"], net["stdpconst"], stdp=True, plastic=net["plastic"], seed=11,
                                  mode=m, raster_steps=steps + 1)
    assert g.info()["mode"] == m and len(net["src"]) == 784 * 1600 + 1600 + 1600 * 1599
    gmid = None
    for ep in range(C3_EPOCHS):
        g.set_rates(stdp_net.rates(net, ep))
        if ep == 0:
            g.run(C3_100MS)
            g.sync()
            gmid = (g.state(), g.weights())
            g.run(stdp_net.REDRAW_STEPS - C3_100MS)
        else:
            g.run(stdp_net.REDRAW_STEPS)
    _, gc, gi = g.read_raster(max_steps=steps + 1, max_ids=net["n"] * steps // 8)
    oc, oi, ost, omid = o32
    n100 = int(oc[:C3_100MS].sum())
    assert np.array_equal(gc[:C3_100MS], oc[:C3_100MS]) and np.array_equal(gi[:n100], oi[:n100])
    np.testing.assert_allclose(gmid[1], omid["weight32"], rtol=RTOL, atol=1e-7)
    np.testing.assert_allclose(gmid[0]["V"], omid["V32"], rtol=RTOL, atol=RTOL * 20.0)
    r_o, cv_o, k_o = T.rate_and_cv(oc, oi, net["n"], steps, stdp_net.DT)
    r_g, cv_g, _ = T.rate_and_cv(gc, gi, net["n"], steps, stdp_net.DT)
    print(f"RATECV c3 {mode}: rate {r_g:.4f} Hz (oracle {r_o:.4f}), CV-ISI {cv_g:.4f} (oracle {cv_o:.4f}, "
          f"{k_o} neurons)")
    assert abs(r_g - r_o) <= 0.01 * r_o and abs(cv_g - cv_o) <= 0.01 * cv_o
    same = np.array_equal(gc, oc) and np.array_equal(gi, oi)
    w = g.weights()
    st = net["plastic"] == 0
    assert np.array_equal(w[st], net["weight"][st])
    if same:
        np.testing.assert_allclose(w, ost["weight32"], rtol=RTOL, atol=1e-7)
    c64, i64, st64, mid64 = o64
    pl = net["plastic"] == 1
    e100 = float(np.max(np.abs(gmid[1][pl].astype(np.float64) - mid64["weight"][pl])))
    print(f"FP64ERR c3 {mode} @100ms: max |w - w_fp64| = {e100:.3e} (weights in [0, 1])")
    assert e100 <= RTOL
    if np.array_equal(c64, gc) and np.array_equal(i64, gi):
        e = float(np.max(np.abs(w[pl].astype(np.float64) - st64["weight"][pl])))
        print(f"FP64ERR c3 {mode} @end: max |w - w_fp64| = {e:.3e}")
    else:
        print(f"FP64ERR c3 {mode} @end: the fp64 raster separates from the fp32 raster within the run")
