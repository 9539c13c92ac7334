"""Failure handling, tested without a GPU fault: allocation failures injected
on the host at every allocation of a build (each returns MGC_ERR_NOMEM and
leaks nothing); invalid synapse lists caught by validation before any kernel
uses them; a raster buffer too small for the run reported as an overflow
while the simulation itself is unaffected; the step groups' bounded waits
run out on a counter nothing advances and leave the device usable; and
run-twice determinism, bit for bit, of the methods that promise it."""
import gc

import numpy as np
import pytest
import torch

import mgb_testlib as T
import mgbrain_b200 as mgb
from cases import load

import bench


def args_of(name):
    c, net, v0 = load(name)
    dsteps, _, _ = T.quantize_delays(net["delay"], net["step"])
    return net, (net["n"], net["type"], net["src"], net["tar"], net["weight"], dsteps,
                 T.default_lifconst(net)), dict(rate=net["rate"], v_init=v0, seed=c["seed"])


def small_fixed(**kw):
    w = bench.workload(scale=0.01)
    return mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], rate=w["rate"], v_init=w["v0"],
                                        conn_seed=5, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("build", ["explicit", "fixed", "partition"])
def test_every_allocation_failure_is_reported_and_freed(build):
    net, args, kw = args_of("c0s")

    def make():
        if build == "explicit":
            return mgb.Simulator.from_arrays(*args, **kw)
        if build == "fixed":
            return small_fixed()
        return mgb.Simulator.from_arrays(*args, **kw, part=(100, 300))

    make().close()                   # warm: library, context, allocator pools
    gc.collect()                     # handles other tests left to the garbage collector go first
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    k = 1
    while True:
        mgb.fault_inject_alloc(k)
        try:
            s = make()
        except mgb.MgcError as e:
            assert e.status == mgb.capi.MGC_ERR_NOMEM, (k, str(e))
            k += 1
            assert k < 500
            continue
        finally:
            mgb.fault_inject_alloc(0)
        s.run(10)                    # within a partition's exchange window
        s.sync()
        s.close()
        break
    assert k > 5                     # the build allocates in several places
    gc.collect()
    torch.cuda.synchronize()
    # nothing leaked: free memory did not shrink (it may grow, when memory
    # other code held is released meanwhile)
    assert torch.cuda.mem_get_info()[0] > free0 - (64 << 20)


@pytest.mark.gpu
def test_invalid_synapses_are_refused():
    net, args, kw = args_of("c0s")
    n = net["n"]
    for field, bad in (("tar", n), ("src", -1), ("src", n + 3)):
        a = list(args)
        arr = np.array(a[2 if field == "src" else 3])
        arr[17] = bad
        a[2 if field == "src" else 3] = arr
        with pytest.raises(mgb.MgcError) as e:
            mgb.Simulator.from_arrays(*a, **kw)
        assert e.value.status == mgb.capi.MGC_ERR_INVALID
    a = list(args)
    d = np.array(a[5])
    d[5] = 0
    a[5] = d
    with pytest.raises(mgb.MgcError):
        mgb.Simulator.from_arrays(*a, **kw)
    s = mgb.Simulator.from_arrays(*args, **kw)   # the device is still fine
    s.run(100)
    s.sync()
    s.close()


@pytest.mark.gpu
def test_raster_overflow_is_reported_and_state_unaffected():
    net, args, kw = args_of("brunel_maker")
    full = mgb.Simulator.from_arrays(*args, **kw)
    tiny = mgb.Simulator.from_arrays(*args, **kw, raster_ids=16)
    full.run(500)
    tiny.run(500)
    _, counts, _ = full.read_raster()
    assert counts.sum() > 16
    with pytest.raises(mgb.MgcError) as e:
        tiny.read_raster()
    assert e.value.status == mgb.capi.MGC_ERR_OVERFLOW
    assert np.array_equal(full.state()["V"], tiny.state()["V"])
    assert np.array_equal(full.state()["fire_cnt"], tiny.state()["fire_cnt"])


@pytest.mark.gpu
@pytest.mark.parametrize("which", [0, 1])
def test_bounded_waits_give_up_and_device_stays_usable(which):
    st, ms = mgb.selftest_wait_timeout(which)
    assert st & 4, st
    assert 0 < ms < 30_000
    s = small_fixed()
    s.set_persistent(2 if which == 0 else 1)
    s.run(2000)
    s.sync()                         # the handle's own step groups finish normally
    assert s.info()["step"] == 2000
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,mode", [("c0s", mgb.MODE_DEFERRED), ("c0s", mgb.MODE_PUSH),
                                       ("lif_mixed", mgb.MODE_PULL), ("stdp_small", mgb.MODE_PULL)])
def test_run_twice_is_bitwise_identical(name, mode):
    c, _, _ = load(name)
    net, args, kw = args_of(name)
    out = []
    for _ in range(2):
        s = mgb.Simulator.from_arrays(*args, **kw, mode=mode, stdp=bool(c["stdp"]))
        s.run(1500)
        _, counts, ids = s.read_raster()
        st = s.state()
        out.append((counts, ids, st["V"].view(np.int32), s.weights().view(np.int32)))
        s.close()
    for x, y in zip(out[0], out[1]):
        assert np.array_equal(x, y)
