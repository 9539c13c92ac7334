"""The MGBrain C++ API (include/mgbrain.h) of mgbrain_b200, exercised by a
program written like the reference's bench mains (tests/cpp/api_driver.cpp):
its NetGen must reproduce the reference's networks and its MGSimulator must
follow the reference's simulate() rules."""
import json
import os
import subprocess

import numpy as np
import pytest

import mgb_testlib as T
from cases import CASES, NAMES, load

ROOT = T.ROOT
LIBDIR = os.path.join(ROOT, "mgbrain_b200", "lib")


@pytest.fixture(scope="session")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "api_driver")
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    "-o", exe, os.path.join(ROOT, "tests", "cpp", "api_driver.cpp"),
                    "-L" + LIBDIR, "-lmgbrain_b200", "-Wl,-rpath," + LIBDIR], check=True)
    return exe


def _env(c):
    return dict(os.environ, MGB_MT_SEED=str(c["mt"]), MGB_RAND_SEED=str(c["rnd"]),
                MGB_SEED=str(c["seed"]))


@pytest.mark.parametrize("name", NAMES)
def test_cpp_netgen_matches_reference(driver, tmp_path, name):
    c, ref, _ = load(name)
    out = str(tmp_path / "n.net")
    subprocess.run([driver, "gen", os.path.join(T.GOLDEN, name + ".spec"), out], check=True,
                   env=_env(c), capture_output=True)
    net = T.read_netfile(out)
    for k in ("src", "tar", "weight", "delay", "type", "rate", "lifconst", "stdpconst"):
        assert np.array_equal(net[k], ref[k]), k
    assert net["nlifconst"] == ref["nlifconst"] and net["nstdpconst"] == ref["nstdpconst"]


@pytest.mark.gpu
@pytest.mark.parametrize("autotune", [0, 64])
@pytest.mark.parametrize("name", [n for n in NAMES if CASES[n].get("simulate")])
def test_cpp_simulate_matches_oracle_and_reference(driver, tmp_path, name, autotune):
    """simulate(t) runs the reference's effective step count (the remainder
    after the last whole min_delay cycle is dropped) and ends in the state
    the oracle reaches after that many steps; with Config::enable_autotune
    the tuner's trial steps before the first step are undone."""
    c, net, v0 = load(name)
    pre = str(tmp_path / "s")
    v0p = os.path.join(T.GOLDEN, name + ".v0")
    r = subprocess.run([driver, "simulate", os.path.join(T.GOLDEN, name + ".spec"), pre,
                        str(c["simulate"]), v0p if os.path.exists(v0p) else "-", str(c["stdp"])],
                       check=True, env=dict(_env(c), MGB_AUTOTUNE=str(autotune)), capture_output=True, text=True)
    assert "fire rate:" in r.stdout
    o = T.OracleSim(net, c["seed"], v0=v0, stdp=c["stdp"])
    steps = T.oracle().mgbo_steps_for_time(np.float32(c["simulate"]), np.float32(net["step"]))
    eff = T.oracle().mgbo_effective_steps(steps, o.dmin)
    counts, ids = o.run(eff)
    ost = o.state()
    n, S = net["n"], len(net["src"])
    b = open(pre + ".state", "rb").read()
    v = np.frombuffer(b, np.float32, n, 0)
    fc = np.frombuffer(b, np.int32, n, 4 * n)
    gc, gi = T.read_raster(pre + ".raster")
    assert len(gc) == eff
    assert np.array_equal(gc, counts) and np.array_equal(gi, ids)
    assert np.array_equal(v.view(np.int32), ost["V32"].view(np.int32))
    assert np.array_equal(fc, ost["fire_cnt"])
    sim_state = os.path.join(T.GOLDEN, name + ".sim.state")
    if os.path.exists(sim_state):
        rs = T.read_state(sim_state, n, S)
        assert np.array_equal(fc, rs["fire_cnt"])
        assert np.array_equal(v.view(np.int32), rs["V"].view(np.int32))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c0s", "brunel_maker"])
def test_cpp_partitions_run_as_separate_handles(driver, tmp_path, name):
    """mgsim(net, part, 3) with SIMPLE partitions: without enable_single_gpu
    each partition is its own handle (exchanging spike ids), with it the
    network is one handle; both end exactly where npart = 1 ends."""
    c, net, _ = load(name)
    v0p = os.path.join(T.GOLDEN, name + ".v0")
    outs = {}
    for tag, extra in (("one", []), ("multi", ["3", "multi"]), ("single", ["3", "single"])):
        pre = str(tmp_path / tag)
        r = subprocess.run([driver, "simulate", os.path.join(T.GOLDEN, name + ".spec"), pre, "0.2",
                            v0p if os.path.exists(v0p) else "-", "0"] + extra,
                           check=True, env=_env(c), capture_output=True, text=True)
        outs[tag] = (open(pre + ".state", "rb").read(), open(pre + ".raster", "rb").read(), r.stdout)
    assert "handles 3" in outs["multi"][2] and "run multi-net on" in outs["multi"][2]
    assert "handles 1" in outs["single"][2] and "run multi-net on single-GPU" in outs["single"][2]
    for tag in ("multi", "single"):
        assert outs[tag][0] == outs["one"][0], tag
        assert outs[tag][1] == outs["one"][1], tag


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cpp_device_netgen_equals_host_netgen(driver, tmp_path, name):
    """config::enable_device_netgen(): gen_net records the projections and the
    simulator generates the synapses on the device; the run ends in exactly
    the state (V, fire counts, weights in synapse order) and raster of the
    host-generated network, and the rand() stream advances as gen_net's."""
    c, _, _ = load(name)
    v0p = os.path.join(T.GOLDEN, name + ".v0")
    outs = {}
    for dev in ("0", "1"):
        pre = str(tmp_path / ("dev" + dev))
        r = subprocess.run([driver, "simulate", os.path.join(T.GOLDEN, name + ".spec"), pre, "0.1",
                            v0p if os.path.exists(v0p) else "-", str(c["stdp"])],
                           check=True, env=dict(_env(c), MGB_DEVICE_NETGEN=dev), capture_output=True, text=True)
        outs[dev] = (open(pre + ".state", "rb").read(), open(pre + ".raster", "rb").read(), r.stdout)
    assert outs["1"][0] == outs["0"][0]
    assert outs["1"][1] == outs["0"][1]
    assert len(outs["0"][1]) > 16
