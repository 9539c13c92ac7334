"""A network split into partitions (one handle per neuron range, spike ids
exchanged every min_delay - 1 steps) runs exactly as the whole network:
merged rasters and concatenated state equal the single handle's, for
synapse-list and device-generated networks, in every step-group mode, for
uneven partition sizes, and across processes exchanging through
torch.distributed.  Misuse is refused with a status, never run."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch

import mgb_testlib as T
import mgbrain_b200 as mgb
from cases import load
from mgbrain_b200.partition import PartitionGroup, merge_rasters, split

import bench

HERE = os.path.dirname(os.path.abspath(__file__))


def explicit_args(name):
    c, net, v0 = load(name)
    dsteps, _, _ = T.quantize_delays(net["delay"], net["step"])
    args = (net["n"], net["type"], net["src"], net["tar"], net["weight"], dsteps, T.default_lifconst(net))
    kw = dict(rate=net["rate"], v_init=v0, seed=c["seed"])
    return net, args, kw


def equal_weights(w):
    return len(np.unique(w[w > 0])) <= 1 and len(np.unique(w[w <= 0])) <= 1


def compare(whole, group, exact_v):
    wf, wc, wi = whole.read_raster()
    pf, pc, pi = group.raster()
    assert pf == wf
    assert np.array_equal(pc, wc), "spike counts per step differ"
    assert np.array_equal(pi, wi), "spike ids differ"
    assert wc.sum() > 0
    ws = whole.state()
    ps = group.state()
    for k in ("refrac", "last_fired", "fire_cnt"):
        assert np.array_equal(ps[k], ws[k]), k
    if exact_v:
        assert np.array_equal(ps["V"].view(np.int32), ws["V"].view(np.int32)), "V not bit-exact"
    else:
        np.testing.assert_allclose(ps["V"], ws["V"], rtol=1e-5, atol=1e-8)
    assert sum(s.info()["events"] for s in group.sims) == whole.info()["events"]


@pytest.mark.gpu
@pytest.mark.parametrize("cap", [None, 64])
@pytest.mark.parametrize("parts", [2, 3])
@pytest.mark.parametrize("name", ["c0s", "brunel_maker", "lif_mixed"])
def test_explicit_partitions_equal_whole(name, parts, cap):
    net, args, kw = explicit_args(name)
    whole = mgb.Simulator.from_arrays(*args, **kw)
    whole.run(2000)
    sims = [mgb.Simulator.from_arrays(*args, **kw, part=p) for p in split(net["n"], parts)]
    for s, (first, count) in zip(sims, split(net["n"], parts)):
        assert s.first == first and s.n == count and s.n_src == net["n"]
        assert s.info()["mode"] == mgb.MODE_DEFERRED
    assert sum(s.S for s in sims) == len(net["src"])
    # unequal weights of one sign: every partition sums in fixed point with
    # the whole network's shift, so the merged state is the same bits
    wi = whole.info()
    for s in sims:
        assert (s.info()["accumulation"], s.info()["fx_shift"]) == (wi["accumulation"], wi["fx_shift"])
    assert wi["accumulation"] == (mgb.ACC_FLOAT if equal_weights(net["weight"]) else mgb.ACC_FIXED)
    g = PartitionGroup(sims, cap_per_step=cap)   # exact exchange, or the device one with 64 ids per step
    g.run(700)
    g.run(1300)
    g.sync()
    compare(whole, g, True)


def fixed(w, **kw):
    return mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], rate=w["rate"], v_init=w["v0"],
                                        conn_seed=11, seed=12, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("cap", [None, 2048])
@pytest.mark.parametrize("persistent", [0, 1, 2, 3])
def test_fixed_indegree_partitions_equal_whole(persistent, cap):
    w = bench.workload(scale=0.02, nu=0.02)
    whole = fixed(w)
    whole.set_persistent(persistent)
    whole.run(3000)
    ranges = [(0, 7001), (7001, 9000), (16001, w["n"] - 16001)]  # uneven, cutting populations
    sims = [fixed(w, part=p) for p in ranges]
    for s in sims:
        s.set_persistent(persistent)
    assert sum(s.S for s in sims) == whole.S
    g = PartitionGroup(sims, cap_per_step=cap)
    assert g.window == 9
    g.run(3000)
    g.sync()
    for s in sims:
        assert s.info()["persistent"] == persistent
    compare(whole, g, True)


@pytest.mark.gpu
def test_partition_misuse_is_refused():
    w = bench.workload(scale=0.01)
    n = w["n"]
    with pytest.raises(mgb.MgcError):
        fixed(w, part=(n - 10, 20))          # past the network's end
    with pytest.raises(mgb.MgcError):
        fixed(w, part=(0, 0))
    projs = [(s, t, k, wt, 1, 5) for (s, t, k, wt, _, _) in w["projs"]]
    with pytest.raises(mgb.MgcError):       # min_delay 1: no exchange window
        mgb.Simulator.fixed_indegree(w["pops"], projs, w["lif"], rate=w["rate"], part=(0, n // 2))
    net, args, kw = explicit_args("stdp_small")
    with pytest.raises(mgb.MgcError):       # plastic weights need the other methods
        mgb.Simulator.from_arrays(*args, **kw, stdp=True, part=(0, net["n"] // 2))
    a, b = fixed(w, part=(0, n // 2)), fixed(w, part=(n // 2, n - n // 2))
    with pytest.raises(mgb.MgcError):       # more steps than the window
        a.run(10)
    with pytest.raises(mgb.MgcError):
        a.autotune(64)
    a.run(4)
    a.run(5)
    with pytest.raises(mgb.MgcError):
        a.run(1)
    buf = torch.empty(a.n * 9, dtype=torch.int32, device="cuda")
    with pytest.raises(mgb.MgcError):       # the window is 9 steps, not 8
        a.part_export(8, buf)
    counts, total = a.part_export(9, buf)
    assert len(counts) == 9 and total == counts.sum()
    small = torch.empty(1, dtype=torch.int32, device="cuda")
    if total > 1:
        with pytest.raises(mgb.MgcError):   # does not fit: reported, counts still given
            a.part_export(9, small)
    with pytest.raises(mgb.MgcError):       # host memory is not accepted as the id buffer
        a.part_export(9, torch.empty(a.n * 9, dtype=torch.int32))
    # an id outside the network refuses the import; nothing is delivered from it
    C = np.zeros((2, 9), np.int32)
    C[1, 3] = 2
    with pytest.raises(mgb.MgcError):      # rank 1's 2 ids do not fit a stride of 1 (checked on the host)
        a.part_import(9, 0, C, torch.tensor([0, 5], dtype=torch.int32, device="cuda"), 1)
    bad = torch.tensor([0, 0, 5, n + 7], dtype=torch.int32, device="cuda")  # 2 ranks x stride 2
    with pytest.raises(mgb.MgcError):      # checked by the import kernel
        a.part_import(9, 0, C, bad, 2)
    with pytest.raises(mgb.MgcError):
        a.sync()
    a.close()
    b.close()


@pytest.mark.gpu
def test_device_exchange_overflow_is_refused():
    """A window with more spikes than the device exchange holds is refused on
    every partition, and the next sync says so."""
    w = bench.workload(scale=0.02, nu=0.05)
    sims = [fixed(w, part=p) for p in split(w["n"], 2)]
    g = PartitionGroup(sims, cap_per_step=1)
    g.run(200)
    for s in sims:
        with pytest.raises(mgb.MgcError) as e:
            s.sync()
        assert "exchange" in str(e.value)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.gpu
def test_two_processes_exchange_through_gloo():
    """Two ranks, each with its partition on this GPU, exchanging spike ids
    through gloo all-gathers; rank 0 compares the merged result with the
    whole network.  (One process per GPU with NCCL is the deployment form;
    here both ranks share the one GPU and their kernels never wait on each
    other.)"""
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK="0", WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "partition_worker.py"), "gpu"], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=600)
        assert p.returncode == 0, e[-3000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    assert outs[0]["equal"], outs[0]
    assert outs[0]["spikes"] > 0
