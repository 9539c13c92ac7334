"""Partition cut and balance statistics computed on the device from the
handle's CSR (mgc_partition_stats) equal the host loops of the reference's
PartitionAnalysis (cost = synapses whose ends lie in different zones; zone
neurons, synapses by source zone, crossing synapses by source and by target
zone), restated here in numpy over the exported CSR."""
import numpy as np
import pytest

import mgbrain_b200 as mgb
from mgbrain_b200.partition import split

import bench
from test_partition_gpu import explicit_args


def host_stats(src, tar, part, nparts, n):
    zs, zt = part[src], part[tar]
    x = zs != zt
    return dict(cut=int(x.sum()), zone_neurons=np.bincount(part[:n], minlength=nparts),
                zone_syn=np.bincount(zs, minlength=nparts), zone_out=np.bincount(zs[x], minlength=nparts),
                zone_in=np.bincount(zt[x], minlength=nparts))


def check(got, want):
    assert got["cut"] == want["cut"]
    for k in ("zone_neurons", "zone_syn", "zone_out", "zone_in"):
        assert np.array_equal(got[k], want[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("nparts", [1, 3, 7])
def test_stats_match_host_loops(nparts):
    net, args, kw = explicit_args("c0s")
    s = mgb.Simulator.from_arrays(*args, **kw)
    n = net["n"]
    part = np.random.default_rng(nparts).integers(0, nparts, n).astype(np.int32)
    src = np.asarray(net["src"], np.int64)
    tar = np.asarray(net["tar"], np.int64)
    check(s.partition_stats(part, nparts), host_stats(src, tar, part, nparts, n))


@pytest.mark.gpu
def test_stats_of_generated_network_and_partition_handle():
    w = bench.workload(scale=0.01)
    mk = dict(rate=w["rate"], v_init=w["v0"], conn_seed=9)
    whole = mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], **mk)
    n = w["n"]
    part = np.zeros(n, np.int32)
    for z, (first, count) in enumerate(split(n, 4)):
        part[first:first + count] = z
    rp, tgt, _, _ = whole.export_csr()
    src = np.repeat(np.arange(n), np.diff(rp))
    want = host_stats(src, tgt.astype(np.int64), part, 4, n)
    check(whole.partition_stats(part, 4), want)
    # a partition handle counts the synapses that target its own neurons
    first, count = split(n, 4)[2]
    p = mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], part=(first, count), **mk)
    sel = (tgt >= first) & (tgt < first + count)
    want_p = host_stats(src[sel], tgt[sel].astype(np.int64), part, 4, n)
    check(p.partition_stats(part, 4), want_p)
    with pytest.raises(mgb.MgcError):
        whole.partition_stats(np.full(n, 4, np.int32), 4)   # zone out of range
