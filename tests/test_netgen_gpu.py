"""NetGen's rules generated on the device (mgc_create_generated) against the
networks the reference's gen_net made: the golden networks (the reference's
own gen_net output), the benchmark configurations at their stated sizes
(the oracle's gen_net, pinned to the reference's), and the rules the
reference cannot express (all-but-self, fixed in-degree) against their
explicit lists.  Same synapses in the same order: the CSR, the weights in
synapse-list order, the delay range and the accumulation plan are equal to
those of the handle built from the list."""
import numpy as np
import pytest

import configs
import mgb_testlib as T
import mgbrain_b200 as mgb
import stdp_net
from cases import CASES, NAMES, load


def list_handle(net, v0=None, seed=1, **kw):
    dsteps, _, _ = T.quantize_delays(net["delay"], net["step"])
    return mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], dsteps,
                                     T.default_lifconst(net), T.default_stdpconst(net), rate=net["rate"], v_init=v0,
                                     seed=seed, **kw)


def generated_handle(spec, net, mt_seed, v0=None, seed=1, **kw):
    pops = [(p[0], p[1]) for p in spec.pops]
    return mgb.Simulator.generated(pops, T.gen_projs(spec, net), T.default_lifconst(net), mt_seed=mt_seed,
                                   stdpconst=T.default_stdpconst(net), rate=net["rate"], v_init=v0, seed=seed, **kw)


def same_network(a, b):
    ra, ta, wa, da = a.export_csr()
    rb, tb, wb, db = b.export_csr()
    assert np.array_equal(ra, rb), "row offsets differ"
    assert np.array_equal(ta, tb) and np.array_equal(da, db), "targets or delays differ"
    assert np.array_equal(wa.view(np.int32), wb.view(np.int32)), "weights differ"
    assert np.array_equal(a.weights().view(np.int32), b.weights().view(np.int32)), "synapse-list order differs"
    ia, ib = a.info(), b.info()
    for k in ("n_neurons", "n_synapses", "min_delay", "max_delay", "mode", "accumulation", "fx_shift"):
        assert ia[k] == ib[k], k


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_golden_networks(name):
    """The reference's own gen_net output (tests/golden/<case>.net) from the
    same mt19937 seed: synapse for synapse, and the same raster after 500 steps."""
    c, gold, v0 = load(name)
    spec = T.parse_spec(open(f"{T.GOLDEN}/{name}.spec").read())
    net = T.oracle_netgen(spec, c["mt"], c["rnd"])   # for the projection index of each synapse
    for k in ("src", "tar", "weight", "delay"):
        assert np.array_equal(net[k], gold[k]), k
    gold = dict(gold, proj=net["proj"])
    a = list_handle(gold, v0, c["seed"], stdp=bool(c["stdp"]))
    b = generated_handle(spec, gold, c["mt"], v0, c["seed"], stdp=bool(c["stdp"]))
    same_network(a, b)
    a.run(500)
    b.run(500)
    _, ca, ia = a.read_raster()
    _, cb, ib = b.read_raster()
    assert np.array_equal(ca, cb) and np.array_equal(ia, ib)


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", ["C0", "C0R", "C1"])
def test_configurations_at_stated_size(cfg):
    c = getattr(configs, cfg)
    spec = T.parse_spec(c["spec"])
    net = T.oracle_netgen(spec, c["mt"], c["rnd"])
    net["lifconst"], net["nlifconst"] = configs.lifconst(*c["lif"]), 1
    state = []
    b = generated_handle(spec, net, c["mt"], state_out=state)
    a = list_handle(net)
    same_network(a, b)
    assert len(state) == 624


@pytest.mark.gpu
def test_generator_state_carries_over():
    """Two fixed-probability projections generated one after the other equal
    the second generated alone from the state the first one left."""
    spec = T.parse_spec("timestep 0.0001\npop 3000 LIFB 0\npop 2000 LIFB 0\n"
                        "conn 0 1 0.001 0.001 0.001 0.001 0.2 STATIC\nconn 1 0 -0.002 -0.002 0.002 0.002 0.05 STATIC\n")
    net = T.oracle_netgen(spec, 77, 1)
    lif = np.zeros(30, np.float32)
    lif[0], lif[4] = 1e-4, 0.02
    pops = [(p[0], p[1]) for p in spec.pops]
    projs = T.gen_projs(spec, net)
    mid = []
    mgb.Simulator.generated(pops, projs[:1], lif, mt_seed=77, state_out=mid)
    second = mgb.Simulator.generated(pops, projs[1:], lif, mt_state=mid)
    sel = net["proj"] == 1
    part = dict(net, src=net["src"][sel], tar=net["tar"][sel], weight=net["weight"][sel], delay=net["delay"][sel],
                lifconst=lif, nlifconst=1)
    same_network(list_handle(part), second)
    assert int(sel.sum()) == round(3000 * 2000 * 0.05) and int((~sel).sum()) == round(3000 * 2000 * 0.2)


@pytest.mark.gpu
def test_rules_beyond_the_reference():
    """C3's layers: all-to-all input -> exc with drawn weights, exc -> inh one to
    one, inh -> exc all but self (the rule the reference cannot express), as
    stdp_net.build lists them; and fixed in-degree against the fixed in-degree
    device generator."""
    net = stdp_net.build(n_in=784, n_exc=400)
    nin, ne = net["n_in"], net["n_exc"]
    n1 = nin * ne
    projs = [dict(src=0, tar=1, rule=mgb.RULE_ALL, weights=net["weight"][:n1], delay=1, plastic=1),
             dict(src=1, tar=2, rule=mgb.RULE_ONE, weight=25.0, delay=1),
             dict(src=2, tar=1, rule=mgb.RULE_ALL_BUT_SELF, weight=-17.0, delay=1)]
    pops = [(nin, mgb.POISSON), (ne, mgb.LIFB), (ne, mgb.LIFB)]
    g = mgb.Simulator.generated(pops, projs, net["lifconst"], stdpconst=net["stdpconst"], stdp=True,
                                mode=mgb.MODE_PUSH)
    a = mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], net["delay"],
                                  net["lifconst"], net["stdpconst"], stdp=True, plastic=net["plastic"],
                                  mode=mgb.MODE_PUSH)
    same_network(a, g)
    # fixed in-degree: the same draws as mgc_create_fixed_indegree
    lif = np.zeros(30, np.float32)
    lif[0], lif[3], lif[4], lif[8] = 1e-4, 0.01, 0.02, 0.002
    pops_f = [(0, 4000, mgb.LIFB), (4000, 1000, mgb.LIFB), (5000, 500, mgb.POISSON)]
    fprojs = [(0, 0, 80, 1e-4, 10, 50), (1, 0, 20, -5e-4, 10, 50), (2, 1, 10, 1e-4, 10, 50)]
    f = mgb.Simulator.fixed_indegree(pops_f, fprojs, lif, conn_seed=33)
    gp = [dict(src=s, tar=t, rule=mgb.RULE_FIXED_INDEGREE, k=k, conn_seed=33, weight=w, delay=d0, delay_max=d1)
          for s, t, k, w, d0, d1 in fprojs]
    gf = mgb.Simulator.generated([(p[1], p[2]) for p in pops_f], gp, lif)
    rf, tf, wf, df = f.export_csr()
    rg, tg, wg, dg = gf.export_csr()
    assert np.array_equal(rf, rg) and np.array_equal(wf, wg)
    # the fixed in-degree builder buckets rows by delay; compare each row as (delay, target) pairs
    for i in np.random.default_rng(1).choice(len(rf) - 1, 300, replace=False):
        a0, a1 = rf[i], rf[i + 1]
        assert sorted(zip(df[a0:a1], tf[a0:a1])) == sorted(zip(dg[a0:a1], tg[a0:a1]))


@pytest.mark.gpu
def test_bad_descriptions_are_refused():
    lif = np.zeros(30, np.float32)
    lif[0] = 1e-4
    with pytest.raises(mgb.MgcError):   # one to one needs equal populations
        mgb.Simulator.generated([(10, mgb.LIFB), (12, mgb.LIFB)], [dict(src=0, tar=1, rule=mgb.RULE_ONE)], lif)
    with pytest.raises(mgb.MgcError):   # population out of range
        mgb.Simulator.generated([(10, mgb.LIFB)], [dict(src=0, tar=3, rule=mgb.RULE_ALL)], lif)
    with pytest.raises(mgb.MgcError):   # a delay of zero steps
        mgb.Simulator.generated([(10, mgb.LIFB)], [dict(src=0, tar=0, rule=mgb.RULE_ALL, delay=0)], lif)
