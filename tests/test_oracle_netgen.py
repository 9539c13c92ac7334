"""The oracle's gen_net restatement against networks the reference's own
gen_net produced (tests/golden/*.net, made by oracle/_ref/ref_gen)."""
import numpy as np
import pytest

import mgb_testlib as T
from cases import CASES, NAMES, load


@pytest.mark.parametrize("name", NAMES)
def test_netgen_matches_reference(name):
    c, ref, _ = load(name)
    spec = T.parse_spec(open(f"{T.GOLDEN}/{name}.spec").read())
    net = T.oracle_netgen(spec, c["mt"], c["rnd"])
    assert net["n"] == ref["n"]
    for k in ("src", "tar", "weight", "delay"):
        assert np.array_equal(net[k], ref[k]), k
    assert np.array_equal(net["type"], ref["type"])
    assert np.array_equal(net["rate"], ref["rate"])


def test_fixed_probability_cap_fills_with_first_pair():
    # netgen.cpp:210-222 walks all gen_num genlist entries; entries never
    # filled (the 1.1p Bernoulli pass fell short of gen_num) stay 0 and
    # become synapses between the first source and first target.
    spec = T.parse_spec("timestep 0.0001\npop 10 LIFB 0\npop 10 LIFB 0\n"
                        "conn 0 1 0.1 0.1 0.001 0.001 0.3 STATIC\n")
    hits = 0
    for seed in range(40):
        net = T.oracle_netgen(spec, seed, 1)
        assert len(net["src"]) == 30  # round(100 * 0.3)
        tail = (net["src"] == 0) & (net["tar"] == 10)
        hits += int(tail.sum() > 1)
    assert hits > 0


def test_connect_duplicate_rule():
    # model.cpp:99: only an existing projection at index > 0 is overwritten
    spec = T.parse_spec("pop 5 LIFB 0\npop 5 LIFB 0\n"
                        "conn 0 1 1 1 0.001 0.001 1 STATIC\n"
                        "conn 0 1 2 2 0.001 0.001 1 STATIC\n"
                        "conn 1 0 1 1 0.001 0.001 1 STATIC\n"
                        "conn 1 0 3 3 0.001 0.001 1 STATIC\n"
                        "conn 0 1 4 4 0.001 0.001 1 STATIC\n")
    # (0,1) at index 0 is appended again; (1,0) at index 2 is overwritten;
    # the last (0,1) match is then index 1 and is overwritten
    assert len(spec.pros) == 3
    assert [(p.src, p.tar, p.wmin) for p in spec.pros] == [(0, 1, 1.0), (0, 1, 4.0), (1, 0, 3.0)]


def test_one_to_one_size_mismatch_rejected():
    spec = T.parse_spec("pop 5 LIFB 0\npop 6 LIFB 0\nconn 0 1 1 1 0.001 0.001 0 STATIC\n")
    assert len(spec.pros) == 0


def test_rand_weight_subtracts_for_nonnegative_floor():
    # netgen.cpp:26-29: a range with floor >= 0 is drawn downwards from floor
    spec = T.parse_spec("timestep 0.0001\ndw 0.01\npop 20 LIFB 0\npop 20 LIFB 0\n"
                        "conn 0 1 0.2 0.5 0.001 0.001 1 STATIC\n")
    net = T.oracle_netgen(spec, 1, 3)
    assert net["weight"].max() <= np.float32(0.2) and net["weight"].min() < 0.0


@pytest.mark.parametrize("cfg", ["C0", "C1", "C0R"])
def test_netgen_matches_reference_at_config_size(cfg, tmp_path):
    """The benchmark configurations at their stated sizes (C0: 1.1e7
    synapses; C1: 3.2e5): the oracle's gen_net against the reference's own
    (oracle/_ref/ref_gen), synapse for synapse."""
    import os

    import configs
    if not os.path.exists(T.REF_GEN):
        pytest.skip("the reference build (oracle/_ref) is absent")
    c = getattr(configs, cfg)
    ref = T.ref_gen(c["spec"], c["mt"], c["rnd"], str(tmp_path / "ref.net"))
    net = T.oracle_netgen(T.parse_spec(c["spec"]), c["mt"], c["rnd"])
    assert net["n"] == ref["n"] and len(net["src"]) == len(ref["src"]) > 0
    for k in ("src", "tar", "weight", "delay"):
        assert np.array_equal(net[k], ref[k]), k
    assert np.array_equal(net["type"], ref["type"]) and np.array_equal(net["rate"], ref["rate"])
    assert np.array_equal(ref["lifconst"], configs.lifconst(*c["lif"]))
