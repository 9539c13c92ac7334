"""The MGBNET02 network file round-trips, and the package's delay
quantisation equals the oracle's restatement of build_multinet on every
golden network."""
import glob
import os

import numpy as np

import mgb_testlib as T
from mgbrain_b200 import netfile

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_roundtrip(tmp_path):
    net = netfile.read_netfile(os.path.join(GOLDEN, "lif_mixed.net"))
    p = str(tmp_path / "x.net")
    netfile.write_netfile(p, net)
    back = netfile.read_netfile(p)
    for k in ("type", "rate", "src", "tar", "weight", "delay", "lifconst", "stdpconst", "pops"):
        assert np.array_equal(back[k], net[k]), k
    assert back["n"] == net["n"] and back["step"] == net["step"]


def test_delay_steps_match_oracle():
    nets = sorted(glob.glob(os.path.join(GOLDEN, "*.net")))
    assert len(nets) >= 6
    for p in nets:
        net = netfile.read_netfile(p)
        q, _, _ = T.quantize_delays(net["delay"], np.float32(net["step"]))
        assert np.array_equal(q, netfile.delay_steps(net)), p
