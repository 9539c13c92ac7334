"""Connection rules the reference's ctype cannot express, added to the C++
API (Model::connect_fixed_indegree, Model::connect_all_but_self): NetGen
builds them into the same Network struct.  The fixed in-degree rule draws
exactly the synapses of the device generator (checked against the oracle's
restatement of that generator); all-but-self leaves out i -> i only."""
import collections
import os
import subprocess

import numpy as np
import pytest

import mgb_testlib as T
from mgbrain_b200 import netfile

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..")

SPEC = """timestep 0.0001
pop 300 LIFB 0
pop 120 LIFB 0
pop 80 POISSON 1
fixed_indegree 0 0 40 0.0001 0.001 0.003 77 STATIC
fixed_indegree 1 0 15 -0.0005 0.001 0.001 77 STATIC
fixed_indegree 2 1 9 0.0002 0.0015 0.0025 77 STATIC
all_but_self 1 1 -0.0003 -0.0003 0.002 0.002 STATIC
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "api_driver")
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(ROOT, "tests", "cpp", "api_driver.cpp"),
                    "-L" + os.path.join(ROOT, "mgbrain_b200", "lib"), "-lmgbrain_b200",
                    "-Wl,-rpath," + os.path.join(ROOT, "mgbrain_b200", "lib")], check=True)
    return exe


def test_fixed_indegree_and_all_but_self(driver, tmp_path):
    spec = tmp_path / "r.spec"
    spec.write_text(SPEC)
    out = str(tmp_path / "r.net")
    subprocess.run([driver, "gen", str(spec), out], check=True, capture_output=True)
    net = netfile.read_netfile(out)
    steps = netfile.delay_steps(net)
    src, tar, w = net["src"], net["tar"], net["weight"]
    # the oracle's restatement of the device generator, same projections
    pops = [(0, 300, 5), (300, 120, 5), (420, 80, 2)]
    projs = [(0, 0, 40, 1e-4, 10, 30), (1, 0, 15, -5e-4, 10, 10), (2, 1, 9, 2e-4, 15, 25)]
    L = T.oracle()
    P = np.array(pops, np.int32)
    a = lambda x, dt: np.ascontiguousarray(x, dt)  # noqa: E731
    keep = [a(P[:, 0], np.int32), a(P[:, 1], np.int32), a(P[:, 2], np.int32),
            a([r[0] for r in projs], np.int32), a([r[1] for r in projs], np.int32),
            a([r[2] for r in projs], np.int32), a([r[3] for r in projs], np.float32),
            a([r[4] for r in projs], np.int32), a([r[5] for r in projs], np.int32)]
    rate = np.zeros(500, np.float32)
    h = L.mgbo_create_fixed_indegree(*[T._p(k) for k in keep[:3]], len(P), *[T._p(k) for k in keep[3:]],
                                     len(projs), T._p(rate), None, T._p(np.zeros(30, np.float32)), 77, 1, 1, 0, 0)
    try:
        S = int(L.mgbo_n_syn(h))
        rp = np.zeros(501, np.int64)
        tg = np.zeros(S, np.int32)
        ow = np.zeros(S, np.float32)
        od = np.zeros(S, np.int32)
        L.mgbo_export_csr(h, T._p(rp), T._p(tg), T._p(ow), T._p(od))
    finally:
        L.mgbo_destroy(h)
    osrc = np.repeat(np.arange(500, dtype=np.int32), np.diff(rp))
    fid = len(src) - 120 * 119            # the fixed in-degree synapses come first
    assert fid == S
    mine = collections.Counter(zip(src[:fid].tolist(), tar[:fid].tolist(), steps[:fid].tolist(),
                                   w[:fid].tolist()))
    theirs = collections.Counter(zip(osrc.tolist(), tg.tolist(), od.tolist(), ow.tolist()))
    assert mine == theirs
    # all-but-self: every pair of pop 1 except i -> i, in row-major order
    abs_src, abs_tar = src[fid:] - 300, tar[fid:] - 300
    pairs = [(i, j) for i in range(120) for j in range(120) if i != j]
    assert list(zip(abs_src.tolist(), abs_tar.tolist())) == pairs
    assert np.all(steps[fid:] == 20)
