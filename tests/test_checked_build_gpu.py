"""The index-checking build (libmgbrain_b200_checked.so, selected with
MGBRAIN_LIB=checked): the GPU parity, step-group, partition, STDP, failure,
batch, checkpoint, edge-case and staged-readout suites pass with every index the kernels
read from memory tested before use, and no test fires (a fired test would
make sync raise).  This is the project's stand-in for a memory checker, which
is not available on the GPU machines here."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SUITES = ["tests/test_parity_gpu.py", "tests/test_persistent_gpu.py", "tests/test_partition_gpu.py",
          "tests/test_stdp_net.py", "tests/test_faults_gpu.py", "tests/test_batch.py",
          "tests/test_checkpoint_gpu.py", "tests/test_edge_cases_gpu.py", "tests/test_raster_stage_gpu.py"]

PROBE = """
import mgbrain_b200 as mgb, bench
assert mgb.capi.LIB_PATH.endswith("libmgbrain_b200_checked.so"), mgb.capi.LIB_PATH
w = bench.workload(scale=0.02, nu=0.02)
for p in (0, 1, 2):
    s = mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], rate=w["rate"], v_init=w["v0"], conn_seed=3)
    s.set_persistent(p)
    s.run(2000)
    s.sync()
    assert s.info()["events"] > 0
print("checked build ok")
"""


@pytest.mark.gpu
def test_parity_suites_pass_with_index_checks():
    env = dict(os.environ, MGBRAIN_LIB="checked")
    lib = os.path.join(ROOT, "mgbrain_b200", "lib", "libmgbrain_b200_checked.so")
    assert os.path.exists(lib), "build the checked library (python -m mgbrain_b200.build --checked)"
    r = subprocess.run([sys.executable, "-c", PROBE], env=env, cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0 and "checked build ok" in r.stdout, r.stderr[-3000:]
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider"] + SUITES,
                       env=env, cwd=ROOT, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-4000:]
