"""NetGen's fixed-probability rule drawn on several host threads (each from
the generator jumped ahead to its stretch of candidate pairs) gives the
network of one thread synapse for synapse; MGBrain::Mt19937 gives
std::mt19937's outputs, its 10,000th is the C++ standard's check value, and
every jump equals the sequential advance (tests/cpp/netgen_threads.cpp)."""
import os
import subprocess

import pytest

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..")

# five fixed-probability projections of different sizes and densities, the
# last so sparse that it may take fewer pairs than its target (the rest of its
# list stays pair (0, 0), as in the reference)
SPEC = """timestep 0.0001
pop 900 LIFB 0
pop 300 LIFB 0
pop 200 POISSON 1
conn 2 0 0.002 0.004 0.001 0.003 0.05 STATIC
conn 0 0 0.0008 0.0008 0.001 0.003 0.1 STATIC
conn 0 1 0.0008 0.0012 0.001 0.002 0.003 STATIC
conn 1 0 -0.004 -0.004 0.001 0.002 0.2 STATIC
conn 1 1 -0.004 -0.002 0.001 0.001 0.0001 STATIC
rate 2 0.01
"""


@pytest.fixture(scope="module")
def prog(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "netgen_threads")
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(ROOT, "tests", "cpp", "netgen_threads.cpp"),
                    "-L" + os.path.join(ROOT, "mgbrain_b200", "lib"), "-lmgbrain_b200",
                    "-Wl,-rpath," + os.path.join(ROOT, "mgbrain_b200", "lib")], check=True)
    return exe


@pytest.mark.parametrize("threads", [2, 3, 7, 32])
def test_threads_give_the_same_network(prog, tmp_path, threads):
    spec = tmp_path / "n.spec"
    spec.write_text(SPEC)
    r = subprocess.run([prog, str(spec), str(threads), "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok ") and int(r.stdout.split()[1]) > 100000
