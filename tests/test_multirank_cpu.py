"""World-size-2 gloo run of the bench's multi-rank host logic on CPU: the
process group comes up on 127.0.0.1, max/sum over ranks are what the timing
takes, and the independent sweep instances are dealt so that every one runs
on exactly one rank."""
import json
import os
import socket
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "multirank_worker.py"), "7"], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=240)
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for o in outs:
        assert o["ws"] == 2
        assert o["max"] == 2.0 and o["sum"] == 30.0
        units = sorted(u for share in o["units"] for u in share)
        assert units == list(range(7))
        assert set(o["units"][0]).isdisjoint(o["units"][1])
