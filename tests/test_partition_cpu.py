"""Host side of the partitioned run, on CPU: gloo ranks with stand-in
partitions exchange spike ids through the driver's two all-gathers (counts,
then ids padded to the largest rank's total) and every rank ends with every
rank's spikes of every step; the range split and the raster merge."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from mgbrain_b200.partition import merge_rasters, split, window_of

HERE = os.path.dirname(os.path.abspath(__file__))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_share_every_spike(world):
    port = free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "partition_worker.py"), "fake", "50"],
                                      env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=240)
        assert p.returncode == 0, e[-3000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for o in outs:
        assert o["window"] == 3 and o["steps"] == 50
        assert o["equal"], o


def test_failed_rank_is_detected_not_waited_for():
    """Rank 1 fails inside a window and leaves; rank 0's next exchange ends
    with an error (peer gone, or the group's 15 s timeout) instead of
    hanging."""
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "partition_worker.py"), "fail"],
                                      env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=240)
        outs.append((p.returncode, json.loads(o.strip().splitlines()[-1])))
    (rc0, o0), (rc1, o1) = outs
    assert rc1 == 3 and o1["detected"] and o1["error"] == "RuntimeError"
    assert rc0 == 0 and o0["detected"], o0
    assert o0["seconds"] < 120
    assert o0["steps"] >= 15        # the windows before the failure completed


def test_split_and_window():
    assert split(10, 3) == [(0, 3), (3, 3), (6, 4)]
    assert sum(c for _, c in split(1_100_000, 8)) == 1_100_000
    assert window_of(10) == 9
    with pytest.raises(ValueError):
        window_of(1)


def test_merge_rasters():
    a = (5, np.array([2, 0, 1]), np.array([1, 3, 2], np.int32))
    b = (5, np.array([1, 1, 0]), np.array([0, 9], np.int32))
    first, counts, ids = merge_rasters([a, b])
    assert first == 5
    assert counts.tolist() == [3, 1, 1]
    assert ids.tolist() == [0, 1, 3, 9, 2]
    with pytest.raises(ValueError):
        merge_rasters([a, (6, b[1], b[2])])
