"""One rank of the multi-process partition tests.  Prints one JSON line.

`gpu`: this rank's partition of a device-generated Brunel network runs on
cuda:0 and exchanges spike ids with the other ranks through gloo; rank 0
then gathers every rank's raster and state and compares them with the whole
network run on its own.

`fail`: no GPU.  As `fake`, but rank 1 raises inside its fifth window and
its process ends without joining the next exchange; the other ranks must
learn of it from their collective (an error, within the process group's
short timeout) instead of waiting for good.

`fake [world steps]`: no GPU.  A stand-in partition with the handle's
exchange interface fires a fixed pseudo-random pattern and keeps the spike
history the way the library does (own spikes first, then the imported ones);
every rank reports the history it ends with, which must hold every rank's
spikes of every step.
"""
import json
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), ".."))
import bench  # noqa: E402


def pattern(n_src, steps, seed=3):
    """Spikes of the fake network: step -> ids (whole-network ids)."""
    rng = np.random.default_rng(seed)
    return [np.flatnonzero(rng.random(n_src) < 0.05).astype(np.int32) for _ in range(steps)]


class FakePartition:
    """Neurons [first, first + n) of n_src with the partition handle's
    run / part_export / part_import contract, on host tensors."""

    def __init__(self, n_src, first, n, min_delay, spikes):
        self.n_src, self.first, self.n, self.min_delay = n_src, first, n, min_delay
        self.spikes = spikes
        self.hist = []          # step -> list of ids
        self.pending = 0

    def info(self):
        return {"min_delay": self.min_delay}

    fail_at = None              # window at which run() raises (failure test)

    def run(self, k):
        assert self.pending + k <= self.min_delay - 1, "ran past the exchange window"
        if self.fail_at is not None and len(self.hist) // max(1, self.min_delay - 1) >= self.fail_at:
            raise RuntimeError("injected rank failure")
        for _ in range(k):
            s = len(self.hist)
            own = self.spikes[s]
            own = own[(own >= self.first) & (own < self.first + self.n)]
            self.hist.append(list(own[::-1]))  # not sorted, as the device's atomics leave it
        self.pending += k

    def part_export(self, k, buf):
        assert k == self.pending
        counts = np.array([len(h) for h in self.hist[-k:]], np.int32)
        flat = np.concatenate([np.array(h, np.int32) for h in self.hist[-k:]]) if counts.sum() else []
        buf[:len(flat)] = torch.from_numpy(np.asarray(flat, np.int32))
        return counts, int(counts.sum())

    def part_import(self, k, self_rank, C, recv, stride):
        assert k == self.pending
        ids = recv.numpy()
        for r in range(C.shape[0]):
            if r == self_rank:
                continue
            off = r * stride
            for j in range(k):
                c = int(C[r, j])
                self.hist[len(self.hist) - k + j] += list(ids[off:off + c])
                off += c
        self.pending = 0


def fake(world_steps):
    import torch.distributed as dist
    from mgbrain_b200.partition import DistributedPartition, split
    ws, rank, _ = bench.dist_init()
    n_src, min_delay = 1000, 4
    spikes = pattern(n_src, world_steps)
    first, n = split(n_src, ws)[rank]
    sim = FakePartition(n_src, first, n, min_delay, spikes)
    part = DistributedPartition(sim, device="cpu")
    part.run(world_steps // 2)
    part.run(world_steps - world_steps // 2)
    ok = all(sorted(int(x) for x in sim.hist[s]) == [int(x) for x in spikes[s]] for s in range(world_steps))
    out = {"rank": rank, "window": part.window, "equal": bool(ok), "steps": len(sim.hist)}
    dist.destroy_process_group()
    print(json.dumps(out), flush=True)


def fail():
    import datetime
    import time

    import torch.distributed as dist
    from mgbrain_b200.partition import DistributedPartition, split
    ws, rank = int(os.environ["WORLD_SIZE"]), int(os.environ["RANK"])
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=15))
    n_src, min_delay = 1000, 4
    spikes = pattern(n_src, 60)
    first, n = split(n_src, ws)[rank]
    sim = FakePartition(n_src, first, n, min_delay, spikes)
    if rank == 1:
        sim.fail_at = 5
    part = DistributedPartition(sim, device="cpu")
    t0 = time.time()
    try:
        part.run(60)
        out = {"rank": rank, "detected": False}
    except Exception as e:  # noqa: BLE001 - any collective error is the detection
        out = {"rank": rank, "detected": True, "error": type(e).__name__, "seconds": time.time() - t0,
               "steps": len(sim.hist)}
    print(json.dumps(out), flush=True)
    os._exit(3 if rank == 1 else 0)   # no destroy: a failed group cannot be torn down collectively


def gpu():
    import torch.distributed as dist
    import mgbrain_b200 as mgb
    from mgbrain_b200.partition import DistributedPartition, split
    ws, rank, _ = bench.dist_init()
    torch.cuda.set_device(0)
    w = bench.workload(scale=0.02, nu=0.02)
    mk = dict(rate=w["rate"], v_init=w["v0"], conn_seed=21, seed=22)
    first, n = split(w["n"], ws)[rank]
    sim = mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], part=(first, n), **mk)
    sim.set_persistent(0)   # graphs: no kernel here spins on a barrier while the ranks share the GPU
    part = DistributedPartition(sim, device="cuda:0")
    steps = 2000
    part.run(steps)
    sim.sync()
    mine = {"raster": sim.read_raster(), "state": sim.state()}
    everyone = [None] * ws
    dist.all_gather_object(everyone, mine)
    out = {"rank": rank, "window": part.window}
    if rank == 0:
        from mgbrain_b200.partition import merge_rasters
        whole = mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], **mk)
        whole.set_persistent(0)
        whole.run(steps)
        wf, wc, wi = whole.read_raster()
        pf, pc, pi = merge_rasters([e["raster"] for e in everyone])
        ws_ = whole.state()
        V = np.concatenate([e["state"]["V"] for e in everyone])
        fc = np.concatenate([e["state"]["fire_cnt"] for e in everyone])
        out["equal"] = bool(pf == wf and np.array_equal(pc, wc) and np.array_equal(pi, wi) and
                            np.array_equal(V.view(np.int32), ws_["V"].view(np.int32)) and
                            np.array_equal(fc, ws_["fire_cnt"]))
        out["spikes"] = int(wc.sum())
        whole.close()
    dist.barrier()
    sim.close()
    dist.destroy_process_group()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    if sys.argv[1] == "fake":
        fake(int(sys.argv[2]) if len(sys.argv) > 2 else 50)
    elif sys.argv[1] == "fail":
        fail()
    else:
        gpu()
