"""Partitioned simulation: one network split into neuron ranges, one handle per
range, with a spike-id exchange every window of steps.

This is the B200 form of MGBrain's multi-GPU run, MGSimulator(net, part,
npart) with npart > 1 (src/simulator/mgsim/adj/mgsim.cpp:337-363, 794-848).
The reference's partitions push cross-partition synaptic events into
per-pair buffers and copy them between GPUs every min_delay/2 steps
(mgcore.cu:470-646).  Here each partition holds the synapses that target its
own neurons, with every source of the network, so only spike ids cross
between partitions: after at most min_delay - 1 steps each partition exports
the ids its neurons fired, the ids are gathered across partitions, and each
partition appends the others' ids to its spike history
(mgc_part_export / mgc_part_import).  A delivery of step x reads spikes of
steps <= x - min_delay only, so every spike is in every history before any
partition delivers it, and the union of the partitions' runs equals the
whole network's run.

Two drivers:
- PartitionGroup: several partition handles in one process (one device or
  several), the gather done by device copies;
- DistributedPartition: one handle per rank of a torch.distributed group.

Two exchanges, by `cap_per_step`:
- None (exact): an all-gather of the counts, then of the ids padded to the
  largest rank's total; the host learns the sizes in between, so each window
  waits for the host (NCCL on device buffers, or gloo through host memory);
- a number: fixed-capacity buffers of cap_per_step ids per step of the
  window, exported, gathered (NCCL all-gather, or device copies) and imported
  on the handles' streams without a host synchronisation.  A window with
  more spikes than the capacity is refused on every rank and the next sync
  raises (mgc_part_export_dev / mgc_part_import_dev).
"""
from __future__ import annotations

import numpy as np
import torch


def window_of(min_delay):
    """Steps per exchange: a delivery of step x reads spikes of steps <= x - min_delay."""
    if min_delay < 2:
        raise ValueError(f"partitions need min_delay >= 2 (got {min_delay})")
    return int(min_delay) - 1


def split(n, parts):
    """Neuron ranges (first, count) of `parts` contiguous partitions of n neurons."""
    bounds = [n * p // parts for p in range(parts + 1)]
    return [(bounds[p], bounds[p + 1] - bounds[p]) for p in range(parts)]


def merge_rasters(rasters):
    """One raster (first step, counts, ids ascending per step) from the
    partitions' rasters of the same steps."""
    first = rasters[0][0]
    steps = len(rasters[0][1])
    per = []
    for f, counts, ids in rasters:
        if f != first or len(counts) != steps:
            raise ValueError("partition rasters cover different steps")
        per.append(np.split(ids, np.cumsum(counts)[:-1]) if steps else [])
    counts = np.zeros(steps, np.int64)
    out = []
    for s in range(steps):
        ids = np.sort(np.concatenate([p[s] for p in per]))
        counts[s] = len(ids)
        out.append(ids)
    return first, counts, (np.concatenate(out).astype(np.int32) if out else np.zeros(0, np.int32))


class PartitionGroup:
    """Partition handles of one network driven together in one process."""

    def __init__(self, sims, devices=None, cap_per_step=None):
        self.sims = list(sims)
        self.devices = [torch.device("cuda", d) for d in (devices or [0] * len(self.sims))]
        self.window = min(window_of(s.info()["min_delay"]) for s in self.sims)
        R = len(self.sims)
        self.cap = None if cap_per_step is None else self.window * int(cap_per_step)
        if self.cap is None:
            # export buffers: a partition emits at most its neurons per step
            self.bufs = [torch.empty(max(1, self.window * s.n), dtype=torch.int32, device=d)
                         for s, d in zip(self.sims, self.devices)]
        else:
            blk = self.window + self.cap
            self.ebufs = [torch.empty(blk, dtype=torch.int32, device=d) for d in self.devices]
            self.gbufs = [torch.empty(R * blk, dtype=torch.int32, device=d) for d in self.devices] if R > 1 else None
            self.streams = [torch.cuda.ExternalStream(s.stream, device=d) for s, d in zip(self.sims, self.devices)]
            self.done = []   # events: the previous window's gathers, before an export buffer is reused

    def run(self, steps):
        left = int(steps)
        while left > 0:
            k = min(self.window, left)
            for s in self.sims:
                s.run(k)
            if self.cap is None:
                self._exchange(k)
            else:
                self._exchange_dev(k)
            left -= k

    def sync(self):
        for s in self.sims:
            s.sync()

    def _exchange(self, k):
        R = len(self.sims)
        counts, totals = [], []
        for s, b in zip(self.sims, self.bufs):
            c, t = s.part_export(k, b)
            counts.append(c)
            totals.append(t)
        C = np.stack(counts)
        stride = max(1, max(totals))
        for r, (s, d) in enumerate(zip(self.sims, self.devices)):
            ids = torch.zeros(R * stride, dtype=torch.int32, device=d)
            for q in range(R):
                if q != r and totals[q]:
                    ids[q * stride:q * stride + totals[q]].copy_(self.bufs[q][:totals[q]])
            torch.cuda.synchronize(d)
            s.part_import(k, r, C, ids, stride)

    def _exchange_dev(self, k):
        R = len(self.sims)
        if R == 1:
            self.sims[0].part_import_dev(k, 0, 1, None, self.cap)   # nothing to gather: closes the window
            return
        blk = k + self.cap
        exported = []
        for q, s in enumerate(self.sims):
            for ev in self.done:             # every gather of the last window read this buffer
                self.streams[q].wait_event(ev)
            s.part_export_dev(k, self.ebufs[q], self.cap)
            ev = torch.cuda.Event()
            ev.record(self.streams[q])
            exported.append(ev)
        self.done = []
        for r, s in enumerate(self.sims):
            st = self.streams[r]
            with torch.cuda.stream(st):
                for q in range(R):   # every block, its own too (its counts are checked against cap)
                    st.wait_event(exported[q])
                    self.gbufs[r][q * blk:(q + 1) * blk].copy_(self.ebufs[q][:blk], non_blocking=True)
            s.part_import_dev(k, r, R, self.gbufs[r], self.cap)
            ev = torch.cuda.Event()
            ev.record(st)
            self.done.append(ev)

    def raster(self):
        return merge_rasters([s.read_raster() for s in self.sims])

    def state(self):
        st = [s.state() for s in self.sims]
        return {k: np.concatenate([x[k] for x in st]) for k in st[0]}


class DistributedPartition:
    """This rank's partition handle; run() is collective over the group.
    `device`: where the handle's exchange buffers live (its CUDA device)."""

    def __init__(self, sim, device=None, group=None, cap_per_step=None):
        import torch.distributed as dist
        self.dist = dist
        self.sim = sim
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.nccl = dist.get_backend(group) == "nccl"
        self.device = torch.device("cuda", 0) if device is None else torch.device(device)
        self.comm_device = self.device if self.nccl else torch.device("cpu")
        w = torch.tensor([window_of(sim.info()["min_delay"])], dtype=torch.int64, device=self.comm_device)
        dist.all_reduce(w, op=dist.ReduceOp.MIN, group=group)
        self.window = int(w.item())
        if cap_per_step is not None and not self.nccl:
            raise ValueError("the device exchange gathers with NCCL (gloo groups use the exact exchange)")
        self.cap = None if cap_per_step is None else self.window * int(cap_per_step)
        if self.cap is None:
            self.buf = torch.empty(max(1, self.window * sim.n), dtype=torch.int32, device=self.device)
        else:
            blk = self.window + self.cap
            self.ebuf = torch.empty(blk, dtype=torch.int32, device=self.device)
            self.gbuf = torch.empty(self.world * blk, dtype=torch.int32, device=self.device)
            self.stream = torch.cuda.ExternalStream(sim.stream, device=self.device)

    def run(self, steps):
        left = int(steps)
        while left > 0:
            k = min(self.window, left)
            self.sim.run(k)
            if self.cap is None:
                self.exchange(k)
            else:
                self.exchange_dev(k)
            left -= k

    def exchange_dev(self, k):
        """Export, all-gather and import on the handle's stream; no host wait."""
        blk = k + self.cap
        self.sim.part_export_dev(k, self.ebuf, self.cap)
        with torch.cuda.stream(self.stream):
            self.dist.all_gather_into_tensor(self.gbuf[:self.world * blk], self.ebuf[:blk], group=self.group)
        self.sim.part_import_dev(k, self.rank, self.world, self.gbuf, self.cap)

    def exchange(self, k):
        dist, R = self.dist, self.world
        counts, total = self.sim.part_export(k, self.buf)
        c = torch.from_numpy(counts.astype(np.int32)).to(self.comm_device)
        gathered = [torch.empty_like(c) for _ in range(R)]
        dist.all_gather(gathered, c, group=self.group)
        C = torch.stack(gathered).cpu().numpy()
        stride = max(1, int(C.sum(axis=1).max()))
        send = torch.zeros(stride, dtype=torch.int32, device=self.device)
        if total:
            send[:total].copy_(self.buf[:total])
        if self.nccl:
            recv = torch.empty(R * stride, dtype=torch.int32, device=self.device)
            dist.all_gather_into_tensor(recv, send, group=self.group)
        else:
            parts = [torch.empty(stride, dtype=torch.int32) for _ in range(R)]
            dist.all_gather(parts, send.cpu(), group=self.group)
            recv = torch.cat(parts).to(self.device)
        if self.device.type == "cuda":
            torch.cuda.synchronize(self.device)  # the import runs on the handle's own stream
        self.sim.part_import(k, self.rank, C, recv, stride)
