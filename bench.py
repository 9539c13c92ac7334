"""Throughput of the mgbrain_b200 simulation core on the large Brunel network.

Workload (one bench step = 10,000 timesteps = 1 s simulated at dt = 0.1 ms):
  1,000,000 LIFB neurons (800k exc, 200k inh; V_th 20 mV, V_reset 10 mV,
  t_ref 2 ms, leak dt/tau_m = 0.005, V0 ~ U[0, 20 mV)) plus 100,000 POISSON
  inputs at 20 Hz (0.002 per step); fixed in-degree 800 exc + 200 inh + 100
  external per neuron (1.1e9 synapses, 8 B each on the device), J = 0.1 mV,
  g = 5, delays uniform in 10..50 steps.  Synthetic, seeded, generated on
  the device.  A driven variant (inputs at 200 Hz) is measured beside it
  because the network as specified is quiescent apart from its inputs, and
  a dense network firing in volleys (pull_variant) for the pull steps.

Metric: synaptic events delivered per second of wall time (value), with
simulated seconds per wall second and the HBM roofline of the dominant
kernel.  `value` is device time over K bench steps (CUDA events on the
core's stream, inputs resident); `e2e` goes through the C ABI with the
POISSON rates copied from pinned host memory and the raster read back every
bench step.  The CSR (8.8 GB) is larger than L2, so no flush is needed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
With N > 1 the network is split into one contiguous neuron range per rank
(strong scaling; spike ids all-gathered through NCCL every min_delay - 1
steps); --workload replicas runs N independent instances instead (weak
scaling).  value is the total over ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "synaptic events/s & sim-s per wall-s, 1M-neuron Brunel; % of HBM roofline"
DT = 1e-4
CHUNK = 10_000            # timesteps per bench step (1 s simulated)
NE, NI, NP = 800_000, 200_000, 100_000
KE, KI, KX = 800, 200, 100
J, G = 1e-4, 5.0
DMIN, DMAX = 10, 50
NU_STEP = 0.002           # 20 Hz at 0.1 ms
NU_DRIVEN = 0.02          # 200 Hz


def workload(scale=1.0, nu=NU_STEP, seed=1):
    ne, ni, nx = int(NE * scale), int(NI * scale), int(NP * scale)
    n = ne + ni + nx
    pops = [(0, ne, 5), (ne, ni, 5), (ne + ni, nx, 2)]   # LIFB, LIFB, POISSON
    projs = []
    for tgt in (0, 1):
        projs += [(0, tgt, KE, J, DMIN, DMAX), (1, tgt, KI, -G * J, DMIN, DMAX),
                  (2, tgt, KX, J, DMIN, DMAX)]
    lif = np.zeros(30, np.float32)
    lif[0], lif[3], lif[4], lif[8] = DT, 0.01, 0.02, 0.002
    rate = np.zeros(n, np.float32)
    rate[ne + ni:] = nu
    v0 = np.random.default_rng(seed).uniform(0.0, 0.02, n).astype(np.float32)
    return dict(n=n, n_lif=ne + ni, pops=pops, projs=projs, lif=lif, rate=rate, v0=v0)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(backend="gloo"):
    """Process group of a multi-rank run: gloo for the host-side timing
    reductions, NCCL where spike ids cross GPUs (partitioned workload)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(x, op):
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"   # NCCL reduces device tensors only
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def allmax(ws, x):
    if ws == 1:
        return x
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX)


def allsum(ws, x):
    if ws == 1:
        return x
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM)


# --------------------------------------------------------------------------
# CPU legs (the oracle restatement of the reference path; no GPU)
# --------------------------------------------------------------------------
def oracle_sim(w, threads):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import mgb_testlib as T
    L = T.oracle()
    P = np.array(w["pops"], np.int32)
    R = w["projs"]
    arr = lambda x, dt: np.ascontiguousarray(x, dt)  # noqa: E731
    keep = [arr(P[:, 0], np.int32), arr(P[:, 1], np.int32), arr(P[:, 2], np.int32),
            arr([r[0] for r in R], np.int32), arr([r[1] for r in R], np.int32),
            arr([r[2] for r in R], np.int32), arr([r[3] for r in R], np.float32),
            arr([r[4] for r in R], np.int32), arr([r[5] for r in R], np.int32)]
    h = L.mgbo_create_fixed_indegree(*[T._p(k) for k in keep[:3]], len(P),
                                     *[T._p(k) for k in keep[3:]], len(R), T._p(w["rate"]),
                                     T._p(w["v0"]), T._p(w["lif"]), 1, 1, threads, 0, 0)
    if not h:
        raise MemoryError("oracle could not allocate the network")
    return L, h, T


def oracle_rate(L, h, steps):
    """events/s of the oracle over `steps` steps (wall clock)."""
    import ctypes as C
    e0 = L.mgbo_events(h)
    nid = C.c_int64()
    t0 = time.perf_counter()
    L.mgbo_run(h, steps, None, None, 0, C.byref(nid))
    dt = time.perf_counter() - t0
    return (L.mgbo_events(h) - e0) / dt, dt


def cpu_baseline(w, sample_steps):
    """The oracle on one thread over the first `sample_steps` steps of the
    network: its events/s, and its raster and V after those steps (kept for
    the parity check of the GPU run)."""
    import ctypes as C
    L, h, T = oracle_sim(w, os.cpu_count() or 1)
    cap = 1 << 24
    counts = np.zeros(sample_steps, np.int64)
    ids = np.zeros(cap, np.int32)
    v = np.zeros(w["n"], np.float32)
    fc = np.zeros(w["n"], np.int32)
    try:
        L.mgbo_set_threads(h, 1)
        e0 = L.mgbo_events(h)
        nid = C.c_int64()
        t0 = time.perf_counter()
        rc = L.mgbo_run(h, sample_steps, T._p(counts), T._p(ids), cap, C.byref(nid))
        dt = time.perf_counter() - t0
        ev = L.mgbo_events(h) - e0
        L.mgbo_read_state_f32(h, T._p(v), None)
        L.mgbo_read_state(h, None, None, None, None, None, T._p(fc), None)
    finally:
        L.mgbo_destroy(h)
    base = {"value": ev / dt, "unit": "events/s", "cores": 1, "kind": "port",
            "sample": f"oracle (C restatement of the reference kernels), 1 thread, first "
                      f"{sample_steps} timesteps of the same network ({dt:.1f} s)"}
    ref = dict(counts=counts, ids=ids[:nid.value] if rc == 0 else None, v=v, fire_cnt=fc)
    return base, ref


def parity_check(w, local, ref, steps, group_mode, window):
    """The GPU's first `steps` steps of the bench network, run from the same
    seeds in the step-group form the timed run used, against the oracle's."""
    sim = make_sim(w, local, seed=1, record=True)
    try:
        sim.set_persistent(group_mode)
        if group_mode == 3 and window:
            sim.set_window(window)
        sim.run(steps)
        sim.sync()
        _, counts, ids = sim.read_raster(max_steps=steps + 1, max_ids=1 << 24)
        st = sim.state()
    finally:
        sim.close()
    v_o = ref["v"]
    raster_equal = ref["ids"] is not None and np.array_equal(counts, ref["counts"]) and np.array_equal(ids, ref["ids"])
    rel = np.abs(st["V"].astype(np.float64) - v_o) / np.maximum(np.abs(v_o.astype(np.float64)), 1e-30)
    return {"steps": steps, "spikes": int(counts.sum()), "raster_equal": bool(raster_equal),
            "v_bit_equal": bool(np.array_equal(st["V"].view(np.int32), v_o.view(np.int32))),
            "v_max_rel": float(rel.max()), "fire_cnt_equal": bool(np.array_equal(st["fire_cnt"], ref["fire_cnt"])),
            "step_group": {"mode": group_mode, "window": window},
            "against": "oracle fp32 (C restatement of the reference kernels), same network and seeds"}


def run_reference(a, ws, rank):
    if rank != 0:
        return
    w = workload()
    cores = os.cpu_count() or 1
    L, h, T = oracle_sim(w, cores)
    sample = a.ref_sample
    try:
        for _ in range(a.warmup):
            oracle_rate(L, h, sample)
        vals, times = [], []
        for _ in range(a.steps):
            v, dt = oracle_rate(L, h, sample)
            vals.append(v)
            times.append(dt)
    finally:
        L.mgbo_destroy(h)
    value = float(np.sum([v * t for v, t in zip(vals, times)]) / np.sum(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "events/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1000 * float(np.mean(times)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "large Brunel (1M LIFB + 100k POISSON @20 Hz, fixed in-degree "
                               "800/200/100, delays 10-50 steps, dt 0.1 ms)",
                   "bench_step": f"{sample} timesteps", "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": value, "unit": "events/s", "cores": cores, "kind": "port",
                         "sample": f"oracle (C restatement of the reference kernels; the reference "
                                   f"has no CPU simulator), {cores} OpenMP threads, {sample} "
                                   f"timesteps per step"},
        "e2e": {"value": value, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "sim_s_per_wall_s": sample * DT / float(np.mean(times)),
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def make_sim(w, device, seed, record=True):
    import mgbrain_b200 as mgb
    return mgb.Simulator.fixed_indegree(
        w["pops"], w["projs"], w["lif"], rate=w["rate"], v_init=w["v0"], conn_seed=1,
        seed=seed, device=device, raster_steps=CHUNK * 4, raster_ids=-1 if not record else 0)


def timed_device(sim, steps_per, k, ws):
    """Device time of k bench steps: CUDA events on the core's stream."""
    import torch
    stream = torch.cuda.ExternalStream(sim.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier(ws)
    ev0 = sim.info()["events"]
    l0 = sim.kernel_launches
    e0.record(stream)
    for _ in range(k):
        sim.run(steps_per)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(ws)
    ms = e0.elapsed_time(e1)
    return ms, sim.info()["events"] - ev0, sim.kernel_launches - l0


def run_ours(a, ws, rank, local):
    import torch

    import mgbrain_b200 as mgb
    torch.cuda.set_device(local)
    hbm, peak_kind = peaks()
    # the second bound of event delivery: one scattered fp32 reduction per event
    red_ceiling, read_ceiling = mgb.capi.measure_scatter(local)
    w = workload(a.scale)
    t0 = time.perf_counter()
    sim = make_sim(w, local, seed=1 + rank, record=False)
    build_s = time.perf_counter() - t0
    info = sim.info()
    if a.no_autotune:
        tune = None
        sim.set_persistent(a.group_mode)
    else:
        tune = sim.autotune(steps_per_trial=640)   # launch shape by measurement
    for _ in range(a.warmup):
        sim.run(CHUNK)
    sim.sync()
    with ClockSampler(local) as clk:
        ms, events, launches = timed_device(sim, CHUNK, a.steps, ws)
    ms_max = allmax(ws, ms)
    ev_all = allsum(ws, events)
    value = ev_all / (ms_max / 1e3)
    sim_s_wall = a.steps * CHUNK * DT / (ms_max / 1e3)
    spikes_per_step = None

    # per-kernel timing with CUDA events (no graphs) for the roofline
    prof_steps = 2000
    ev_p0 = sim.info()["events"]
    kms = sim.profile(prof_steps)
    ev_p = sim.info()["events"] - ev_p0
    n_lif = w["n_lif"]
    neuron_bytes = 24.0 * n_lif            # per launch (spike-id bytes are negligible here)
    push_bytes = 8.0 * ev_p / prof_steps
    kern = {
        "neuron_update": {"avg_us": 1e3 * kms[0] / prof_steps, "bytes": neuron_bytes},
        "event_push": {"avg_us": 1e3 * kms[1] / prof_steps, "bytes": push_bytes},
    }
    for k_, v in kern.items():
        v["achieved_gbs"] = v["bytes"] / (v["avg_us"] * 1e-6) / 1e9 if v["avg_us"] > 0 else 0.0
        v["frac"] = v["achieved_gbs"] / hbm
        v["share"] = kms[0 if k_ == "neuron_update" else 1] / max(1e-9, sum(kms))
    steps_timed = a.steps * CHUNK
    group_mode = sim.info()["persistent"]
    sim_window = sim.info()["window"] if group_mode == 3 else None
    if 0 < launches <= steps_timed and steps_timed % launches == 0:
        # the fused method: one kernel per step (k_fused) or one per step group
        # (k_steps / k_pipe / k_window); each launch covers steps_timed /
        # launches steps and its average duration is the timed region over its launches
        per_launch = steps_timed // launches
        dom = {0: "k_fused", 1: "k_steps", 2: "k_pipe", 3: "k_window"}[group_mode]
        dur_us = 1e3 * ms / launches
        dbytes = per_launch * (neuron_bytes + 8.0 * events / steps_timed)
        achieved = dbytes / (dur_us * 1e-6) / 1e9
    else:
        dom = max(kern, key=lambda k_: kern[k_]["avg_us"])
        dur_us, dbytes, achieved = kern[dom]["avg_us"], kern[dom]["bytes"], kern[dom]["achieved_gbs"]
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            t = json.load(open(tpath)).get(dom)
            # ncu DRAM bytes per step, scaled to this workload's size and to
            # the steps one launch covers
            if t is not None:
                per = steps_timed // launches if launches else 1
                traffic = t["bytes_per_step"] * a.scale * per
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                "bytes_per_launch": dbytes, "avg_launch_us": dur_us,
                "steps_per_launch": steps_timed // launches if launches else None}

    # end to end through the C ABI: rates H2D from pinned memory, run, raster D2H
    sim.close()
    sim = make_sim(w, local, seed=1 + rank, record=True)
    if not a.no_autotune:
        sim.autotune(steps_per_trial=640)
    pinned = torch.empty(w["n"], dtype=torch.float32, pin_memory=True)
    pinned.numpy()[:] = w["rate"]
    import ctypes as C
    L = mgb.lib()
    for _ in range(1):
        sim.run(CHUNK)
        sim.read_raster(max_steps=CHUNK * 4, max_ids=w["n"] * 16)  # also drops the autotuner's steps
    torch.cuda.synchronize()
    barrier(ws)
    h2d = d2h = 0
    ev0 = sim.info()["events"]
    t0 = time.perf_counter()
    # each bench step: its rates from pinned memory, its steps, and its raster
    # staged on the device; the raster of the step before is collected (copied
    # out and sorted) while this one runs
    for i in range(a.e2e_steps):
        mgb.capi.check(L.mgc_set_rates(sim._h, C.c_void_p(pinned.data_ptr()), w["n"]))
        h2d += 4 * w["n"]
        sim.run(CHUNK)
        sim.stage_raster()
        if i >= 1:
            _, counts, ids = sim.collect_raster(max_steps=CHUNK, max_ids=w["n"] * 8)
            d2h += 4 * len(counts) + 4 * len(ids)
    _, counts, ids = sim.collect_raster(max_steps=CHUNK, max_ids=w["n"] * 8)
    d2h += 4 * len(counts) + 4 * len(ids)
    sim.sync()
    e2e_s = allmax(ws, time.perf_counter() - t0)
    e2e_ev = allsum(ws, sim.info()["events"] - ev0)
    e2e = {"value": e2e_ev / e2e_s, "unit": "events/s",
           "h2d_bytes_per_step": int(h2d / a.e2e_steps), "d2h_bytes_per_step": int(d2h / a.e2e_steps),
           "sim_s_per_wall_s": a.e2e_steps * CHUNK * DT / e2e_s}
    sim.close()

    # driven variant (inputs at 200 Hz): the same network with activity
    driven = None
    if not a.no_driven:
        wd = workload(a.scale, nu=NU_DRIVEN)
        simd = make_sim(wd, local, seed=1 + rank, record=False)
        simd.autotune(steps_per_trial=640)
        simd.run(CHUNK // 2)
        simd.sync()
        dms, dev, _ = timed_device(simd, CHUNK, 1, ws)
        dms = allmax(ws, dms)
        dev = allsum(ws, dev)
        kd0 = simd.info()["events"]
        kmd = simd.profile(500)
        evd = simd.info()["events"] - kd0
        push_us = 1e3 * kmd[1] / 500
        driven = {"inputs_hz": 200, "events_per_s": dev / (dms / 1e3),
                  "sim_s_per_wall_s": CHUNK * DT / (dms / 1e3),
                  "event_push": {"avg_us": push_us, "bytes": 8.0 * evd / 500,
                                 "achieved_gbs": 8.0 * evd / 500 / (push_us * 1e-6) / 1e9,
                                 "frac": 8.0 * evd / 500 / (push_us * 1e-6) / 1e9 / hbm},
                  "neuron_update_avg_us": 1e3 * kmd[0] / 500,
                  "whole_step_frac_of_reduction_ceiling": dev / (dms / 1e3) / ws / red_ceiling}
        simd.close()
        # the same driven network with its inputs summed in 64-bit fixed
        # point (what a network with unequal weights of one sign runs):
        # the cost of order-independent sums
        simf = make_sim(wd, local, seed=1 + rank, record=False)
        simf.set_accumulation(mgb.ACC_FIXED)
        simf.autotune(steps_per_trial=640)
        simf.run(CHUNK // 2)
        simf.sync()
        fms, fev, _ = timed_device(simf, CHUNK, 1, ws)
        fms, fev = allmax(ws, fms), allsum(ws, fev)
        driven["fixed_point"] = {"events_per_s": fev / (fms / 1e3), "sim_s_per_wall_s": CHUNK * DT / (fms / 1e3),
                                 "step_group": simf.info()["persistent"], "fx_shift": simf.info()["fx_shift"]}
        simf.close()

    pull = None
    if rank == 0 and not a.no_pull:
        try:
            pull = pull_variant(local)
        except Exception as e:  # a side leg: its failure does not void the line
            pull = {"unavailable": f"{type(e).__name__}: {e}"}

    cpu = parity = None
    if rank == 0 and not a.no_cpu:
        try:
            cpu, ref = cpu_baseline(w, a.cpu_sample)
        except Exception as e:  # the host may lack the memory for the full network
            cpu, ref = {"value": None, "unit": "events/s", "cores": 1, "kind": "port",
                        "sample": f"not run: {e}"}, None
        if ref is not None:
            parity = parity_check(w, local, ref, a.cpu_sample, group_mode, sim_window)
    reference_gpu = None
    if rank == 0 and not a.no_refgpu:
        try:
            reference_gpu = refgpu_compare(a, local)
        except Exception as e:  # a baseline leg: its failure does not void the line
            reference_gpu = {"workload": "refgpu", "unavailable": f"{type(e).__name__}: {e}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": ws,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_max / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded, generated on the device)",
            "config": {"workload": "large Brunel: 1M LIFB (800k/200k) + 100k POISSON @20 Hz, fixed "
                                   "in-degree 800/200/100, J 0.1 mV, g 5, delays U{10..50} steps, "
                                   "dt 0.1 ms",
                       "scale": a.scale, "synapses": info["n_synapses"], "bench_step": "1 s simulated "
                       "(10,000 timesteps)", "l2": "inputs larger than L2 (8.8 GB CSR)",
                       "parallelism": "replicas" if ws > 1 else "single GPU",
                       "step_group": {"mode": group_mode, "kernel": dom, "window": sim_window}},
            "sim_s_per_wall_s": sim_s_wall,
            "events_per_step": ev_all / (a.steps * CHUNK * ws),
            "roofline": roofline, "kernels": kern, "e2e": e2e, "cpu_baseline": cpu,
            "clocks": clk.summary(), "gpu_launches": int(launches), "parity": parity,
            "reference_gpu": reference_gpu,
            "build_s": build_s, "autotune": tune, "driven_variant": driven, "pull_variant": pull,
            "delivery_ceiling": {"reductions_per_s": red_ceiling, "stream_read_gbs": read_ceiling / 1e9,
                                 "how": "mgc_measure_scatter: 1e8 random fp32 red.add into 2^20 "
                                        "accumulators fed by streamed 8-byte records; plain stream "
                                        "of the same records"},
        }
        print(json.dumps(line), flush=True)


def pull_variant(local, steps=3000, warm=1000):
    """Pull steps on the load they are for: the bursting network of
    mgbrain_b200.brunel.burst_network (10k LIFB, 1.1e7 synapses, volleys of
    more than half the neurons).  Device time of `steps` steps after `warm`,
    with the autotuner's choice (which times pull thresholds too), the
    windowed group pushing, and the windowed group with pull steps at three
    thresholds ((spike, delay) pairs per step); the end states of the
    windowed runs compared with the push-only one."""
    from mgbrain_b200 import brunel
    net = brunel.burst_network()
    S = len(net["src"])
    out = {"network": "burst: 8k exc + 2k inh LIFB, 1k POISSON @100 Hz, in-degree 800/200/100, J 0.1 mV, g 2, "
                      "one 1.5 ms delay (tests/burst_net.py); fires in volleys",
           "synapses": S, "steps": steps, "forms": {}}
    ref = None
    for label, pull, tune in (("autotuned", 0, True), ("push_window8", 0, False),
                              ("pull_500", 500, False), ("pull_1500", 1500, False), ("pull_3000", 3000, False)):
        sim = brunel.burst_simulator(net, device=local, raster_ids=-1)
        if tune:
            t = sim.autotune(steps_per_trial=640)
            form = {"persistent": t["persistent"], "window": t["window"], "chunk_len": t["chunk_len"],
                    "pull_min_pairs": t["pull_min"]}
        else:
            sim.set_persistent(3)
            sim.set_window(8)
            sim.set_pull(pull)
            form = {"persistent": 3, "window": 8, "pull_min_pairs": pull}
        left = warm + steps - sim.info()["step"]
        sim.run(max(0, left - steps))
        sim.sync()
        ms, ev, _ = timed_device(sim, steps, 1, 1)
        st = sim.state()
        end = (sim.info()["step"], st["V"].tobytes(), st["fire_cnt"].tobytes())
        if label == "push_window8":
            ref = end
        out["forms"][label] = {"us_per_step": 1e3 * ms / steps, "events_per_s": ev / (ms / 1e3),
                               "events_per_step": ev / steps, "form": form,
                               "end_state_equal_push": None if ref is None or tune else end == ref}
        sim.close()
    best = min((v["us_per_step"], k) for k, v in out["forms"].items() if k.startswith("pull"))
    out["best_pull"] = best[1]
    out["speedup_over_push"] = out["forms"]["push_window8"]["us_per_step"] / best[0]
    return out


def run_partition(a, ws, rank, local):
    """The large Brunel network split into one partition per rank (strong
    scaling): each rank simulates its neuron range on its GPU and the ranks
    all-gather spike ids every min_delay - 1 = 9 steps (NCCL; at one rank the
    exchange has nothing to send and measures the windowing's own cost).
    Device time on the partition's stream, max over ranks; at one rank the
    end state is compared with the unpartitioned handle's."""
    import torch

    import mgbrain_b200 as mgb
    from mgbrain_b200.partition import DistributedPartition, PartitionGroup, split
    torch.cuda.set_device(local)
    w = workload(a.scale)
    first, count = split(w["n"], ws)[rank]
    t0 = time.perf_counter()
    sim = mgb.Simulator.fixed_indegree(w["pops"], w["projs"], w["lif"], rate=w["rate"], v_init=w["v0"],
                                       conn_seed=1, seed=1, device=local, raster_ids=-1, part=(first, count))
    sim.sync()
    build_s = time.perf_counter() - t0
    cap = None if a.exchange == "exact" else max(256, count // 32)   # ids per step and partition
    if ws > 1:
        part = DistributedPartition(sim, device=f"cuda:{local}", cap_per_step=cap)
    else:
        part = PartitionGroup([sim], [local], cap_per_step=cap)
    for _ in range(a.warmup):
        part.run(CHUNK)
    torch.cuda.synchronize()
    barrier(ws)
    stream = torch.cuda.ExternalStream(sim.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0 = sim.info()["events"]
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(a.steps):
            part.run(CHUNK)
        e1.record(stream)
        e1.synchronize()
    sim.sync()   # raises if an exchange window was refused (the run would miss spikes)
    ms = allmax(ws, e0.elapsed_time(e1))
    events = allsum(ws, sim.info()["events"] - ev0)
    launches = sim.kernel_launches
    hbm, peak_kind = peaks()
    # the dominant kernel's algorithmic bytes over the timed region: 24 B per
    # LIFB neuron-step of this partition plus 8 B per delivered event
    lif_here = max(0, min(first + count, w["n_lif"]) - first)
    steps_timed = a.steps * CHUNK
    dbytes = 24.0 * lif_here * steps_timed + 8.0 * (events / ws)
    achieved = allmax(ws, dbytes / (ms / 1e3) / 1e9) if ms > 0 else 0.0
    # end to end through the C ABI: each bench step the rates from pinned
    # host memory, the steps with their exchanges, the fire counts read back
    pinned = torch.empty(count, dtype=torch.float32, pin_memory=True)
    pinned.numpy()[:] = w["rate"][first:first + count]
    import ctypes as C
    L = mgb.lib()
    torch.cuda.synchronize()
    barrier(ws)
    ev_e = sim.info()["events"]
    t0 = time.perf_counter()
    for _ in range(a.e2e_steps):
        mgb.capi.check(L.mgc_set_rates(sim._h, C.c_void_p(pinned.data_ptr()), count))
        part.run(CHUNK)
        fc = sim.state()["fire_cnt"]
    sim.sync()
    e2e_s = allmax(ws, time.perf_counter() - t0)
    e2e_ev = allsum(ws, sim.info()["events"] - ev_e)
    line = {"metric": METRIC, "value": events / (ms / 1e3), "unit": "events/s",
            "n_gpus": ws, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded, generated on the device)",
            "config": {"workload": "large Brunel: 1M LIFB (800k/200k) + 100k POISSON @20 Hz, fixed in-degree "
                                   "800/200/100, J 0.1 mV, g 5, delays U{10..50} steps, dt 0.1 ms, split into "
                                   "one contiguous neuron range per GPU",
                       "scale": a.scale, "bench_step": "1 s simulated (10,000 timesteps)",
                       "l2": "inputs larger than L2 (8.8 GB CSR)",
                       "parallelism": f"partitions x{ws} (spike ids all-gathered every {part.window} steps)"},
            "sim_s_per_wall_s": a.steps * CHUNK * DT / (ms / 1e3), "build_s": build_s,
            "window_steps": part.window,
            "partition": {"first": first, "neurons": count, "synapses": sim.S},
            "exchange": ("none (one partition)" if ws == 1 else
                         "NCCL all-gather of counts, then of ids (host waits)" if cap is None else
                         f"NCCL all-gather of fixed buffers on the stream, {cap} ids per step"),
            "roofline": {"bound": "hbm", "kernel": "step groups of the partition", "achieved": achieved,
                         "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": None},
            "e2e": {"value": e2e_ev / e2e_s, "unit": "events/s", "h2d_bytes_per_step": 4 * count,
                    "d2h_bytes_per_step": 4 * count},
            "gpu_launches": int(launches), "cpu_baseline": None, "clocks": clk.summary()}
    if ws == 1:
        whole = make_sim(w, local, seed=1, record=False)
        whole.run(CHUNK * (a.warmup + a.steps + a.e2e_steps))
        ws_ = whole.state()
        st = sim.state()
        line["identical_to_whole"] = bool(np.array_equal(st["V"].view(np.int32), ws_["V"].view(np.int32)) and
                                          np.array_equal(st["fire_cnt"], ws_["fire_cnt"]))
        whole.close()
    sim.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def split_raster(counts, ids, starts, steps):
    """Per-instance rasters (ids relative to the instance) from a batch raster."""
    offs = np.concatenate([[0], np.cumsum(counts)])
    step_of = np.repeat(np.arange(len(counts)), counts)
    inst = np.searchsorted(starts, ids, side="right") - 1
    out = []
    for i in range(len(starts) - 1):
        m = inst == i
        c = np.bincount(step_of[m], minlength=steps)[:steps]
        out.append((c, ids[m] - starts[i]))
    return out


def rank_share(count, ws, rank):
    """Indices of the independent units (sweep instances) rank `rank` of `ws`
    advances: dealt round-robin, so every unit runs on exactly one rank."""
    return [i for i in range(count) if i % ws == rank]


def run_sweep(a, ws, rank, local):
    """Parameter sweep of independent Brunel instances (N log-uniform in
    [1e3, 1e5], K = min(N/10, 1000), g ~ U[3, 7], nu_ext ~ U[10, 30] Hz).
    Batched + learned form: all of this rank's instances in one handle,
    autotuned, with the step scheduler calibrated, its network trained on the
    batch's own group trace and the learned mode on while timed.  Plain form:
    each instance in its own handle, run one after the other for the same
    steps.  Rasters of the two forms are compared instance by instance.  Instances are dealt to ranks round-robin
    (weak scaling: no collective on the data path)."""
    import torch

    import mgbrain_b200 as mgb
    from mgbrain_b200 import brunel
    torch.cuda.set_device(local)
    insts = brunel.sweep_instances(count=a.sweep_count)
    mine = [insts[i] for i in rank_share(len(insts), ws, rank)]
    T = a.sweep_steps
    n_all = sum(brunel.sweep_block(p)["n"] for p in mine)
    steps_cap = T + 8192                     # also holds the autotuner's and the scheduler's steps
    cap = lambda n: max(4096, n * steps_cap // 200)  # room for a mean rate of 50 Hz
    raster = dict(raster_steps=steps_cap)
    t0 = time.perf_counter()
    sim, starts = brunel.sweep_batch(mine, seed=1, raster_ids=cap(n_all), **raster)
    build_s = time.perf_counter() - t0
    info = sim.info()
    tune = sim.autotune(steps_per_trial=64)
    sim.read_raster(max_steps=steps_cap, max_ids=cap(n_all))  # drops the trial steps
    # the learned scheduler: calibrated threshold, trained on this batch's trace
    thr = sim.sched_calibrate(groups=8)
    sim.sched_collect(True, reset=True)
    sim.run(64 * 40)
    sim.sched_collect(False)
    loss = sim.sched_train(epochs=300, lr=3e-3, seed=7)
    sim.sched_mode(mgb.SCHED_LEARNED)
    sim.read_raster(max_steps=steps_cap, max_ids=cap(n_all))
    pre_steps = sim.info()["step"]
    for _ in range(a.warmup):
        sim.run(T)
        sim.read_raster(max_steps=T, max_ids=cap(n_all))
    with ClockSampler(local) as clk:
        ms, events, launches = timed_device(sim, T, 1, ws)
    _, counts, ids = sim.read_raster(max_steps=T, max_ids=cap(n_all))
    per_inst = split_raster(counts, ids, starts, T)
    sched = sim.sched_report()
    sim.close()
    batch_ev_s = allsum(ws, events) / (allmax(ws, ms) / 1e3)

    plain_ms = plain_events = 0.0
    plain_launches = 0
    same = 0
    for i in range(len(mine)):
        alone_n = brunel.sweep_block(mine[i])["n"]
        alone = brunel.sweep_alone(mine, i, seed=1, raster_ids=cap(alone_n), **raster)
        alone.run(pre_steps)  # the steps the batch spent in its autotuner and scheduler set-up
        alone.read_raster(max_steps=steps_cap, max_ids=cap(alone_n))
        for _ in range(a.warmup):
            alone.run(T)
            alone.read_raster(max_steps=T, max_ids=cap(alone_n))
        m_i, e_i, l_i = timed_device(alone, T, 1, 1)
        _, ca, ia = alone.read_raster(max_steps=T, max_ids=cap(alone_n))
        alone.close()
        plain_ms += m_i
        plain_events += e_i
        plain_launches += l_i
        cb, ib = per_inst[i]
        same += int(np.array_equal(cb, ca) and np.array_equal(ib, ia))
    plain_ev_s = allsum(ws, plain_events) / (allmax(ws, plain_ms) / 1e3)
    same = int(allsum(ws, same))
    if rank == 0:
        line = {
            "metric": "aggregate synaptic events/s on the parameter sweep, batched vs plain",
            "value": batch_ev_s, "unit": "events/s", "n_gpus": ws, "steps": T, "warmup": a.warmup,
            "higher_is_better": True, "scaling": "weak", "dtype": "f32",
            "data": "synthetic (seeded, generated on the device)",
            "config": {"workload": f"{a.sweep_count} Brunel instances, N log-uniform [1e3, 1e5], "
                                   "K = min(N/10, 1000) (80/20) + K/10 external, g ~ U[3, 7], "
                                   "nu_ext ~ U[10, 30] Hz, delay 1.5 ms, dt 0.1 ms",
                       "instances_per_gpu": len(mine), "neurons_gpu0": info["n_neurons"],
                       "synapses_gpu0": info["n_synapses"], "steps_per_form": T},
            "batched": {"events_per_s": batch_ev_s, "ms": ms, "kernel_launches": launches,
                        "build_s": build_s, "autotune": tune,
                        "scheduler": {"mode": "learned", "calibrated_threshold": thr, "train_loss": loss,
                                      "groups": sched["groups"], "misses": sched["misses"],
                                      "variant_groups": sched["variant_groups"]}},
            "plain": {"events_per_s": plain_ev_s, "ms": plain_ms, "kernel_launches": plain_launches},
            "batched_over_plain": batch_ev_s / plain_ev_s if plain_ev_s else None,
            "rasters_identical": f"{same}/{a.sweep_count}",
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)


def run_sched(a, ws, rank, local):
    """Step scheduler on a drive that alternates every 3 step groups (64
    steps each) between 20 Hz and 200 Hz inputs, on the Brunel network at
    --scale: the same steps under the static variant, the threshold rule and
    the learned rule (trained on the GPU on the first groups' trace); rasters
    compared, misses and wall time per mode reported.  The threshold comes
    from mgc_sched_calibrate."""
    import torch

    import mgbrain_b200 as mgb
    torch.cuda.set_device(local)
    group, g_train, g_eval = 64, a.sched_train_groups, a.sched_eval_groups
    w = workload(a.scale)
    rate_hi = w["rate"].copy()
    rate_hi[w["n_lif"]:] = NU_DRIVEN
    pinned = {k: torch.empty(w["n"], dtype=torch.float32, pin_memory=True) for k in ("lo", "hi")}
    pinned["lo"].numpy()[:] = w["rate"]
    pinned["hi"].numpy()[:] = rate_hi
    L = mgb.lib()
    import ctypes as C

    def drive(sim, g0, groups, loads=None):
        # rates for each group enqueued from pinned memory: no host sync
        # (unless the per-group loads are wanted)
        for g in range(g0, g0 + groups):
            src = pinned["hi" if (g // 3) % 2 == 0 else "lo"]
            mgb.capi.check(L.mgc_set_rates(sim._h, C.c_void_p(src.data_ptr()), w["n"]))
            e0 = sim.info()["events"] if loads is not None else 0
            sim.run(group)
            if loads is not None:
                loads.append(((g // 3) % 2 == 0, (sim.info()["events"] - e0) / group))

    sims = {m: make_sim(w, local, seed=1, record=True) for m in ("static", "threshold", "learned")}
    calib = sims["static"]
    calib.run(group)
    thr = calib.sched_calibrate(groups=16)
    rep_c = calib.sched_report()
    calib.close()
    sims["static"] = make_sim(w, local, seed=1, record=True)
    loads = []
    for m, sim in sims.items():
        sim.run(group)
        sim.sched_threshold(thr, rep_c["hi_variant"])
        sim.sched_collect(True, reset=True)
        drive(sim, 0, g_train, loads if m == "static" else None)
        sim.sched_collect(False)
        sim.read_raster(max_steps=1 << 20, max_ids=w["n"] * 64)
    t0 = time.perf_counter()
    loss = sims["learned"].sched_train(epochs=400, lr=3e-3, seed=7)
    train_s = time.perf_counter() - t0
    sims["threshold"].sched_mode(mgb.SCHED_THRESHOLD)
    sims["learned"].sched_mode(mgb.SCHED_LEARNED)
    out = {}
    rasters = {}
    for m, sim in sims.items():
        sim.sched_report(reset=True)
        stream = torch.cuda.ExternalStream(sim.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        drive(sim, g_train, g_eval)
        e1.record(stream)
        e1.synchronize()
        rep = sim.sched_report()
        rasters[m] = sim.read_raster(max_steps=1 << 20, max_ids=w["n"] * 64)
        out[m] = {"ms": e0.elapsed_time(e1), "groups": rep["groups"], "misses": rep["misses"],
                  "miss_rate": rep["misses"] / rep["groups"] if rep["groups"] else None,
                  "variant_groups": rep["variant_groups"]}
        if m == "learned":
            out[m]["mean_abs_log_err"] = rep["mean_abs_log_err"]
    # the same rule with its threshold between the two drive levels, where
    # every change of the drive can make a decision miss
    hi = float(np.median([x for h, x in loads if h]))
    lo = float(np.median([x for h, x in loads if not h]))
    thr_mid = float(np.sqrt(hi * lo))
    imposed = {}
    for m in ("threshold", "learned"):
        sim = sims[m]
        sim.sched_threshold(thr_mid, 1)
        sim.sched_report(reset=True)
        drive(sim, g_train + g_eval, g_eval)
        rep = sim.sched_report()
        imposed[m] = {"groups": rep["groups"], "misses": rep["misses"],
                      "miss_rate": rep["misses"] / rep["groups"] if rep["groups"] else None}
    sims["static"].sched_threshold(thr_mid, 1)
    drive(sims["static"], g_train + g_eval, g_eval)
    for m, sim in sims.items():
        c, i = sim.read_raster(max_steps=1 << 20, max_ids=w["n"] * 64)[1:]
        rasters[m] = (None, np.concatenate([rasters[m][1], c]), np.concatenate([rasters[m][2], i]))
    same = all(np.array_equal(rasters[m][1], rasters["static"][1]) and
               np.array_equal(rasters[m][2], rasters["static"][2]) for m in rasters)
    if rank == 0:
        print(json.dumps({
            "metric": "step-schedule misses and wall time, periodic drive",
            "config": {"workload": f"Brunel network at scale {a.scale}, inputs alternating 20/200 Hz every "
                                   "3 groups of 64 steps", "train_groups": g_train, "eval_groups": g_eval},
            "calibrated_threshold_events_per_step": thr, "hi_variant": rep_c["hi_variant"],
            "train_loss": loss, "train_s": train_s, "modes": out,
            "imposed_threshold": {"events_per_step": thr_mid, "low_load": lo, "high_load": hi, "modes": imposed},
            "rasters_identical": same,
        }), flush=True)
    for sim in sims.values():
        sim.close()


def run_refgpu(a, ws, rank, local):
    if rank != 0:
        return
    print(json.dumps(refgpu_compare(a, local)), flush=True)


def brunel_maker(nsyn, step):
    """ModelMaker::make_brunel (src/model/maker.h:10-25) as populations and
    projections for the device generator: 50 % POISSON inputs, 40 % exc, 10 %
    inh LIFB, every projection fixed-probability 0.1, the maker's weights and
    1.6 ms delay, computed in the same float / double mix."""
    import math
    import mgbrain_b200 as mgb
    prob = np.float32(0.1)
    size = int(math.sqrt(float(np.float32(nsyn)) / (float(prob) * 0.5)))
    pops = [(size * 5 // 10, mgb.POISSON), (size * 4 // 10, mgb.LIFB), (size * 1 // 10, mgb.LIFB)]
    w1 = float(np.float32(0.0001 * 20000 / size))
    w2 = float(np.float32(-0.0005 * 20000 / size))
    delay = int(np.floor(np.float32(0.0016) / np.float32(step) + np.float32(0.5)))
    P, E, I = 0, 1, 2
    projs = [dict(src=s_, tar=t_, rule=mgb.RULE_PROB, prob=float(prob), weight=w, delay=delay)
             for s_, t_, w in ((P, E, w1), (P, I, w1), (E, E, w1), (E, I, w1), (I, I, w2), (I, E, w2))]
    return pops, projs


def refgpu_compare(a, local):
    """The reference's own benchmark network (ModelMaker::make_brunel with
    --ref-syn synapses, Poisson inputs at 20 Hz, generated by the reference's
    gen_net) simulated for --ref-seconds by the reference's own
    MGSimulator::simulate on this GPU (its kernels built for sm_100a in
    oracle/_ref, Poisson draws through the shared counter-based generator)
    and by this core; wall times, and whether the end states agree.  A
    baseline leg: the reference's kernels are measured, not shipped."""
    import shutil
    import tempfile

    import mgbrain_b200 as mgb
    from mgbrain_b200 import netfile
    ref_gen = os.path.join(ROOT, "oracle", "_ref", "ref_gen")
    ref_sim = os.path.join(ROOT, "oracle", "_ref", "ref_sim")
    if not (os.path.exists(ref_gen) and os.path.exists(ref_sim)):
        return {"workload": "refgpu", "unavailable": "oracle/_ref is not built (make -C oracle ref)"}
    tmp = tempfile.mkdtemp()
    try:
        spec = os.path.join(tmp, "net.spec")
        with open(spec, "w") as f:
            f.write(f"timestep 0.0001\nmaker brunel {int(a.ref_syn)}\nrate 0 0.002\n")
        env = dict(os.environ, MGB_REF_MT_SEED="1", MGB_REF_RAND_SEED="1", MGB_REF_SEED="7")
        path = os.path.join(tmp, "net.net")
        t0 = time.perf_counter()
        subprocess.run([ref_gen, "gen", spec, path], check=True, env=env, capture_output=True)
        gen_s = time.perf_counter() - t0
        net = netfile.read_netfile(path)
        prefix = os.path.join(tmp, "ref")
        with ClockSampler(local) as clk_ref:
            r = subprocess.run([ref_sim, "simulate", path, prefix, str(a.ref_seconds), "-", "0"], check=True,
                               env=env, capture_output=True, text=True)
        ref_wall = float(r.stdout.split("wall")[1].split()[0])
        n, S = net["n"], len(net["src"])
        b = open(prefix + ".state", "rb").read()
        ref_v = np.frombuffer(b, np.float32, n, 0)
        ref_cnt = np.frombuffer(b, np.int32, n, 20 * n)
        t0 = time.perf_counter()
        sim = mgb.Simulator.from_arrays(n, net["type"], net["src"], net["tar"], net["weight"],
                                        netfile.delay_steps(net), netfile.default_lifconst(net),
                                        netfile.default_stdpconst(net), rate=net["rate"], seed=7, device=local,
                                        raster_ids=-1)
        sim.sync()
        build_s = time.perf_counter() - t0
        info = sim.info()
        steps = mgb.effective_steps(int(round(a.ref_seconds / net["step"])), info["min_delay"])
        import torch
        stream = torch.cuda.ExternalStream(sim.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk_ours:
            t0 = time.perf_counter()
            e0.record(stream)
            sim.run(steps)
            e1.record(stream)
            sim.sync()
            ours_wall = time.perf_counter() - t0
        ours_dev = e0.elapsed_time(e1) / 1e3
        st = sim.state()
        events = sim.info()["events"]
        # the same network generated on the device from the same mt19937 seed
        # (mgc_create_generated): synapse for synapse the reference's list
        pops, projs = brunel_maker(a.ref_syn, net["step"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gen = mgb.Simulator.generated(pops, projs, netfile.default_lifconst(net), mt_seed=1, rate=net["rate"],
                                      seed=7, device=local, raster_ids=-1)
        gen.sync()
        gen_dev_s = time.perf_counter() - t0
        ra, ta, wa, da = sim.export_csr()
        rb, tb, wb, db = gen.export_csr()
        netgen_identical = bool(np.array_equal(ra, rb) and np.array_equal(ta, tb) and np.array_equal(da, db) and
                                np.array_equal(wa.view(np.int32), wb.view(np.int32)))
        gen.close()
        sim.close()
        return {
            "workload": "refgpu",
            "netgen": {"reference_gen_net_s": gen_s, "ours_device_s": gen_dev_s, "identical": netgen_identical,
                       "how": "mgc_create_generated from the same mt19937 seed, CSR and weights compared with the "
                              "handle built from the reference gen_net's list"},
            "config": {"network": f"the reference's make_brunel, {S} synapses, {n} neurons, inputs 20 Hz, "
                                  f"dt 0.1 ms, generated by the reference's gen_net",
                       "seconds": a.ref_seconds, "steps": steps},
            "reference_simulate_wall_s": ref_wall, "ours_run_wall_s": ours_wall, "ours_device_s": ours_dev,
            "speedup_wall": ref_wall / ours_wall, "ours_events_per_s": events / ours_wall,
            "reference_events_per_s": events / ref_wall, "ours_build_s": build_s, "gen_s": gen_s,
            "fire_cnt_identical": bool(np.array_equal(st["fire_cnt"], ref_cnt)),
            "V_identical": bool(np.array_equal(st["V"].view(np.int32), ref_v.view(np.int32))),
            "spikes": int(st["fire_cnt"].sum()),
            "clocks": {"reference": clk_ref.summary(), "ours": clk_ours.summary()},
        }
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-sample", type=int, default=300)
    ap.add_argument("--ref-sample", type=int, default=200)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-driven", action="store_true")
    ap.add_argument("--no-pull", action="store_true", help="skip the bursting network's pull-step leg")
    ap.add_argument("--no-refgpu", action="store_true",
                    help="skip the reference's own kernels on this GPU (reference_gpu key)")
    ap.add_argument("--ref-syn", type=float, default=1e8)
    ap.add_argument("--ref-seconds", type=float, default=1.0)
    ap.add_argument("--workload", default="brunel1m",
                    choices=["brunel1m", "replicas", "sweep", "sched", "refgpu", "partition"],
                    help="brunel1m: the 1M-neuron network (default); sweep: batched vs plain "
                         "parameter sweep; sched: the step scheduler's modes on a periodic drive; refgpu: "
                         "the reference's own simulator and this core on the reference's benchmark network; "
                         "partition: the 1M-neuron network split over the ranks, spike ids exchanged")
    ap.add_argument("--exchange", choices=["device", "exact"], default="device",
                    help="partition workload: the device exchange (fixed capacity, no host wait) or the exact one")
    ap.add_argument("--sched-train-groups", type=int, default=200)
    ap.add_argument("--sched-eval-groups", type=int, default=300)
    ap.add_argument("--sweep-count", type=int, default=256)
    ap.add_argument("--sweep-steps", type=int, default=10000)
    ap.add_argument("--group-mode", type=int, default=0, choices=[0, 1, 2, 3],
                    help="with --kernel-profile or --no-autotune: 0 graphs of k_fused, 1 k_steps groups, "
                         "2 k_pipe groups, 3 k_window groups (window of min(8, minimum delay) steps)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the autotuner and run --group-mode (for launch lists)")
    ap.add_argument("--kernel-profile", choices=["quiet", "driven", "burst", "stdp"],
                    help="only build the network at --scale, run --warmup bench steps, 300 "
                         "steps as timed, and 300 profiled steps (separate kernels); for ncu captures. "
                         "burst: the bursting network with pull steps (--pull-min), 300 steps after the warm-up; "
                         "stdp: config 3's STDP network (ring push with STDP), 710 steps")
    ap.add_argument("--pull-min", type=int, default=1500,
                    help="with --kernel-profile burst: the pull-step threshold (arriving (spike, delay) pairs)")
    a = ap.parse_args()
    multi = int(os.environ.get("WORLD_SIZE", "1")) > 1
    split = a.impl == "ours" and (a.workload == "partition" or (a.workload == "brunel1m" and multi))
    ws, rank, local = dist_init("nccl" if split else "gloo")
    try:
        if split:
            # several GPUs: the one network split over them (strong scaling);
            # independent replicas with --workload replicas
            run_partition(a, ws, rank, local)
        elif a.workload == "sweep":
            run_sweep(a, ws, rank, local)
        elif a.workload == "sched":
            run_sched(a, ws, rank, local)
        elif a.workload == "refgpu":
            run_refgpu(a, ws, rank, local)
        elif a.kernel_profile == "stdp":
            # config 3's STDP network at its stated size, the ring push with
            # STDP fused (AUTO's method for plastic networks): one input epoch
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            import stdp_net
            import mgbrain_b200 as mgb
            net = stdp_net.build(n_in=784, n_exc=1600)
            sim = mgb.Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"],
                                            net["delay"], net["lifconst"], net["stdpconst"], stdp=True,
                                            plastic=net["plastic"], seed=11, device=local, raster_ids=-1)
            sim.set_rates(stdp_net.rates(net, 0))
            sim.run(stdp_net.REDRAW_STEPS + 10)
            sim.sync()
            print(json.dumps({"kernel_profile": "stdp", "info": sim.info()}))
        elif a.kernel_profile == "burst":
            # the bursting network with pull steps (the windowed group, 8 steps)
            from mgbrain_b200 import brunel
            sim = brunel.burst_simulator(brunel.burst_network(), device=local, raster_ids=-1)
            sim.set_persistent(3)
            sim.set_window(8)
            sim.set_pull(a.pull_min)
            sim.run(CHUNK * a.warmup)
            sim.run(300)
            sim.sync()
            print(json.dumps({"kernel_profile": "burst", "pull_min": a.pull_min, "info": sim.info()}))
        elif a.kernel_profile:
            w = workload(a.scale, nu=NU_DRIVEN if a.kernel_profile == "driven" else NU_STEP)
            sim = make_sim(w, local, seed=1, record=False)
            sim.set_persistent(a.group_mode)
            sim.run(CHUNK * a.warmup)
            sim.run(300)           # the timed region's kernels (k_fused per step)
            ms = sim.profile(300)  # then the step split into its kernel classes
            print(json.dumps({"kernel_profile": a.kernel_profile, "scale": a.scale,
                              "ms_per_300_steps": ms, "info": sim.info()}))
        elif a.impl == "reference":
            run_reference(a, ws, rank)
        else:
            run_ours(a, ws, rank, local)   # one GPU, or --workload replicas
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
