"""Brunel-type workloads built through the C ABI: the large network
(1M LIFB neurons, fixed in-degree) and the parameter sweep of many
independent instances of uneven size.  Sizes, seeds and distributions are
the workload definitions; the networks are generated on the device."""
from __future__ import annotations

import numpy as np

from .capi import LIFB, POISSON, Simulator

DT = 1e-4
J = 1e-4                 # 0.1 mV
DELAY_STEPS = 15         # 1.5 ms


def brunel_lifconst(dt=DT):
    """LIFB constants: V_th 20 mV, V_reset 10 mV, t_ref 2 ms (leak 0.005)."""
    c = np.zeros(30, np.float32)
    c[0], c[3], c[4], c[8] = dt, 0.01, 0.02, 0.002
    return c


def large_brunel(scale=1.0, nu_step=0.002, g=5.0, dmin=10, dmax=50, seed=1):
    """1M LIFB (80/20) + 100k POISSON inputs, in-degree 800 exc + 200 inh +
    100 external, delays uniform in [dmin, dmax] steps."""
    ne, ni, nx = int(800_000 * scale), int(200_000 * scale), int(100_000 * scale)
    n = ne + ni + nx
    pops = [(0, ne, LIFB), (ne, ni, LIFB), (ne + ni, nx, POISSON)]
    projs = []
    for tgt in (0, 1):
        projs += [(0, tgt, 800, J, dmin, dmax), (1, tgt, 200, -g * J, dmin, dmax),
                  (2, tgt, 100, J, dmin, dmax)]
    rate = np.zeros(n, np.float32)
    rate[ne + ni:] = nu_step
    v0 = np.random.default_rng(seed).uniform(0.0, 0.02, n).astype(np.float32)
    return dict(n=n, n_lif=ne + ni, pops=pops, projs=projs, lif=brunel_lifconst(), rate=rate, v0=v0)


def sweep_instances(count=256, n_min=1_000, n_max=100_000, seed=2026):
    """Instance parameters of the sweep: N log-uniform in [n_min, n_max],
    in-degree K = min(N/10, 1000) split 80/20 exc/inh plus K/10 external,
    g ~ U[3, 7], external rate ~ U[10, 30] Hz."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        N = int(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        g = float(rng.uniform(3.0, 7.0))
        nu = float(rng.uniform(10.0, 30.0))
        out.append(dict(N=N, g=g, nu=nu, conn_seed=1000 + i, v0_seed=5000 + i))
    return out


def sweep_block(p, dt=DT):
    """One sweep instance as a block (populations relative to the block)."""
    N = p["N"]
    ne = int(0.8 * N)
    ni = N - ne
    nx = max(1, N // 10)
    K = min(N // 10, 1000)
    ke = int(0.8 * K)
    ki = K - ke
    kx = max(1, K // 10)
    pops = [(0, ne, LIFB), (ne, ni, LIFB), (ne + ni, nx, POISSON)]
    projs = []
    for tgt in (0, 1):
        projs += [(0, tgt, ke, J, DELAY_STEPS, DELAY_STEPS),
                  (1, tgt, ki, -p["g"] * J, DELAY_STEPS, DELAY_STEPS),
                  (2, tgt, kx, J, DELAY_STEPS, DELAY_STEPS)]
    n = ne + ni + nx
    rate = np.zeros(n, np.float32)
    rate[ne + ni:] = np.float32(p["nu"] * dt)
    v0 = np.random.default_rng(p["v0_seed"]).uniform(0.0, 0.02, n).astype(np.float32)
    return dict(pops=pops, projs=projs, rate=rate, v_init=v0, conn_seed=p["conn_seed"], n=n,
                S=sum(pops[r[1]][1] * r[2] for r in projs))


def sweep_batch(instances, seed=1, **kw):
    """All instances in one handle; returns (sim, block starts)."""
    blocks = [sweep_block(p) for p in instances]
    sim = Simulator.batch(blocks, brunel_lifconst(), seed=seed, **kw)
    starts = np.cumsum([0] + [b["n"] for b in blocks])
    return sim, starts


def sweep_alone(instances, i, seed=1, **kw):
    """Instance i in a handle of its own, drawing as it does in the batch."""
    blocks = [sweep_block(p) for p in instances]
    start = int(sum(b["n"] for b in blocks[:i]))
    proj_off = 6 * i
    b = blocks[i]
    return Simulator.fixed_indegree(b["pops"], b["projs"], brunel_lifconst(), rate=b["rate"],
                                    v_init=b["v_init"], conn_seed=b["conn_seed"], seed=seed,
                                    id_offset=start, proj_offset=proj_off, **kw)


def burst_network(ne=8000, ni=2000, nx=1000, ke=800, ki=200, kx=100, J=1e-4, g=2.0, d=15, rate=0.01, seed=0):
    """A Brunel network in the synchronous regime, the load pull steps
    (Simulator.set_pull) are for: ne exc + ni inh LIFB with the large
    network's neuron constants, nx POISSON inputs at `rate` per step, fixed
    in-degree ke exc / ki inh / kx inputs per neuron (sources drawn with
    numpy's default_rng(seed)), J, g = 2 (excitation dominates), one delay of
    d steps.  It fires in volleys: in some steps more than half of the
    neurons spike, and their events (about ke + ki per spike) arrive
    together d steps later.  Returns the synapse list and the arrays
    Simulator.from_arrays takes (delays in steps)."""
    rng = np.random.default_rng(seed)
    n = ne + ni + nx
    types = np.array([LIFB] * (ne + ni) + [POISSON] * nx, np.int8)
    k = ke + ki + kx
    src = np.empty((ne + ni, k), np.int32)
    src[:, :ke] = rng.integers(0, ne, (ne + ni, ke))
    src[:, ke:ke + ki] = ne + rng.integers(0, ni, (ne + ni, ki))
    src[:, ke + ki:] = ne + ni + rng.integers(0, nx, (ne + ni, kx))
    src = src.reshape(-1)
    tar = np.repeat(np.arange(ne + ni, dtype=np.int32), k)
    w = np.where(src < ne, J, np.where(src < ne + ni, -g * J, J)).astype(np.float32)
    r = np.zeros(n, np.float32)
    r[ne + ni:] = rate
    v0 = np.random.default_rng(seed + 1).uniform(0.0, 0.02, n).astype(np.float32)
    return dict(n=n, type=types, rate=r, src=src, tar=tar, weight=w, dsteps=np.full(len(src), d, np.int32),
                lifconst=brunel_lifconst(), v0=v0, d=d)


def burst_simulator(net, seed=3, **kw):
    """The handle of a burst_network (Simulator.from_arrays)."""
    return Simulator.from_arrays(net["n"], net["type"], net["src"], net["tar"], net["weight"], net["dsteps"],
                                 net["lifconst"], rate=net["rate"], v_init=net["v0"], seed=seed, **kw)
