"""Networks as files: the MGBNET02 format (a `Network` as the reference's
`NetGen::gen_net` fills it, src/model/network.h:28-68) and the constants and
delay steps the reference derives from it when it builds the simulator.

Layout (little-endian): "MGBNET02", i32 n_pops, i32 n, i64 S, f32 step,
f32 dw, i32 nlifconst, i32 nstdpconst, f32 lifconst[30], f32 stdpconst[6],
i32 pops[n_pops][4], i8 type[n], f32 rate[n], i32 src[S], i32 tar[S],
f32 weight[S], f32 delay[S] (seconds)."""
from __future__ import annotations

import numpy as np

MAGIC = b"MGBNET02"


def read_netfile(path):
    with open(path, "rb") as f:
        b = f.read()
    if b[:8] != MAGIC:
        raise ValueError(f"{path}: not an MGBNET02 file")
    o = 8
    n_pops, n = (int(x) for x in np.frombuffer(b, np.int32, 2, o)); o += 8  # Python ints: offsets pass 2^31
    S = int(np.frombuffer(b, np.int64, 1, o)[0]); o += 8
    step, dw = np.frombuffer(b, np.float32, 2, o); o += 8
    nl, ns = (int(x) for x in np.frombuffer(b, np.int32, 2, o)); o += 8
    lif = np.frombuffer(b, np.float32, 30, o).copy(); o += 120
    stdp = np.frombuffer(b, np.float32, 6, o).copy(); o += 24
    pops = np.frombuffer(b, np.int32, 4 * n_pops, o).reshape(n_pops, 4).copy(); o += 16 * n_pops
    typ = np.frombuffer(b, np.int8, n, o).copy(); o += n
    rate = np.frombuffer(b, np.float32, n, o).copy(); o += 4 * n
    src = np.frombuffer(b, np.int32, S, o).copy(); o += 4 * S
    tar = np.frombuffer(b, np.int32, S, o).copy(); o += 4 * S
    w = np.frombuffer(b, np.float32, S, o).copy(); o += 4 * S
    d = np.frombuffer(b, np.float32, S, o).copy(); o += 4 * S
    return dict(n=n, type=typ, rate=rate, src=src, tar=tar, weight=w, delay=d,
                step=float(step), dw=float(dw), nlifconst=int(nl), nstdpconst=int(ns),
                lifconst=lif, stdpconst=stdp, pops=pops)


def write_netfile(path, net):
    n, S = int(net["n"]), len(net["src"])
    pops = np.asarray(net["pops"], np.int32).reshape(-1, 4)
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(np.array([len(pops), n], np.int32).tobytes())
        f.write(np.array([S], np.int64).tobytes())
        f.write(np.array([net["step"], net["dw"]], np.float32).tobytes())
        f.write(np.array([net.get("nlifconst", 0), net.get("nstdpconst", 0)], np.int32).tobytes())
        f.write(np.asarray(net.get("lifconst", np.zeros(30)), np.float32).tobytes())
        f.write(np.asarray(net.get("stdpconst", np.zeros(6)), np.float32).tobytes())
        f.write(pops.tobytes())
        f.write(np.asarray(net["type"], np.int8).tobytes())
        f.write(np.asarray(net["rate"], np.float32).tobytes())
        for k, dt in (("src", np.int32), ("tar", np.int32), ("weight", np.float32), ("delay", np.float32)):
            f.write(np.asarray(net[k], dt).tobytes())


def default_lifconst(net):
    """LIFECONSTS the reference kernels see (mgsim.cpp:165-172, mgcore.cu:32-63,
    :685-748): the network's array when set; else the __constant__ initialiser
    when only STDP constants are set; else copy_consts_gpu's default array."""
    if net.get("nlifconst", 0):
        return np.asarray(net["lifconst"], np.float32)
    c = np.zeros(30, np.float32)
    c[21:26] = [0.951229453, 0.967216074, 0.0799999982, 0.0599999987, 0.90483743]
    c[5], c[6], c[8], c[10], c[11] = 0.25, 10.0, 0.0004, 1.0, 1.0
    if net.get("nstdpconst", 0):
        c[0], c[4] = 0.0001, 0.02
    else:
        c[0], c[4] = net["step"], 15.0
    return c


def default_stdpconst(net):
    if net.get("nstdpconst", 0):
        return np.asarray(net["stdpconst"], np.float32)
    return np.array([0.1, -0.01, 17, 34, 40, 0], np.float32)


def delay_steps(net):
    """Delays in steps as build_multinet quantises them (mgsim.cpp:49):
    round(delay / step) in fp32, halves away from zero."""
    q = np.asarray(net["delay"], np.float32) / np.float32(net["step"])
    return np.floor(q + np.float32(0.5)).astype(np.int32)
