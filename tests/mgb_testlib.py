"""Test helpers: the oracle (ctypes), the model-description parser, the
network/raster file readers and the reference-driver runner.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use
this module; the oracle it loads is the checker, never the product.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "libmgb_oracle.so")
REF_GEN = os.path.join(ORACLE_DIR, "_ref", "ref_gen")
REF_SIM = os.path.join(ORACLE_DIR, "_ref", "ref_sim")
GOLDEN = os.path.join(ROOT, "tests", "golden")

TYPES = {"RAW": 0, "LIF0": 1, "POISSON": 2, "LIF": 3, "LIFE": 4, "LIFB": 5}
F32, F64 = 0, 1


# --------------------------------------------------------------------------
# oracle binding
# --------------------------------------------------------------------------
class MgboPop(C.Structure):
    _fields_ = [("num", C.c_int32), ("type", C.c_int32), ("source", C.c_int32)]


class MgboProj(C.Structure):
    _fields_ = [("src", C.c_int32), ("tar", C.c_int32), ("wmin", C.c_float),
                ("wmax", C.c_float), ("dmin", C.c_float), ("dmax", C.c_float),
                ("ctype", C.c_float), ("stype", C.c_int32)]


class MgboSynlist(C.Structure):
    _fields_ = [("n_syn", C.c_int64), ("src", C.POINTER(C.c_int32)),
                ("tar", C.POINTER(C.c_int32)), ("weight", C.POINTER(C.c_float)),
                ("delay", C.POINTER(C.c_float)), ("proj", C.POINTER(C.c_int32))]


_oracle = None


def oracle():
    """Load (building if needed) the CPU oracle."""
    global _oracle
    if _oracle is not None:
        return _oracle
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", ORACLE_DIR], check=True, capture_output=True)
    L = C.CDLL(ORACLE_SO)
    vp, i32, i64, u64, f32 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64, C.c_float
    L.mgbo_netgen.restype = C.c_int
    L.mgbo_netgen.argtypes = [C.POINTER(MgboPop), C.c_int, C.POINTER(MgboProj), C.c_int,
                              C.c_uint32, i64, f32, f32, C.c_int, C.POINTER(MgboSynlist)]
    L.mgbo_synlist_free.argtypes = [C.POINTER(MgboSynlist)]
    L.mgbo_model_connect.restype = C.c_int
    L.mgbo_model_connect.argtypes = [C.POINTER(MgboProj), C.c_int, C.POINTER(MgboPop), MgboProj,
                                     C.POINTER(C.c_int)]
    L.mgbo_quantize_delays.argtypes = [vp, i64, f32, vp, C.POINTER(i32), C.POINTER(i32)]
    L.mgbo_steps_for_time.restype = i64
    L.mgbo_steps_for_time.argtypes = [f32, f32]
    L.mgbo_effective_steps.restype = i64
    L.mgbo_effective_steps.argtypes = [i64, i32]
    L.mgbo_create.restype = vp
    L.mgbo_create.argtypes = [i32, vp, vp, vp, i64, vp, vp, vp, vp, vp, vp, i32, vp, u64, i32, i32]
    L.mgbo_create_fixed_indegree.restype = vp
    L.mgbo_create_fixed_indegree.argtypes = [vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, i32, vp, vp,
                                             vp, u64, u64, i32, i32, i32]
    L.mgbo_set_id_offset.argtypes = [vp, i32]
    L.mgbo_set_fx.argtypes = [vp, i32]
    L.mgbo_set_fx.restype = C.c_int
    L.mgbo_run.restype = C.c_int
    L.mgbo_run.argtypes = [vp, i64, vp, vp, i64, C.POINTER(i64)]
    L.mgbo_set_rates.argtypes = [vp, vp]
    L.mgbo_set_threads.argtypes = [vp, i32]
    for name in ("mgbo_events", "mgbo_step", "mgbo_n_syn"):
        getattr(L, name).restype = i64
        getattr(L, name).argtypes = [vp]
    for name in ("mgbo_ring_len", "mgbo_min_delay"):
        getattr(L, name).restype = i32
        getattr(L, name).argtypes = [vp]
    L.mgbo_read_state.argtypes = [vp] + [vp] * 7
    L.mgbo_read_state_f32.argtypes = [vp, vp, vp]
    L.mgbo_export_csr.argtypes = [vp, vp, vp, vp, vp]
    L.mgbo_destroy.argtypes = [vp]
    _oracle = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# --------------------------------------------------------------------------
# model description (oracle/mgb_spec.h grammar)
# --------------------------------------------------------------------------
@dataclass
class Spec:
    text: str
    dt: float = 0.001          # Config::STEP default (macro.cpp:3)
    dw: float = 0.01           # Config::DW default (macro.cpp:5)
    shuffle: int = 0
    pops: list = field(default_factory=list)    # (num, type, source)
    pros: list = field(default_factory=list)    # MgboProj
    rates: list = field(default_factory=list)   # (pop, rate)


def _f32(x):
    return float(np.float32(x))


def _connect(spec, src, tar, wmin, wmax, dmin, dmax, ctype, stype):
    L = oracle()
    pops = (MgboPop * max(1, len(spec.pops)))(*[MgboPop(n, t, s) for n, t, s in spec.pops])
    arr = (MgboProj * (len(spec.pros) + 1))(*spec.pros)
    ok = C.c_int(0)
    p = MgboProj(src, tar, _f32(wmin), _f32(wmax), _f32(dmin), _f32(dmax), _f32(ctype), stype)
    n = L.mgbo_model_connect(arr, len(spec.pros), pops, p, C.byref(ok))
    spec.pros = [arr[i] for i in range(n)]


def _maker(spec, which, nsyn):
    """ModelMaker::make_brunel / make_vogel (src/model/maker.h:10-43),
    with the same float/double conversions."""
    if which == "brunel":
        con_prob = np.float32(0.1)
        pop_size = int(math.sqrt(float(np.float32(nsyn)) / (float(con_prob) * 0.5)))
        base = len(spec.pops)
        spec.pops += [(pop_size * 5 // 10, TYPES["POISSON"], 1),
                      (pop_size * 4 // 10, TYPES["LIFB"], 0),
                      (pop_size * 1 // 10, TYPES["LIFB"], 0)]
        w1 = _f32(0.0001 * 20000 / pop_size)
        w2 = _f32(-0.0005 * 20000 / pop_size)
        d1 = _f32(0.0016)
        p, e, i = base, base + 1, base + 2
        for s, t, w in ((p, e, w1), (p, i, w1), (e, e, w1), (e, i, w1), (i, i, w2), (i, e, w2)):
            _connect(spec, s, t, w, w, d1, d1, con_prob, 0)
    elif which == "vogel":
        con_prob = np.float32(0.02)
        pop_size = int(np.sqrt(np.float32(nsyn) / con_prob))
        base = len(spec.pops)
        spec.pops += [(pop_size * 8 // 10, TYPES["LIFE"], 0), (pop_size * 2 // 10, TYPES["LIFE"], 0)]
        w1 = _f32(0.4 * 16000000 / pop_size / pop_size)
        w2 = _f32(-5.1 * 16000000 / pop_size / pop_size)
        d1 = _f32(0.0008)
        pe, pi = base, base + 1
        for s, t, w in ((pe, pe, w1), (pe, pi, w1), (pi, pe, w2), (pi, pi, w2)):
            _connect(spec, s, t, w, w, d1, d1, con_prob, 0)
    else:
        raise ValueError(which)


def parse_spec(text: str) -> Spec:
    spec = Spec(text=text)
    for raw in text.splitlines():
        tok = raw.split()
        if not tok or tok[0].startswith("#"):
            continue
        kw = tok[0]
        if kw == "timestep":
            spec.dt = _f32(tok[1])
        elif kw == "dw":
            spec.dw = _f32(tok[1])
        elif kw == "shuffle":
            spec.shuffle = int(tok[1])
        elif kw in ("lifconst", "life_const", "stdpconst"):
            pass  # constants travel inside the generated network file
        elif kw == "pop":
            spec.pops.append((int(tok[1]), TYPES[tok[2]], int(tok[3])))
        elif kw == "conn":
            s, t = int(tok[1]), int(tok[2])
            wmin, wmax, dmin, dmax, ct = (float(x) for x in tok[3:8])
            _connect(spec, s, t, wmin, wmax, dmin, dmax, ct, 1 if tok[8] == "STDP" else 0)
        elif kw == "maker":
            _maker(spec, tok[1], int(tok[2]))
        elif kw == "rate":
            spec.rates.append((int(tok[1]), _f32(tok[2])))
        else:
            raise ValueError("unknown spec keyword " + kw)
    return spec


def oracle_netgen(spec: Spec, mt_seed: int, rand_seed: int):
    """gen_net restated by the oracle; returns a network dict like read_netfile."""
    L = oracle()
    pops = (MgboPop * max(1, len(spec.pops)))(*[MgboPop(n, t, s) for n, t, s in spec.pops])
    pros = (MgboProj * max(1, len(spec.pros)))(*spec.pros)
    out = MgboSynlist()
    rc = L.mgbo_netgen(pops, len(spec.pops), pros, len(spec.pros), mt_seed, rand_seed,
                       spec.dw, spec.dt, spec.shuffle, C.byref(out))
    assert rc == 0
    S = out.n_syn

    def take(ptr, dt):
        if S == 0:
            return np.zeros(0, dt)
        return np.ctypeslib.as_array(ptr, shape=(S,)).astype(dt).copy()

    net = {
        "src": take(out.src, np.int32), "tar": take(out.tar, np.int32),
        "weight": take(out.weight, np.float32), "delay": take(out.delay, np.float32),
        "proj": take(out.proj, np.int32),
    }
    L.mgbo_synlist_free(C.byref(out))
    n = sum(p[0] for p in spec.pops)
    types = np.concatenate([np.full(p[0], p[1], np.int8) for p in spec.pops]) if spec.pops \
        else np.zeros(0, np.int8)
    rate = np.zeros(n, np.float32)
    starts = np.cumsum([0] + [p[0] for p in spec.pops])
    for pop, r in spec.rates:
        rate[starts[pop]:starts[pop + 1]] = r
    net.update(n=n, type=types, rate=rate, step=spec.dt, dw=spec.dw,
               pops=np.array([[i, p[0], p[2], p[1]] for i, p in enumerate(spec.pops)], np.int32))
    return net


# --------------------------------------------------------------------------
# files
# --------------------------------------------------------------------------
# the network file format and the reference's constant selection live in
# the package; re-exported for the tests
from mgbrain_b200.netfile import read_netfile, write_netfile  # noqa: E402,F401


def read_raster(path):
    b = open(path, "rb").read()
    steps = int(np.frombuffer(b, np.int64, 1, 0)[0])
    counts = np.frombuffer(b, np.int64, steps, 8).copy()
    ids = np.frombuffer(b, np.int32, int(counts.sum()), 8 + 8 * steps).copy()
    return counts, ids


def read_state(path, n, S):
    b = open(path, "rb").read()
    o = 0
    out = {}
    for k, dt in (("V", np.float32), ("Iexc", np.float32), ("Iinh", np.float32),
                  ("refrac", np.int32), ("last_fired", np.int32), ("fire_cnt", np.int32)):
        out[k] = np.frombuffer(b, dt, n, o).copy()
        o += 4 * n
    out["weight"] = np.frombuffer(b, np.float32, S, o).copy()
    return out


# --------------------------------------------------------------------------
# simulation through the oracle
# --------------------------------------------------------------------------
from mgbrain_b200.netfile import default_lifconst, default_stdpconst  # noqa: E402,F401


def quantize_delays(delay_s, step):
    L = oracle()
    d = np.ascontiguousarray(delay_s, np.float32)
    out = np.zeros(len(d), np.int32)
    lo, hi = C.c_int32(), C.c_int32()
    L.mgbo_quantize_delays(_p(d), len(d), step, _p(out), C.byref(lo), C.byref(hi))
    return out, lo.value, hi.value


class OracleSim:
    def __init__(self, net, seed, v0=None, stdp=0, plastic=None, precision=F32, nthreads=1):
        L = oracle()
        self.L = L
        self.n = int(net["n"])
        self.S = len(net["src"])
        self.dsteps, self.dmin, self.dmax = quantize_delays(net["delay"], net["step"])
        keep = [np.ascontiguousarray(net["type"], np.int8),
                np.ascontiguousarray(net["rate"], np.float32),
                None if v0 is None else np.ascontiguousarray(v0, np.float32),
                np.ascontiguousarray(net["src"], np.int32),
                np.ascontiguousarray(net["tar"], np.int32),
                np.ascontiguousarray(net["weight"], np.float32),
                self.dsteps, default_lifconst(net), default_stdpconst(net),
                None if plastic is None else np.ascontiguousarray(plastic, np.uint8)]
        self.precision = precision
        self.h = L.mgbo_create(self.n, _p(keep[0]), _p(keep[1]), _p(keep[2]), self.S,
                               _p(keep[3]), _p(keep[4]), _p(keep[5]), _p(keep[6]), _p(keep[7]),
                               _p(keep[8]), stdp, _p(keep[9]), seed, precision, nthreads)
        assert self.h, "oracle create failed"

    def run(self, steps, record=True):
        counts = np.zeros(steps, np.int64)
        cap = self.n * steps if record else 0
        ids = np.zeros(max(cap, 1), np.int32) if record else None
        nid = C.c_int64()
        rc = self.L.mgbo_run(self.h, steps, _p(counts), _p(ids), cap, C.byref(nid))
        assert rc == 0
        return counts, (ids[:nid.value].copy() if record else None)

    def set_rates(self, rate):
        r = np.ascontiguousarray(rate, np.float32)
        self.L.mgbo_set_rates(self.h, _p(r))

    def set_fx(self, shift):
        """Fixed-point accumulation with the CUDA core's shift (before the
        first step): the core's order-independent sums, bit for bit."""
        assert self.L.mgbo_set_fx(self.h, int(shift)) == 0

    def state(self):
        n, S = self.n, self.S
        out = {k: np.zeros(n, np.float64) for k in ("V", "Iexc", "Iinh")}
        for k in ("refrac", "last_fired", "fire_cnt"):
            out[k] = np.zeros(n, np.int32)
        out["weight"] = np.zeros(S, np.float64)
        self.L.mgbo_read_state(self.h, _p(out["V"]), _p(out["Iexc"]), _p(out["Iinh"]),
                               _p(out["refrac"]), _p(out["last_fired"]), _p(out["fire_cnt"]),
                               _p(out["weight"]))
        if self.precision == F32:
            v = np.zeros(n, np.float32)
            w = np.zeros(S, np.float32)
            self.L.mgbo_read_state_f32(self.h, _p(v), _p(w))
            out["V32"], out["weight32"] = v, w
        return out

    @property
    def events(self):
        return self.L.mgbo_events(self.h)

    @property
    def ring_len(self):
        return self.L.mgbo_ring_len(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.mgbo_destroy(self.h)
            self.h = None


def split_raster(counts, ids):
    """Per-step arrays of spike ids."""
    offs = np.concatenate([[0], np.cumsum(counts)])
    return [ids[offs[i]:offs[i + 1]] for i in range(len(counts))]


def ref_gen(spec_text, mt_seed, rand_seed, out_path):
    """Run the reference's own gen_net (oracle/_ref/ref_gen)."""
    spec_path = out_path + ".spec"
    with open(spec_path, "w") as f:
        f.write(spec_text)
    env = dict(os.environ, MGB_REF_MT_SEED=str(mt_seed), MGB_REF_RAND_SEED=str(rand_seed))
    subprocess.run([REF_GEN, "gen", spec_path, out_path], check=True, env=env,
                   capture_output=True)
    return read_netfile(out_path)


def ref_steps(net, v0, seed, steps, workdir, stdp=0, rates_off=None):
    """The reference kernels (oracle/_ref/ref_sim, its own sm_100a build) run
    for exactly `steps` steps on `net` (written as a network file), POISSON
    draws keyed by `seed`; from step rates_off on every POISSON rate is 0.
    Returns (counts, ids, state), or None when the reference build is absent."""
    if not os.path.exists(REF_SIM):
        return None
    netp = os.path.join(workdir, "net.mgbnet")
    write_netfile(netp, net)
    v0p = "-"
    if v0 is not None:
        v0p = os.path.join(workdir, "v0.f32")
        np.ascontiguousarray(v0, np.float32).tofile(v0p)
    out = os.path.join(workdir, "ref")
    args = [REF_SIM, "steps", netp, out, str(int(steps)), v0p, str(int(stdp))]
    if rates_off is not None:
        args.append(str(int(rates_off)))
    env = dict(os.environ, MGB_REF_SEED=str(int(seed)))
    subprocess.run(args, check=True, env=env, capture_output=True)
    counts, ids = read_raster(out + ".raster")
    return counts, ids, read_state(out + ".state", int(net["n"]), len(net["src"]))


def rate_and_cv(counts, ids, n, steps, dt):
    """Mean rate (Hz) over all n neurons, and the mean CV of the inter-spike
    intervals over the neurons with at least three spikes (and how many)."""
    step_of = np.repeat(np.arange(len(counts)), counts)
    order = np.lexsort((step_of, ids))
    sid, sst = ids[order], step_of[order]
    cvs = []
    bounds = np.flatnonzero(np.diff(sid)) + 1
    for a, b in zip(np.r_[0, bounds], np.r_[bounds, len(sid)]):
        if b - a >= 3:
            isi = np.diff(sst[a:b]).astype(np.float64)
            cvs.append(isi.std() / isi.mean())
    return len(ids) / (n * steps * dt), (float(np.mean(cvs)) if cvs else 0.0), len(cvs)


def fx_shift_for(bound, min_exp, exact):
    """The fixed-point shift rule of the CUDA core's builder (build.cu,
    fx_shift_for): the sums must fit 61 bits, and no finer than needed to make
    every weight an exact multiple of 2^-shift."""
    k = 0
    if bound > 0.0:
        e = int(np.frexp(np.float64(bound))[1])
        k = 61 - e
        if exact:
            k = min(k, 24 - int(min_exp))
    return max(-100, min(120, k))


def fx_plan(net, stdp=False, plastic=None, wlim=0.0):
    """(hetero, shift) of a synapse list as the core's builder computes them:
    hetero when some target receives unequal weights of one sign (or weights
    are plastic)."""
    n = int(net["n"])
    tar = np.asarray(net["tar"], np.int64)
    w = np.asarray(net["weight"], np.float32)
    pl = np.zeros(len(w), bool)
    if stdp:
        pl = np.ones(len(w), bool) if plastic is None else np.asarray(plastic) != 0
    mag = np.abs(w.astype(np.float64))
    mag = np.where(pl, np.maximum(mag, float(wlim)), mag)
    bound = float(np.bincount(tar, weights=mag, minlength=n).max()) if len(w) else 0.0
    nz = w[w != 0]
    min_exp = int(np.frexp(nz)[1].min()) if len(nz) else 1 << 20
    hetero = False
    for sel in (w > 0, w <= 0):
        if sel.any():
            lo = np.full(n, np.inf)
            hi = np.full(n, -np.inf)
            np.minimum.at(lo, tar[sel], w[sel].astype(np.float64))
            np.maximum.at(hi, tar[sel], w[sel].astype(np.float64))
            hetero |= bool(np.any(hi > lo))
    return hetero or bool(pl.any()), fx_shift_for(bound, min_exp, not pl.any())


def equal_per_sign(w):
    w = np.asarray(w)
    return len(np.unique(w[w > 0])) <= 1 and len(np.unique(w[w <= 0])) <= 1


def gen_projs(spec, net):
    """The projections of a model description as mgc_create_generated takes
    them; ranged weights and delays (which NetGen draws with glibc rand())
    come from `net`, the list gen_net made for the same description (its
    per-synapse projection index says whose they are)."""
    import mgbrain_b200 as mgb
    out = []
    proj = np.asarray(net["proj"])
    dsteps, _, _ = quantize_delays(net["delay"], net["step"])
    for r, p in enumerate(spec.pros):
        if p.ctype == 1.0:
            rule = mgb.RULE_ALL
        elif p.ctype == 0.0:
            rule = mgb.RULE_ONE
        else:
            rule = mgb.RULE_PROB
        # plastic: every synapse takes part when STDP is on (Config::STDP), as in gen_net
        d = dict(src=p.src, tar=p.tar, rule=rule, prob=float(p.ctype), plastic=1)
        sel = proj == r
        if p.wmin == p.wmax:
            d["weight"] = float(p.wmin)
        else:
            d["weights"] = np.asarray(net["weight"])[sel]
        if p.dmin == p.dmax:
            d["delay"] = int(quantize_delays(np.array([p.dmin], np.float32), spec.dt)[0][0])
        else:
            d["delays"] = dsteps[sel]
        out.append(d)
    return out
