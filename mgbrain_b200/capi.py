"""ctypes binding of the C ABI in include/mgc.h.

The library is the in-tree build mgbrain_b200/lib/libmgbrain_b200.so.  There
is no fallback: if it is missing or cannot run on this machine, every entry
point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

# MGBRAIN_LIB=checked selects the index-checking build (every index the
# kernels read from memory is tested before use; a failure is reported by
# sync), for debugging a network or the library.
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib",
                        "libmgbrain_b200_checked.so" if os.environ.get("MGBRAIN_LIB") == "checked"
                        else "libmgbrain_b200.so")

MGC_OK, MGC_ERR_INVALID, MGC_ERR_CUDA, MGC_ERR_NOMEM, MGC_ERR_OVERFLOW, MGC_ERR_NODEVICE = range(6)
RAW, LIF0, POISSON, LIF, LIFE, LIFB = range(6)
MODE_AUTO, MODE_PUSH, MODE_DEFERRED, MODE_PULL = 0, 1, 2, 3
SCHED_STATIC, SCHED_THRESHOLD, SCHED_LEARNED = 0, 1, 2
ACC_FLOAT, ACC_FIXED = 0, 1
RULE_PROB, RULE_ALL, RULE_ONE, RULE_ALL_BUT_SELF, RULE_FIXED_INDEGREE = range(5)
MLP_IN, MLP_HIDDEN, MLP_OUT, MLP_PARAMS = 20, 32, 5, 837

EXPORTED = (
    "mgc_create", "mgc_create_fixed_indegree", "mgc_run", "mgc_sync", "mgc_set_rates",
    "mgc_read_raster", "mgc_read_state", "mgc_read_weights", "mgc_export_csr", "mgc_get_info",
    "mgc_get_stream", "mgc_effective_steps", "mgc_destroy", "mgc_last_error",
    "mgc_kernel_launches", "mgc_profile_steps", "mgc_create_batch", "mgc_row_offsets_static",
    "mgc_measure_scatter", "mgc_autotune", "mgc_autotune_rewind", "mgc_set_persistent", "mgc_set_window", "mgc_set_pull", "mgc_checkpoint_size",
    "mgc_checkpoint_save", "mgc_checkpoint_load", "mgc_sched_set_mode", "mgc_sched_set_threshold",
    "mgc_sched_calibrate", "mgc_sched_collect", "mgc_sched_train", "mgc_sched_report", "mgc_mlp_gradient",
    "mgc_create_partition", "mgc_create_fixed_indegree_partition", "mgc_part_export", "mgc_part_import",
    "mgc_fault_inject_alloc", "mgc_selftest_wait_timeout", "mgc_partition_stats", "mgc_part_export_dev",
    "mgc_part_import_dev", "mgc_raster_stage", "mgc_raster_collect", "mgc_set_accumulation",
    "mgc_create_generated", "mgc_gen_count",
)


class MgcError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"mgc status {status}: {msg}")
        self.status = status


class NetDesc(C.Structure):
    _fields_ = [
        ("n_neurons", C.c_int32), ("type", C.c_void_p), ("rate", C.c_void_p),
        ("v_init", C.c_void_p), ("n_synapses", C.c_int64), ("syn_src", C.c_void_p),
        ("syn_tar", C.c_void_p), ("syn_weight", C.c_void_p), ("syn_delay", C.c_void_p),
        ("syn_plastic", C.c_void_p), ("lifconst", C.c_float * 30), ("stdpconst", C.c_float * 6),
        ("stdp", C.c_int32), ("mode", C.c_int32), ("seed", C.c_uint64), ("device", C.c_int32),
        ("raster_steps", C.c_int64), ("raster_ids", C.c_int64), ("id_offset", C.c_int32),
    ]


class FixedInDegreeDesc(C.Structure):
    _fields_ = [
        ("n_pops", C.c_int32), ("pop_start", C.c_void_p), ("pop_num", C.c_void_p),
        ("pop_type", C.c_void_p), ("n_proj", C.c_int32), ("pr_src", C.c_void_p),
        ("pr_tar", C.c_void_p), ("pr_k", C.c_void_p), ("pr_w", C.c_void_p),
        ("pr_dmin", C.c_void_p), ("pr_dmax", C.c_void_p), ("rate", C.c_void_p),
        ("v_init", C.c_void_p), ("lifconst", C.c_float * 30), ("conn_seed", C.c_uint64),
        ("seed", C.c_uint64), ("mode", C.c_int32), ("device", C.c_int32),
        ("raster_steps", C.c_int64), ("raster_ids", C.c_int64), ("id_offset", C.c_int32),
        ("proj_offset", C.c_int32),
    ]


class GenProj(C.Structure):
    _fields_ = [
        ("src", C.c_int32), ("tar", C.c_int32), ("rule", C.c_int32), ("prob", C.c_float), ("k", C.c_int32),
        ("conn_seed", C.c_uint64), ("weight", C.c_float), ("delay", C.c_int32), ("delay_max", C.c_int32),
        ("weights", C.c_void_p), ("delays", C.c_void_p), ("plastic", C.c_int32),
    ]


class GenDesc(C.Structure):
    _fields_ = [
        ("n_pops", C.c_int32), ("pop_num", C.c_void_p), ("pop_type", C.c_void_p), ("n_proj", C.c_int32),
        ("proj", C.c_void_p), ("mt_state", C.c_uint32 * 624), ("mt_state_out", C.c_void_p),
        ("rate", C.c_void_p), ("v_init", C.c_void_p), ("lifconst", C.c_float * 30), ("stdpconst", C.c_float * 6),
        ("stdp", C.c_int32), ("mode", C.c_int32), ("seed", C.c_uint64), ("device", C.c_int32),
        ("raster_steps", C.c_int64), ("raster_ids", C.c_int64),
    ]


def mt19937_seed_words(seed):
    """The 624 words of MT19937 seeded with `seed` (Matsumoto and Nishimura's
    initialisation, as std::mt19937(seed) does), in the order mgc_gen_desc
    takes them."""
    x = [int(seed) & 0xFFFFFFFF]
    for k in range(1, 624):
        x.append((1812433253 * (x[-1] ^ (x[-1] >> 30)) + k) & 0xFFFFFFFF)
    return x


class TuneReport(C.Structure):
    _fields_ = [
        ("trials", C.c_int32), ("chunk_len", C.c_int32), ("blocks_per_sm", C.c_int32),
        ("persistent", C.c_int32), ("window", C.c_int32), ("pull_min", C.c_int32),
        ("ms_per_step", C.c_double), ("default_ms_per_step", C.c_double), ("steps", C.c_int64),
    ]


class SchedStats(C.Structure):
    _fields_ = [
        ("mode", C.c_int32), ("trained", C.c_int32), ("groups", C.c_int64), ("misses", C.c_int64),
        ("variant_groups", C.c_int64 * 2), ("mean_abs_log_err", C.c_double), ("threshold", C.c_double),
        ("hi_variant", C.c_int32), ("static_variant", C.c_int32), ("recorded_groups", C.c_int32),
        ("reserved", C.c_int32),
    ]


class Info(C.Structure):
    _fields_ = [
        ("n_neurons", C.c_int32), ("ring_len", C.c_int32), ("min_delay", C.c_int32),
        ("max_delay", C.c_int32), ("n_synapses", C.c_int64), ("step", C.c_int64),
        ("events", C.c_int64), ("mode", C.c_int32), ("graph_steps", C.c_int32),
        ("device_bytes", C.c_int64), ("persistent", C.c_int32), ("first_neuron", C.c_int32),
        ("total_neurons", C.c_int32), ("window", C.c_int32), ("accumulation", C.c_int32),
        ("fx_shift", C.c_int32),
    ]


_lib = None


def lib():
    """Load the in-tree CUDA library; raises when it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build the CUDA extension first "
            "(python -c 'import __graft_entry__ as g; g.build()')")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
    L.mgc_create.argtypes = [C.POINTER(NetDesc), C.POINTER(vp)]
    L.mgc_create_fixed_indegree.argtypes = [C.POINTER(FixedInDegreeDesc), C.POINTER(vp)]
    L.mgc_create_batch.argtypes = [C.POINTER(FixedInDegreeDesc), i32, C.POINTER(vp)]
    L.mgc_create_partition.argtypes = [C.POINTER(NetDesc), i32, i32, C.POINTER(vp)]
    L.mgc_create_fixed_indegree_partition.argtypes = [C.POINTER(FixedInDegreeDesc), i32, i32, C.POINTER(vp)]
    L.mgc_part_export.argtypes = [vp, i32, vp, vp, i64, C.POINTER(i64)]
    L.mgc_part_import.argtypes = [vp, i32, i32, i32, vp, vp, i64]
    L.mgc_fault_inject_alloc.argtypes = [i64]
    L.mgc_partition_stats.argtypes = [vp, vp, i32, C.POINTER(i64), vp, vp, vp, vp]
    L.mgc_partition_stats.restype = C.c_int
    L.mgc_raster_stage.argtypes = [vp]
    L.mgc_raster_collect.argtypes = [vp, vp, vp, i64, vp, i64, vp, vp]
    L.mgc_raster_stage.restype = C.c_int
    L.mgc_raster_collect.restype = C.c_int
    L.mgc_part_export_dev.argtypes = [vp, i32, vp, i64]
    L.mgc_part_import_dev.argtypes = [vp, i32, i32, i32, vp, i64]
    L.mgc_part_export_dev.restype = C.c_int
    L.mgc_part_import_dev.restype = C.c_int
    L.mgc_selftest_wait_timeout.argtypes = [i32, i32, C.POINTER(i32), C.POINTER(C.c_double)]
    for name in ("mgc_create_partition", "mgc_create_fixed_indegree_partition", "mgc_part_export",
                 "mgc_part_import", "mgc_fault_inject_alloc", "mgc_selftest_wait_timeout"):
        getattr(L, name).restype = C.c_int
    L.mgc_run.argtypes = [vp, i64]
    L.mgc_sync.argtypes = [vp]
    L.mgc_set_rates.argtypes = [vp, vp, i32]
    L.mgc_read_raster.argtypes = [vp, vp, vp, i64, vp, i64, vp, vp]
    L.mgc_read_state.argtypes = [vp] * 7
    L.mgc_read_weights.argtypes = [vp, vp]
    L.mgc_export_csr.argtypes = [vp] * 5
    L.mgc_get_info.argtypes = [vp, C.POINTER(Info)]
    L.mgc_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.mgc_profile_steps.argtypes = [vp, i64, vp]
    L.mgc_effective_steps.argtypes = [i64, i32]
    L.mgc_effective_steps.restype = i64
    L.mgc_destroy.argtypes = [vp]
    L.mgc_destroy.restype = None
    L.mgc_last_error.restype = C.c_char_p
    L.mgc_kernel_launches.argtypes = [vp]
    L.mgc_kernel_launches.restype = i64
    L.mgc_row_offsets_static.argtypes = [vp, i64, i32, vp, vp]
    L.mgc_row_offsets_static.restype = C.c_int
    L.mgc_measure_scatter.argtypes = [i32, i64, i32, i32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.mgc_measure_scatter.restype = C.c_int
    L.mgc_autotune.argtypes = [vp, i64, C.POINTER(TuneReport)]
    L.mgc_autotune.restype = C.c_int
    L.mgc_autotune_rewind.argtypes = [vp, i64, C.POINTER(TuneReport)]
    L.mgc_autotune_rewind.restype = C.c_int
    L.mgc_set_persistent.argtypes = [vp, i32]
    L.mgc_set_persistent.restype = C.c_int
    L.mgc_set_pull.argtypes = [vp, i32]
    L.mgc_set_pull.restype = C.c_int
    L.mgc_set_window.argtypes = [vp, i32]
    L.mgc_set_window.restype = C.c_int
    L.mgc_create_generated.argtypes = [C.POINTER(GenDesc), C.POINTER(vp)]
    L.mgc_create_generated.restype = C.c_int
    L.mgc_gen_count.argtypes = [C.POINTER(GenDesc), i32]
    L.mgc_gen_count.restype = i64
    L.mgc_set_accumulation.argtypes = [vp, i32]
    L.mgc_set_accumulation.restype = C.c_int
    L.mgc_checkpoint_size.argtypes = [vp, C.POINTER(i64)]
    L.mgc_checkpoint_save.argtypes = [vp, vp, i64]
    L.mgc_checkpoint_load.argtypes = [vp, vp, i64]
    for name in ("mgc_checkpoint_size", "mgc_checkpoint_save", "mgc_checkpoint_load"):
        getattr(L, name).restype = C.c_int
    L.mgc_sched_set_mode.argtypes = [vp, i32]
    L.mgc_sched_set_threshold.argtypes = [vp, C.c_double, i32]
    L.mgc_sched_calibrate.argtypes = [vp, i32, C.POINTER(C.c_double)]
    L.mgc_sched_collect.argtypes = [vp, i32, i32]
    L.mgc_sched_train.argtypes = [vp, i32, C.c_float, C.c_uint64, C.POINTER(C.c_float)]
    L.mgc_sched_report.argtypes = [vp, C.POINTER(SchedStats), i32]
    L.mgc_mlp_gradient.argtypes = [i32, vp, vp, vp, i32, vp, vp]
    for name in ("mgc_sched_set_mode", "mgc_sched_set_threshold", "mgc_sched_calibrate", "mgc_sched_collect",
                 "mgc_sched_train", "mgc_sched_report", "mgc_mlp_gradient"):
        getattr(L, name).restype = C.c_int
    for name in ("mgc_create", "mgc_create_fixed_indegree", "mgc_create_batch", "mgc_run", "mgc_sync", "mgc_set_rates",
                 "mgc_read_raster", "mgc_read_state", "mgc_read_weights", "mgc_export_csr",
                 "mgc_get_info", "mgc_get_stream", "mgc_profile_steps"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(status):
    if status != MGC_OK:
        raise MgcError(status, lib().mgc_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def measure_scatter(device=0, n_events=100_000_000, n_targets=1 << 20, reps=3):
    """(reductions/s, read bytes/s): the delivery ceilings of this device."""
    red, rd = C.c_double(), C.c_double()
    check(lib().mgc_measure_scatter(int(device), int(n_events), int(n_targets), int(reps), C.byref(red),
                                    C.byref(rd)))
    return red.value, rd.value


def mlp_gradient(params, x, y, device=0):
    """(loss, grad) of the scheduler MLP at `params` on samples x [n][20],
    targets y [n][5], computed by the library's training kernel."""
    p = np.ascontiguousarray(params, np.float32)
    xs = np.ascontiguousarray(x, np.float32)
    ys = np.ascontiguousarray(y, np.float32)
    g = np.zeros(MLP_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    check(lib().mgc_mlp_gradient(int(device), _ptr(p), _ptr(xs), _ptr(ys), int(xs.shape[0]), _ptr(g), _ptr(loss)))
    return float(loss[0]), g


def fault_inject_alloc(n):
    """The n-th device allocation from now fails as out of memory (0: off)."""
    check(lib().mgc_fault_inject_alloc(int(n)))


def selftest_wait_timeout(which, device=0):
    """(status bits, ms): a step-group wait (0 phase wait, 1 grid barrier)
    run against a counter nothing advances; 4 = it gave up."""
    st, ms = C.c_int32(), C.c_double()
    check(lib().mgc_selftest_wait_timeout(int(device), int(which), C.byref(st), C.byref(ms)))
    return st.value, ms.value


def effective_steps(steps, min_delay):
    return int(lib().mgc_effective_steps(int(steps), int(min_delay)))


class Simulator:
    """One simulation handle of the CUDA core (an MGSimulator for npart=1)."""

    def __init__(self, handle, n, S, keep=()):
        self._h = C.c_void_p(handle)
        self.n = n
        self.S = S
        self.first = 0     # partition handles: whole-network id of neuron 0
        self.n_src = n     # CSR rows (the whole network's neurons for a partition)
        self._keep = keep

    # ---- construction ---------------------------------------------------
    @classmethod
    def from_arrays(cls, n, type_, src, tar, weight, delay_steps, lifconst, stdpconst=None,
                    rate=None, v_init=None, stdp=False, plastic=None, seed=1, device=0,
                    mode=MODE_AUTO, raster_steps=0, raster_ids=0, part=None):
        """part: (first, count) builds the partition of neurons [first, first+count)
        of this network (mgc_create_partition)."""
        L = lib()
        arrs = dict(
            type=np.ascontiguousarray(type_, np.int8),
            rate=None if rate is None else np.ascontiguousarray(rate, np.float32),
            v_init=None if v_init is None else np.ascontiguousarray(v_init, np.float32),
            src=np.ascontiguousarray(src, np.int32), tar=np.ascontiguousarray(tar, np.int32),
            weight=np.ascontiguousarray(weight, np.float32),
            delay=np.ascontiguousarray(delay_steps, np.int32),
            plastic=None if plastic is None else np.ascontiguousarray(plastic, np.uint8),
        )
        d = NetDesc()
        d.n_neurons = int(n)
        d.type, d.rate, d.v_init = _ptr(arrs["type"]), _ptr(arrs["rate"]), _ptr(arrs["v_init"])
        d.n_synapses = len(arrs["src"])
        d.syn_src, d.syn_tar = _ptr(arrs["src"]), _ptr(arrs["tar"])
        d.syn_weight, d.syn_delay = _ptr(arrs["weight"]), _ptr(arrs["delay"])
        d.syn_plastic = _ptr(arrs["plastic"])
        d.lifconst[:] = [float(x) for x in np.asarray(lifconst, np.float32)]
        sc = np.asarray(stdpconst if stdpconst is not None else [0.1, -0.01, 17, 34, 40, 0], np.float32)
        d.stdpconst[:] = [float(x) for x in sc]
        d.stdp, d.mode, d.seed, d.device = int(bool(stdp)), int(mode), int(seed), int(device)
        d.raster_steps, d.raster_ids = int(raster_steps), int(raster_ids)
        h = C.c_void_p()
        if part is not None:
            check(L.mgc_create_partition(C.byref(d), int(part[0]), int(part[1]), C.byref(h)))
            return cls._partition(h.value)
        check(L.mgc_create(C.byref(d), C.byref(h)))
        return cls(h.value, int(n), d.n_synapses)

    @classmethod
    def _partition(cls, handle):
        s = cls(handle, 0, 0)
        i = s.info()
        s.n, s.S = i["n_neurons"], i["n_synapses"]
        s.first, s.n_src = i["first_neuron"], i["total_neurons"]
        return s

    @staticmethod
    def _block_desc(pops, projs, lifconst, rate=None, v_init=None, conn_seed=1, seed=1, device=0,
                    mode=MODE_AUTO, raster_steps=0, raster_ids=0, id_offset=0, proj_offset=0):
        """A FixedInDegreeDesc plus the arrays it points into (keep both alive)."""
        P = np.asarray(pops, np.int64).reshape(-1, 3)
        R = list(projs)
        a = dict(
            ps=np.ascontiguousarray(P[:, 0], np.int32), pn=np.ascontiguousarray(P[:, 1], np.int32),
            pt=np.ascontiguousarray(P[:, 2], np.int32),
            rs=np.array([r[0] for r in R], np.int32), rt=np.array([r[1] for r in R], np.int32),
            rk=np.array([r[2] for r in R], np.int32), rw=np.array([r[3] for r in R], np.float32),
            rd0=np.array([r[4] for r in R], np.int32), rd1=np.array([r[5] for r in R], np.int32),
            rate=None if rate is None else np.ascontiguousarray(rate, np.float32),
            v0=None if v_init is None else np.ascontiguousarray(v_init, np.float32),
        )
        d = FixedInDegreeDesc()
        d.n_pops = len(P)
        d.pop_start, d.pop_num, d.pop_type = _ptr(a["ps"]), _ptr(a["pn"]), _ptr(a["pt"])
        d.n_proj = len(R)
        d.pr_src, d.pr_tar, d.pr_k, d.pr_w = _ptr(a["rs"]), _ptr(a["rt"]), _ptr(a["rk"]), _ptr(a["rw"])
        d.pr_dmin, d.pr_dmax = _ptr(a["rd0"]), _ptr(a["rd1"])
        d.rate, d.v_init = _ptr(a["rate"]), _ptr(a["v0"])
        d.lifconst[:] = [float(x) for x in np.asarray(lifconst, np.float32)]
        d.conn_seed, d.seed, d.mode, d.device = int(conn_seed), int(seed), int(mode), int(device)
        d.raster_steps, d.raster_ids = int(raster_steps), int(raster_ids)
        d.id_offset, d.proj_offset = int(id_offset), int(proj_offset)
        n = int((P[:, 0] + P[:, 1]).max())
        S = int(sum(int(P[r[1], 1]) * int(r[2]) for r in R))
        return d, a, n, S

    @classmethod
    def fixed_indegree(cls, pops, projs, lifconst, **kw):
        """pops: list of (start, num, type); projs: (src_pop, tar_pop, k, w, dmin, dmax);
        keywords: rate, v_init, conn_seed, seed, device, mode, raster_steps, raster_ids,
        id_offset, proj_offset; part=(first, count) builds that partition of the
        network (mgc_create_fixed_indegree_partition)."""
        part = kw.pop("part", None)
        d, keep, n, S = cls._block_desc(pops, projs, lifconst, **kw)
        h = C.c_void_p()
        if part is not None:
            check(lib().mgc_create_fixed_indegree_partition(C.byref(d), int(part[0]), int(part[1]), C.byref(h)))
            return cls._partition(h.value)
        check(lib().mgc_create_fixed_indegree(C.byref(d), C.byref(h)))
        return cls(h.value, n, S)

    @classmethod
    def generated(cls, pops, projs, lifconst, mt_seed=None, mt_state=None, stdpconst=None, rate=None,
                  v_init=None, stdp=False, seed=1, device=0, mode=MODE_AUTO, raster_steps=0, raster_ids=0,
                  state_out=None):
        """The network NetGen's rules make, generated on the device
        (mgc_create_generated).  pops: list of (num, type); projs: dicts with
        src, tar, rule and prob / k, conn_seed, weight or weights (array in
        synapse order), delay (steps) or delays (array), delay_max, plastic.
        mt_seed seeds NetGen's mt19937 (or mt_state gives its 624 words);
        state_out: a list that receives the generator's words afterwards."""
        keep = []
        P = list(pops)
        pn = np.array([p[0] for p in P], np.int32)
        pt = np.array([p[1] for p in P], np.int8)
        arr = (GenProj * max(1, len(projs)))()
        for i, r in enumerate(projs):
            g = arr[i]
            g.src, g.tar, g.rule = int(r["src"]), int(r["tar"]), int(r["rule"])
            g.prob, g.k, g.conn_seed = float(r.get("prob", 0.0)), int(r.get("k", 0)), int(r.get("conn_seed", 1))
            g.weight, g.delay = float(r.get("weight", 0.0)), int(r.get("delay", 1))
            g.delay_max, g.plastic = int(r.get("delay_max", r.get("delay", 1))), int(bool(r.get("plastic", 0)))
            if r.get("weights") is not None:
                w = np.ascontiguousarray(r["weights"], np.float32)
                keep.append(w)
                g.weights = _ptr(w)
            if r.get("delays") is not None:
                dl = np.ascontiguousarray(r["delays"], np.int32)
                keep.append(dl)
                g.delays = _ptr(dl)
        d = GenDesc()
        d.n_pops, d.pop_num, d.pop_type = len(P), _ptr(pn), _ptr(pt)
        d.n_proj, d.proj = len(projs), C.cast(arr, C.c_void_p)
        words = mt_state if mt_state is not None else mt19937_seed_words(5489 if mt_seed is None else mt_seed)
        d.mt_state[:] = [int(x) & 0xFFFFFFFF for x in words]
        out_words = (C.c_uint32 * 624)()
        d.mt_state_out = C.cast(out_words, C.c_void_p)
        rate_a = None if rate is None else np.ascontiguousarray(rate, np.float32)
        v0_a = None if v_init is None else np.ascontiguousarray(v_init, np.float32)
        d.rate, d.v_init = _ptr(rate_a), _ptr(v0_a)
        d.lifconst[:] = [float(x) for x in np.asarray(lifconst, np.float32)]
        sc = np.asarray(stdpconst if stdpconst is not None else [0.1, -0.01, 17, 34, 40, 0], np.float32)
        d.stdpconst[:] = [float(x) for x in sc]
        d.stdp, d.mode, d.seed, d.device = int(bool(stdp)), int(mode), int(seed), int(device)
        d.raster_steps, d.raster_ids = int(raster_steps), int(raster_ids)
        counts = [int(lib().mgc_gen_count(C.byref(d), i)) for i in range(len(projs))]
        for i, r in enumerate(projs):
            for key in ("weights", "delays"):
                if r.get(key) is not None and len(r[key]) != counts[i]:
                    raise ValueError(f"projection {i}: {key} holds {len(r[key])}, the rule makes {counts[i]}")
        h = C.c_void_p()
        check(lib().mgc_create_generated(C.byref(d), C.byref(h)))
        if state_out is not None:
            state_out[:] = list(out_words)
        return cls(h.value, int(pn.sum()), int(sum(counts)))

    @classmethod
    def batch(cls, blocks, lifconst, seed=1, device=0, mode=MODE_AUTO, raster_steps=0, raster_ids=0):
        """Independent networks side by side in one handle.  blocks: dicts with
        pops, projs and optional rate, v_init, conn_seed (populations relative
        to the block)."""
        descs, keep, n, S = [], [], 0, 0
        for b in blocks:
            d, a, nb, sb = cls._block_desc(b["pops"], b["projs"], lifconst, rate=b.get("rate"),
                                           v_init=b.get("v_init"), conn_seed=b.get("conn_seed", 1),
                                           seed=seed, device=device, mode=mode,
                                           raster_steps=raster_steps, raster_ids=raster_ids)
            descs.append(d)
            keep.append(a)
            n += nb
            S += sb
        arr = (FixedInDegreeDesc * len(descs))(*descs)
        h = C.c_void_p()
        check(lib().mgc_create_batch(arr, len(descs), C.byref(h)))
        return cls(h.value, n, S)

    # ---- stepping -------------------------------------------------------
    def run(self, steps):
        check(lib().mgc_run(self._h, int(steps)))

    def sync(self):
        check(lib().mgc_sync(self._h))

    def set_rates(self, rate):
        r = np.ascontiguousarray(rate, np.float32)
        check(lib().mgc_set_rates(self._h, _ptr(r), self.n))
        self.sync()  # the host array may be pageable and temporary

    @property
    def stream(self):
        s = C.c_void_p()
        check(lib().mgc_get_stream(self._h, C.byref(s)))
        return s.value or 0

    # ---- readout --------------------------------------------------------
    def read_raster(self, max_steps=1 << 20, max_ids=None):
        """(first step, spikes per step, ids per step in ascending order)."""
        if max_ids is None:
            max_ids = max(1 << 20, max(1, self.n) * 64)   # the device raster's default capacity
        counts = np.empty(max_steps, np.int64)
        ids = np.empty(max_ids, np.int32)
        first, ns, ni = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().mgc_read_raster(self._h, C.byref(first), _ptr(counts), max_steps, _ptr(ids),
                                    max_ids, C.byref(ns), C.byref(ni)))
        # copies: the (mostly untouched) capacity buffers are not kept alive
        return first.value, counts[:ns.value].copy(), ids[:ni.value].copy()

    def stage_raster(self):
        """Enqueues a device copy of the raster so far and starts a new one
        (mgc_raster_stage); no host wait."""
        check(lib().mgc_raster_stage(self._h))

    def collect_raster(self, max_steps=1 << 20, max_ids=None):
        """The oldest staged raster, as read_raster returns one."""
        if max_ids is None:
            max_ids = max(1 << 20, max(1, self.n) * 64)   # the device raster's default capacity
        counts = np.empty(max_steps, np.int64)
        ids = np.empty(max_ids, np.int32)
        first, ns, ni = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().mgc_raster_collect(self._h, C.byref(first), _ptr(counts), max_steps, _ptr(ids),
                                       max_ids, C.byref(ns), C.byref(ni)))
        return first.value, counts[:ns.value].copy(), ids[:ni.value].copy()

    def state(self):
        n = self.n
        out = {k: np.zeros(n, np.float32) for k in ("V", "Iexc", "Iinh")}
        for k in ("refrac", "last_fired", "fire_cnt"):
            out[k] = np.zeros(n, np.int32)
        check(lib().mgc_read_state(self._h, _ptr(out["V"]), _ptr(out["Iexc"]), _ptr(out["Iinh"]),
                                   _ptr(out["refrac"]), _ptr(out["last_fired"]), _ptr(out["fire_cnt"])))
        return out

    def weights(self):
        w = np.zeros(self.S, np.float32)
        check(lib().mgc_read_weights(self._h, _ptr(w)))
        return w

    def export_csr(self):
        rp = np.zeros(self.n_src + 1, np.int64)
        t = np.zeros(self.S, np.int32)
        w = np.zeros(self.S, np.float32)
        d = np.zeros(self.S, np.int32)
        check(lib().mgc_export_csr(self._h, _ptr(rp), _ptr(t), _ptr(w), _ptr(d)))
        return rp, t, w, d

    def partition_stats(self, part, nparts):
        """Cut and balance of a neuron partition over this handle's synapses
        (mgc_partition_stats): dict with cut and the per-zone arrays."""
        p = np.ascontiguousarray(part, np.int32)
        out = {k: np.zeros(int(nparts), np.int64) for k in ("zone_neurons", "zone_syn", "zone_out", "zone_in")}
        cut = C.c_int64()
        check(lib().mgc_partition_stats(self._h, _ptr(p), int(nparts), C.byref(cut), _ptr(out["zone_neurons"]),
                                        _ptr(out["zone_syn"]), _ptr(out["zone_out"]), _ptr(out["zone_in"])))
        out["cut"] = int(cut.value)
        return out

    # ---- partitions -------------------------------------------------------
    def part_export(self, count, ids):
        """Spike ids of the `count` steps run since the last import, written into
        `ids` (a contiguous int32 device tensor of the handle's device, or None
        for the counts only); returns (counts per step, total)."""
        counts = np.zeros(max(1, int(count)), np.int32)
        total = C.c_int64()
        ptr, cap = (C.c_void_p(ids.data_ptr()), ids.numel()) if ids is not None else (None, 0)
        check(lib().mgc_part_export(self._h, int(count), _ptr(counts), ptr, int(cap), C.byref(total)))
        return counts[:int(count)], int(total.value)

    def part_import(self, count, self_rank, counts, ids, stride):
        """Appends the other partitions' spikes: counts [nranks][count] (host),
        partition r's ids at ids[r * stride:] (contiguous int32 device tensor)."""
        c = np.ascontiguousarray(counts, np.int32)
        check(lib().mgc_part_import(self._h, int(count), int(c.shape[0]), int(self_rank), _ptr(c),
                                    C.c_void_p(ids.data_ptr()) if ids is not None else None, int(stride)))

    def part_export_dev(self, count, buf, cap):
        """Enqueues the window's export into the device tensor buf (count + cap
        int32: counts, then ids); no host synchronisation."""
        check(lib().mgc_part_export_dev(self._h, int(count), C.c_void_p(buf.data_ptr()), int(cap)))

    def part_import_dev(self, count, self_rank, nranks, bufs, cap):
        """Enqueues the import from the device tensor bufs (nranks blocks of
        count + cap int32, as an all-gather of the export buffers lays them)."""
        ptr = C.c_void_p(bufs.data_ptr()) if bufs is not None else None
        check(lib().mgc_part_import_dev(self._h, int(count), int(nranks), int(self_rank), ptr, int(cap)))

    def autotune(self, steps_per_trial=640, rewind=False):
        """Times the launch configurations and keeps the fastest; the trial
        steps advance the simulation (report["steps"] of them), or with
        rewind=True are undone through a checkpoint, so that the simulation
        continues from where it was (mgc_autotune_rewind; read the raster
        first)."""
        r = TuneReport()
        fn = lib().mgc_autotune_rewind if rewind else lib().mgc_autotune
        check(fn(self._h, int(steps_per_trial), C.byref(r)))
        return {k: getattr(r, k) for k, _ in TuneReport._fields_ if k != "reserved"}

    # ---- step scheduler ---------------------------------------------------
    def sched_mode(self, mode):
        check(lib().mgc_sched_set_mode(self._h, int(mode)))

    def sched_threshold(self, threshold, hi_variant=1):
        check(lib().mgc_sched_set_threshold(self._h, float(threshold), int(hi_variant)))

    def sched_calibrate(self, groups=16):
        t = C.c_double()
        check(lib().mgc_sched_calibrate(self._h, int(groups), C.byref(t)))
        return t.value

    def sched_collect(self, on=True, reset=False):
        check(lib().mgc_sched_collect(self._h, int(bool(on)), int(bool(reset))))

    def sched_train(self, epochs=200, lr=3e-3, seed=1):
        loss = C.c_float()
        check(lib().mgc_sched_train(self._h, int(epochs), float(lr), int(seed), C.byref(loss)))
        return loss.value

    def sched_report(self, reset=False):
        r = SchedStats()
        check(lib().mgc_sched_report(self._h, C.byref(r), int(bool(reset))))
        d = {k: getattr(r, k) for k, _ in SchedStats._fields_ if k != "reserved"}
        d["variant_groups"] = [r.variant_groups[0], r.variant_groups[1]]
        return d

    def checkpoint(self):
        """The simulation state as bytes (mgc_checkpoint_save)."""
        n = C.c_int64()
        check(lib().mgc_checkpoint_size(self._h, C.byref(n)))
        buf = np.empty(n.value, np.uint8)
        check(lib().mgc_checkpoint_save(self._h, _ptr(buf), n.value))
        return buf.tobytes()

    def restore(self, data):
        """Continues from a checkpoint of the same network (mgc_checkpoint_load)."""
        buf = np.frombuffer(data, np.uint8)
        check(lib().mgc_checkpoint_load(self._h, _ptr(buf), buf.size))

    def set_persistent(self, mode=1):
        """0: CUDA graphs of single-step kernels; 1: cooperative step groups
        with a grid barrier per step; 2: pipelined step groups; 3: windowed
        step groups (set_window)."""
        check(lib().mgc_set_persistent(self._h, int(mode)))

    def set_accumulation(self, mode):
        """ACC_FLOAT (fp32 additions) or ACC_FIXED (order-independent 64-bit
        fixed point), before the first step (mgc_set_accumulation)."""
        check(lib().mgc_set_accumulation(self._h, int(mode)))

    def set_pull(self, min_pairs):
        """Pull steps of the windowed group: a step whose arrivals come from at
        least min_pairs (spike, delay) pairs is delivered by pull (mgc_set_pull);
        0 turns them off.  Results are unchanged."""
        check(lib().mgc_set_pull(self._h, int(min_pairs)))

    def set_window(self, steps):
        """Steps per window of the windowed step group (1..min(8, min delay))."""
        check(lib().mgc_set_window(self._h, int(steps)))

    def profile(self, steps):
        """Milliseconds spent in (neuron update, event push, STDP) over `steps`
        steps, measured with CUDA events recorded between the kernels (the
        steps and events are replayed as CUDA graphs of 64 steps)."""
        ms = np.zeros(3, np.float32)
        check(lib().mgc_profile_steps(self._h, int(steps), _ptr(ms)))
        return [float(x) for x in ms]

    def info(self):
        i = Info()
        check(lib().mgc_get_info(self._h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in Info._fields_}

    @property
    def kernel_launches(self):
        return int(lib().mgc_kernel_launches(self._h))

    def close(self):
        if self._h:
            lib().mgc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
