/*
 * mgc.h — C ABI of the mgbrain_b200 single-GPU simulation core.
 *
 * Plain pointers and sizes only; every call returns an mgc_status (0 = ok)
 * and never exits the process.  One handle owns its device memory and its
 * CUDA stream; handles share no global state, so several can live on one
 * device.  Calls on one handle must not race each other.
 *
 * Each entry point names the reference interface it replaces
 * (RAICLab-SNNGroup/MGBrain, file:line).
 */
#ifndef MGC_H
#define MGC_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum mgc_status {
    MGC_OK = 0,
    MGC_ERR_INVALID = 1,   /* bad argument or network description */
    MGC_ERR_CUDA = 2,      /* CUDA runtime error (mgc_last_error has the text) */
    MGC_ERR_NOMEM = 3,     /* device or host allocation failed */
    MGC_ERR_OVERFLOW = 4,  /* raster buffer overflowed; returned data is truncated */
    MGC_ERR_NODEVICE = 5   /* no CUDA device / extension built for another GPU */
} mgc_status;

/* NeuronType values, src/macro.h:40-48. */
enum { MGC_RAW = 0, MGC_LIF0 = 1, MGC_POISSON = 2, MGC_LIF = 3, MGC_LIFE = 4, MGC_LIFB = 5 };

/* Event delivery method.  Both give every neuron the same input sum. */
enum {
    MGC_MODE_AUTO = 0,     /* DEFERRED when the network allows it, else PUSH */
    MGC_MODE_PUSH = 1,     /* push from spiking rows into the M-slot delay ring at
                              the emission step (mgcore.cu:271-305); required
                              when weights are plastic */
    MGC_MODE_DEFERRED = 2, /* rows bucketed by delay; at step s the spikes of
                              step s-d push their delay-d bucket into one
                              L2-resident accumulator per neuron (static
                              weights, < 2^32 synapses, <= 2048 delay values) */
    MGC_MODE_PULL = 3      /* one pass per target over its incoming synapses
                              each step, adding spiking sources in a fixed
                              order (deterministic for any weights) with STDP
                              fused in; cost grows with all synapses, so AUTO
                              never takes it (PUSH with STDP fused and
                              fixed-point sums is deterministic too, and
                              faster on the measured plastic networks);
                              explicit networks only */
};

typedef struct mgc_sim mgc_sim;

/* Network handed over as the reference's Network holds it
 * (src/model/network.h:50-68) after build_multinet's delay quantisation
 * (src/simulator/mgsim/adj/mgsim.cpp:49): neurons in id order, synapses in
 * list order.  All arrays are host memory and are copied; the caller may
 * free them after mgc_create returns. */
typedef struct mgc_net_desc {
    int32_t n_neurons;
    const int8_t* type;        /* [n] NeuronType */
    const float* rate;         /* [n] POISSON per-step probability, or NULL (0) */
    const float* v_init;       /* [n] initial V, or NULL (lifconst[1] for all) */
    int64_t n_synapses;
    const int32_t* syn_src;    /* [S] */
    const int32_t* syn_tar;    /* [S] */
    const float* syn_weight;   /* [S] */
    const int32_t* syn_delay;  /* [S] delay in steps, >= 1 */
    const uint8_t* syn_plastic;/* [S] or NULL: every synapse plastic when stdp */
    float lifconst[30];        /* LIFECONSTS, mgcore.cu:32-63 */
    float stdpconst[6];        /* STDPCONSTS, mgcore.cu:73-80 */
    int32_t stdp;              /* Config::STDP */
    int32_t mode;              /* MGC_MODE_* */
    uint64_t seed;             /* key of the POISSON draws */
    int32_t device;            /* CUDA device ordinal */
    int64_t raster_steps;      /* steps the raster holds between reads (0: default) */
    int64_t raster_ids;        /* spike ids it holds between reads (0: default, <0: off) */
    int32_t id_offset;         /* added to neuron ids in the POISSON draws (a network
                                  simulated as part of a larger one draws as there) */
} mgc_net_desc;

/* Procedural fixed in-degree network built on the device.  Population p
 * occupies neuron ids [pop_start[p], pop_start[p]+pop_num[p]).  Projection
 * r gives every neuron of pop pr_tar[r] exactly pr_k[r] synapses whose
 * sources are drawn uniformly, with replacement, from pop pr_src[r], with
 * weight pr_w[r] and delay uniform in [pr_dmin[r], pr_dmax[r]] steps,
 * from Philox4x32-10 keyed by conn_seed with counter (target + id_offset, k,
 * r + proj_offset): a block of a larger network given the offsets it has
 * there generates the same synapses and POISSON draws as inside it. */
typedef struct mgc_fixed_indegree_desc {
    int32_t n_pops;
    const int32_t* pop_start;
    const int32_t* pop_num;
    const int32_t* pop_type;
    int32_t n_proj;
    const int32_t* pr_src;
    const int32_t* pr_tar;
    const int32_t* pr_k;
    const float* pr_w;
    const int32_t* pr_dmin;
    const int32_t* pr_dmax;
    const float* rate;         /* [n] or NULL */
    const float* v_init;       /* [n] or NULL */
    float lifconst[30];
    uint64_t conn_seed;
    uint64_t seed;
    int32_t mode;
    int32_t device;
    int64_t raster_steps;
    int64_t raster_ids;
    int32_t id_offset;
    int32_t proj_offset;
} mgc_fixed_indegree_desc;

typedef struct mgc_info {
    int32_t n_neurons;
    int32_t ring_len;          /* M = max_delay + 1 (mgsim.cpp:71) */
    int32_t min_delay;         /* mgsim.cpp:51 */
    int32_t max_delay;
    int64_t n_synapses;
    int64_t step;              /* steps simulated so far */
    int64_t events;            /* synaptic events delivered so far */
    int32_t mode;
    int32_t graph_steps;       /* steps per captured CUDA graph */
    int64_t device_bytes;      /* device memory held by the handle */
    int32_t persistent;        /* steps run as step groups: 0 no (graphs), 1 barrier per step, 2 pipelined,
                                  3 windowed */
    int32_t first_neuron;      /* partition handles: whole-network id of neuron 0 (else 0) */
    int32_t total_neurons;     /* partition handles: neurons of the whole network (else n_neurons) */
    int32_t window;            /* steps per window of the windowed step group (0: minimum delay 1) */
    int32_t accumulation;      /* MGC_ACC_FLOAT or MGC_ACC_FIXED (mgc_set_accumulation) */
    int32_t fx_shift;          /* fixed-point accumulation: weights are added as rint(w * 2^fx_shift) */
} mgc_info;

/* How a neuron's input of one step is summed.  FLOAT: fp32 additions, as the
 * reference's atomicAdd does them (mgcore.cu:112-115); the sum of unequal
 * weights of one sign then depends on the order in which they land, which
 * the scattered reductions do not fix (nor do the reference's atomics), so
 * the last bits of V can differ from run to run.  FIXED: each weight is
 * added as the integer rint(w * 2^fx_shift) into a 64-bit accumulator, and
 * the neuron update converts the sum to fp32 once (round to nearest) and
 * scales it by 2^-fx_shift: the sum does not depend on the order, so every
 * run gives the same bits.  The builder picks fx_shift so that every weight
 * is an exact multiple of 2^-fx_shift while any neuron's sum of one step
 * still fits the integer (with plastic weights only the second); the input
 * is then the exact sum of the fp32 weights, rounded once.  A new handle
 * takes FIXED when some neuron receives unequal weights of one sign (or
 * weights are plastic) and the method is DEFERRED or PUSH, else FLOAT (with
 * one weight per sign, fp32 sums of the same value are the same in any
 * order, and equal the reference's bit for bit).  The PULL method always
 * adds in a fixed order in fp32.  FIXED doubles the accumulators' memory
 * (8 bytes per neuron and buffer). */
enum { MGC_ACC_FLOAT = 0, MGC_ACC_FIXED = 1 };

/* Replaces MGSimulator::MGSimulator(Network&, std::vector<int>&, int)
 * (src/simulator/mgsim/adj/mgsim.cpp:337-363) for npart=1: build_multinet
 * (mgsim.cpp:8-144), copy_subnet_gpu (mgnet.cpp:92-146), init_state
 * (mgcore.cu:665-669) and copy_consts_gpu (mgcore.cu:685-748). */
mgc_status mgc_create(const mgc_net_desc* desc, mgc_sim** out);

/* Device-side network generation for networks too large to list on the
 * host; no reference counterpart (netgen.cpp:39-229 is host-only and
 * cannot express a fixed in-degree). */
mgc_status mgc_create_fixed_indegree(const mgc_fixed_indegree_desc* desc, mgc_sim** out);

/* ---- Network generation on the device by NetGen's rules ------------------
 * The synapses NetGen::gen_net (src/model/netgen.cpp:39-229) would make,
 * generated on the device and turned into the CSR there: no host synapse
 * list (the reference's gen_net is an O(sn*tn) host loop that also keeps
 * about 90 bytes per synapse in host memory).  Populations occupy
 * consecutive ids in population order, as gen_net assigns them; projections
 * are generated in order, each synapse in the rule's order, so the synapse
 * list (mgc_read_weights order) is gen_net's.  Rules:
 *   MGC_RULE_PROB  the fixed-probability rule (netgen.cpp:169-186): pair k of
 *                  the row-major sn x tn pairs is taken, while fewer than
 *                  gen_num = round(float(sn*tn) * prob) are taken, when the
 *                  k-th output of NetGen's mt19937 modulo sn*tn is below
 *                  gen_num * 1.1; list slots left over are pair (0, 0).  The
 *                  candidate pairs are cut into stretches generated at once,
 *                  each from the generator jumped ahead to its start.
 *   MGC_RULE_ALL   every pair (m, n), row-major (ctype 1).
 *   MGC_RULE_ONE   pairs (k, k), k < sn (ctype 0).
 *   MGC_RULE_ALL_BUT_SELF  every pair with m != n, row-major (no reference
 *                  counterpart; Model::connect_all_but_self).
 *   MGC_RULE_FIXED_INDEGREE  k sources per target drawn as by
 *                  mgc_create_fixed_indegree with counter (target, draw,
 *                  projection index) (Model::connect_fixed_indegree).
 * Weights and delays: one value per projection, or (ranges, which NetGen
 * draws with glibc rand() in synapse order, netgen.cpp:19-38) host arrays
 * of the projection's synapses in order, drawn by the caller.  The shuffle
 * placement (Config::SHUFFLE_GEN) stays on the host. */
enum { MGC_RULE_PROB = 0, MGC_RULE_ALL = 1, MGC_RULE_ONE = 2, MGC_RULE_ALL_BUT_SELF = 3,
       MGC_RULE_FIXED_INDEGREE = 4 };

typedef struct mgc_gen_proj {
    int32_t src, tar;          /* population indices */
    int32_t rule;              /* MGC_RULE_* */
    float prob;                /* MGC_RULE_PROB: Projection::ctype */
    int32_t k;                 /* MGC_RULE_FIXED_INDEGREE: sources per target */
    uint64_t conn_seed;        /* MGC_RULE_FIXED_INDEGREE: key of its draws */
    float weight;              /* every synapse's weight when weights is NULL */
    int32_t delay;             /* delay in steps when delays is NULL (FIXED_INDEGREE: the least) */
    int32_t delay_max;         /* MGC_RULE_FIXED_INDEGREE: delays uniform in [delay, delay_max] */
    const float* weights;      /* host [mgc_gen_count] weights in synapse order, or NULL */
    const int32_t* delays;     /* host [mgc_gen_count] delays in steps, or NULL */
    int32_t plastic;           /* the projection's synapses learn (with stdp) */
} mgc_gen_proj;

typedef struct mgc_gen_desc {
    int32_t n_pops;
    const int32_t* pop_num;    /* [n_pops] neurons */
    const int8_t* pop_type;    /* [n_pops] NeuronType */
    int32_t n_proj;
    const mgc_gen_proj* proj;  /* [n_proj], in gen_net's order */
    uint32_t mt_state[624];    /* NetGen's mt19937 before the first projection, in logical
                                  order: the next 624 outputs are one twist of these words
                                  (a freshly seeded generator: its seeding words as they are) */
    uint32_t* mt_state_out;    /* [624] or NULL: the generator after the network, same order */
    const float* rate;         /* [n] or NULL */
    const float* v_init;       /* [n] or NULL */
    float lifconst[30];
    float stdpconst[6];
    int32_t stdp;
    int32_t mode;
    uint64_t seed;
    int32_t device;
    int64_t raster_steps;
    int64_t raster_ids;
} mgc_gen_desc;

/* Builds the network of `desc` on the device (see above); everything else
 * as mgc_create.  Fails with MGC_ERR_INVALID for more than 2^31-1 synapses. */
mgc_status mgc_create_generated(const mgc_gen_desc* desc, mgc_sim** out);

/* Synapses projection r of desc generates (the length of its weights and
 * delays arrays), or -1 for a bad projection. */
int64_t mgc_gen_count(const mgc_gen_desc* desc, int32_t r);

/* Many independent fixed in-degree networks advanced together in one
 * handle (a parameter sweep).  Block b's neurons occupy ids
 * [start_b, start_b + n_b), start_b = sizes of the blocks before it; its
 * populations are given relative to start_b.  Block b generates the
 * synapses it would generate alone with id_offset = start_b and
 * proj_offset = projections of the earlier blocks, and with the batch's
 * POISSON seed (blocks[0].seed) its raster equals that lone run's.  All
 * blocks share blocks[0]'s LIF constants, mode, device and raster sizes.
 * No reference counterpart (the reference simulates one network). */
mgc_status mgc_create_batch(const mgc_fixed_indegree_desc* blocks, int32_t n_blocks, mgc_sim** out);

/* Partitions: one network split into neuron ranges [first, first + count),
 * one handle per range, each on its own device (or several on one).  Replaces
 * MGSimulator(Network&, std::vector<int>& part, int npart) with npart > 1
 * (mgsim.cpp:337-363, build_multinet's per-partition split :8-144) and its
 * exchange: the reference's partitions push cross-partition events into
 * per-pair spike buffers and copy them between GPUs every min_delay/2 steps
 * (simulate_sparse, mgsim.cpp:794-848; trans_spikes_sparse /
 * recvs_spikes_sparse, mgcore.cu:470-646).  Here a partition holds the
 * synapses that TARGET its neurons, with every source of the network, and
 * the partitions exchange spike ids: after at most min_delay - 1 steps
 * (mgc_run refuses more), each exports the spike ids of those steps
 * (mgc_part_export), the caller gathers them across partitions (NCCL
 * all-gather, or any copy), and each imports the others' (mgc_part_import).
 * The union of the partitions' rasters and state equals the whole network's
 * run.  Static weights only (the deferred method), min_delay >= 2.  The
 * description is that of the whole network; ids in rasters, exports and
 * imports are whole-network ids; state and rates are the partition's
 * neurons.  Autotuning, profiling and scheduler calibration (which run steps
 * of their own) are refused on partition handles.  No reference counterpart
 * for the fixed in-degree form. */
mgc_status mgc_create_partition(const mgc_net_desc* desc, int32_t first, int32_t count, mgc_sim** out);
mgc_status mgc_create_fixed_indegree_partition(const mgc_fixed_indegree_desc* desc, int32_t first, int32_t count,
                                               mgc_sim** out);

/* Spike ids of the `count` steps run since the last import (count must
 * equal that number), oldest step first: counts[j] (host array) = spikes of
 * step j of the window, ids (device memory of the handle's device, or
 * mapped page-locked host memory; ids_cap entries) = their ids, step after
 * step; *total = their sum.  Waits for the handle's stream.  MGC_ERR_OVERFLOW
 * (counts and *total still set) when they do not fit ids_cap; ids_cap = 0
 * queries the counts only. */
mgc_status mgc_part_export(mgc_sim* sim, int32_t count, int32_t* counts, int32_t* ids, int64_t ids_cap,
                           int64_t* total);

/* Appends the other partitions' spikes of the same `count` steps: counts
 * (host, [nranks][count]) are every partition's exports, ids (device
 * memory as above) holds partition r's ids at ids + r * stride, in its
 * export order; the entries of `self` are skipped.  Waits for the handle's
 * stream.  An id outside the network refuses the whole import
 * (MGC_ERR_INVALID; the handle then refuses further imports and mgc_sync
 * reports it). */
mgc_status mgc_part_import(mgc_sim* sim, int32_t count, int32_t nranks, int32_t self, const int32_t* counts,
                           const int32_t* ids, int64_t stride);

/* The same exchange kept on the device, for callers that gather on the
 * device (NCCL all-gather on the handle's stream, or device copies): no host
 * synchronisation, a fixed capacity.  mgc_part_export_dev enqueues on the
 * handle's stream the window's export into buf (device memory, count + cap
 * ints): buf[0..count) = spikes per step, buf[count..) = their ids, cut at
 * cap ids.  mgc_part_import_dev enqueues the import from bufs, nranks such
 * blocks of count + cap ints side by side (rank r's at bufs + r*(count+cap),
 * the layout an all-gather of the export buffers gives); nranks = 1 only
 * closes the window.  The caller orders the gather between the two on the
 * handle's stream (mgc_get_stream).  A window in which any rank exported
 * more than cap ids is refused on every rank, and so are invalid counts or
 * ids: every later mgc_sync returns MGC_ERR_INVALID, since the steps after
 * a refused window miss its spikes (repeat the run with a larger cap). */
mgc_status mgc_part_export_dev(mgc_sim* sim, int32_t count, int32_t* buf, int64_t cap);
mgc_status mgc_part_import_dev(mgc_sim* sim, int32_t count, int32_t nranks, int32_t self, const int32_t* bufs,
                               int64_t cap);

/* Host-side fault injection for callers' error paths: the n-th device
 * allocation from now (n >= 1) fails as if the device were out of memory;
 * 0 turns it off.  The entry point that meets it returns MGC_ERR_NOMEM and
 * frees what it had allocated.  No reference counterpart (the reference's
 * CUDACHECK exits the process, cudamem.cuh:8-18). */
mgc_status mgc_fault_inject_alloc(int64_t n);

/* Self-test of the step groups' bounded waits, with no fault: runs the
 * pipelined group's phase wait (which = 0) or the per-step grid barrier
 * (which = 1) against a counter that nothing advances.  *status gets the
 * device status bits (4: the wait gave up, as mgc_sync reports it for a
 * step group), *ms the kernel's duration; the device stays usable.  No
 * reference counterpart (the reference has no waits inside kernels). */
mgc_status mgc_selftest_wait_timeout(int32_t device, int32_t which, int32_t* status, double* ms);

/* Enqueues `steps` steps on the handle's stream and returns without
 * waiting.  Replaces the step loop of MGSimulator::simulate_sparse
 * (mgsim.cpp:794-857) calling mgsim_step_sparse (mgcore.cu:535-554);
 * the caller applies the reference's step-count rule (see
 * mgc_effective_steps).  Steps continue from the previous call. */
mgc_status mgc_run(mgc_sim* sim, int64_t steps);

/* Waits for the handle's stream and reports device-side errors. */
mgc_status mgc_sync(mgc_sim* sim);

/* Copies n POISSON per-step probabilities from host memory (pinned memory
 * makes the copy asynchronous); takes effect from the next enqueued step.
 * Replaces writing Neuron::rate before construction (e.g.
 * bench/single_brunel.cpp:46-50). */
mgc_status mgc_set_rates(mgc_sim* sim, const float* rate, int32_t n);

/* Copies out the raster recorded since the previous read and clears it:
 * counts[i] = spikes of step first_step+i, ids = their neuron ids, ascending
 * inside each step.  The reference records no raster; its only output is
 * fire_cnt (mgsim.cpp:596-615). */
mgc_status mgc_read_raster(mgc_sim* sim, int64_t* first_step, int64_t* counts, int64_t counts_cap,
                           int32_t* ids, int64_t ids_cap, int64_t* n_steps, int64_t* n_ids);

/* The same readout without stopping the device, for readers that read while
 * the simulation goes on: mgc_raster_stage enqueues on the handle's stream a
 * device copy of the raster recorded so far into one of two staging buffers
 * and starts a new raster (no host wait); mgc_raster_collect waits only for
 * the oldest staged copy and returns it as mgc_read_raster does, while the
 * steps enqueued after that stage keep running.  At most two stages are
 * outstanding; mgc_read_raster refuses while one is.  No reference
 * counterpart. */
mgc_status mgc_raster_stage(mgc_sim* sim);
mgc_status mgc_raster_collect(mgc_sim* sim, int64_t* first_step, int64_t* counts, int64_t counts_cap,
                              int32_t* ids, int64_t ids_cap, int64_t* n_steps, int64_t* n_ids);

/* Copies neuron state to host arrays of n entries; any pointer may be NULL.
 * Replaces get_subnet_firecnt (mgnet.cpp:148-158) / copy_subnet_cpu
 * (mgnet.cpp:283-300). */
mgc_status mgc_read_state(mgc_sim* sim, float* v, float* i_exc, float* i_inh, int32_t* refrac,
                          int32_t* last_fired, int32_t* fire_cnt);

/* Copies the S synaptic weights in synapse-list order (mgc_create networks). */
mgc_status mgc_read_weights(mgc_sim* sim, float* weight);

/* Copies the CSR the core built: row_ptr[n+1], tgt[S], weight[S], delay[S]
 * (any may be NULL). */
mgc_status mgc_export_csr(mgc_sim* sim, int64_t* row_ptr, int32_t* tgt, float* weight, int32_t* delay);

/* Cut and balance statistics of a neuron partition over the handle's
 * synapses, computed on the device: replaces PartitionAnalysis's host loops
 * (src/partition/analysis.cpp: getCostNum, getZoneNeu, getZoneSyn,
 * getZoneOut, getZoneIn).  part[i] (host, one entry per network neuron,
 * 0 <= part[i] < nparts <= 4096) is neuron i's zone.  Outputs (host arrays
 * of nparts, any may be NULL): zone_neurons[z] = neurons in z; zone_syn[z] =
 * synapses whose source is in z; zone_out[z] / zone_in[z] = synapses that
 * cross zones, by source zone / by target zone; *cut = all crossing
 * synapses.  A partition handle counts the synapses it holds (those that
 * target its neurons). */
mgc_status mgc_partition_stats(mgc_sim* sim, const int32_t* part, int32_t nparts, int64_t* cut,
                               int64_t* zone_neurons, int64_t* zone_syn, int64_t* zone_out, int64_t* zone_in);

mgc_status mgc_get_info(mgc_sim* sim, mgc_info* info);

/* Runs `steps` steps with each kernel class bracketed by CUDA events (the
 * steps and their event records are captured in batches of 64 as CUDA
 * graphs, so the kernels run back to back as in mgc_run): ms[0] neuron
 * update, ms[1] event delivery (with STDP, which runs inside the push or
 * the pull), ms[2] 0 (kept for the layout), summed over the steps.  No reference counterpart (the
 * reference was profiled externally with nvprof, shell/single.sh:15). */
mgc_status mgc_profile_steps(mgc_sim* sim, int64_t steps, float* ms);

typedef struct mgc_tune_report {
    int32_t trials;               /* configurations timed */
    int32_t chunk_len;            /* chosen synapses per delivery task (deferred method) */
    int32_t blocks_per_sm;        /* chosen resident blocks per SM of the step's main kernel (0: the
                                     ring or pull method's push on fewer blocks than SMs) */
    int32_t persistent;           /* chosen step-group mode of the fused method (mgc_set_persistent) */
    int32_t window;               /* chosen window of the windowed step group (mgc_set_window) */
    int32_t pull_min;             /* chosen pull-step threshold (mgc_set_pull), 0: none */
    double ms_per_step;           /* time per step of the chosen configuration */
    double default_ms_per_step;   /* time per step of the builder's configuration */
    int64_t steps;                /* steps simulated by the trials */
} mgc_tune_report;

/* Autotuner: times `steps_per_trial` steps (rounded up to whole graphs) of
 * each launch configuration — synapses per delivery task (the threads a
 * spike's delay segment gets) x resident blocks per SM of the step kernel,
 * then (fused method) the best of those as a persistent step group, one
 * cooperative launch of up to 1024 steps with a bounded grid barrier between
 * steps — starting with the builder's choice, and keeps the fastest.  The trials are
 * real steps: the simulation advances by report->steps.  The configuration
 * changes which warp adds which synapse, and so the order of the fp32
 * additions into a neuron's input: no result changes with one weight per
 * sign; with unequal weights of one sign the last bits of V may (as between
 * two runs of the reference's atomics).  The windowed step group
 * (mgc_set_persistent mode 3) is among the trials, and so are its pull steps
 * (mgc_set_pull) at thresholds of n/3, n/8 and n/20 arriving (spike, delay)
 * pairs, on networks of at most 2^27 synapses with a minimum delay >= 2
 * (their incoming rows are kept only when a threshold wins).  No reference counterpart
 * (its launch shapes are fixed, mgcore.cu:535-554). */
mgc_status mgc_autotune(mgc_sim* sim, int64_t steps_per_trial, mgc_tune_report* report);

/* mgc_autotune without advancing the simulation: saves a checkpoint of the
 * state, runs the trials and loads the checkpoint back (also after a failed
 * trial), so that the handle keeps the chosen launch configuration and
 * continues from the step it was at, as a handle that ran no trial would
 * (the raster restarts empty there; on a handle that records a raster,
 * refused while it holds steps not yet read).  report->steps counts the trials' steps, which are undone.  Host
 * memory of mgc_checkpoint_size bytes is held during the call.  No reference
 * counterpart. */
mgc_status mgc_autotune_rewind(mgc_sim* sim, int64_t steps_per_trial, mgc_tune_report* report);

/* How the fused method runs: 0 CUDA graphs of single-step kernels; 1
 * cooperative step groups of up to
 * 1024 steps with a grid barrier between steps; 2 pipelined step groups
 * (minimum delay >= 4): during step s each block delivers the arrivals of
 * step s+2 and waits only until every block has finished step s-2; 3
 * windowed step groups (minimum delay >= 2): the arrivals of a window of W
 * steps (mgc_set_window) are delivered before it, then every neuron advances
 * the W steps with its state in registers, two grid barriers per window.
 * Default: 2 when the minimum delay is >= 4, else 1; the autotuner may pick
 * another.  If the device cannot keep all blocks of a group resident, the
 * call falls back to 0.  Results are the same in every mode; while a schedule mode other than
 * static, recording or calibration is on, graphs are used.  All waits are
 * bounded (a time-out makes mgc_sync return MGC_ERR_CUDA).  No reference
 * counterpart. */
mgc_status mgc_set_persistent(mgc_sim* sim, int32_t mode);

/* Pull steps (deferred method, minimum delay >= 2, not for partition
 * handles): in the windowed step group (mgc_set_persistent mode 3), a step
 * whose arrivals come from at least `min_pairs` (spike, delay) pairs is
 * delivered by pull instead of push: one warp per target walks the target's
 * incoming row and adds the weights of the synapses whose source spiked at
 * the step minus the delay (the spike history kept as a bitmap per step),
 * with no atomics.  A pull reads every incoming synapse, so it pays off only
 * on steps where a large part of the network's sources send (synchronous
 * bursts: one burst of a dense network can put hundreds of events on every
 * target in one step).  The choice is made on the device per step from the
 * spike counts the delivery already holds; results are those of the push
 * bit for bit (fixed-point sums exact; fp32 sums need one weight per sign,
 * else the call returns MGC_ERR_INVALID).  The first call builds the
 * incoming rows (8 bytes per synapse) and the bitmaps; the windowed group
 * writes a bitmap for every step it updates while pull steps are on, and a
 * step is pulled only when every step its arrivals come from has one (steps
 * run in another form, or before the call, or before a checkpoint load,
 * have none: their arrivals are pushed).  0 turns pull steps off (the rows
 * stay).  No reference counterpart (the reference always pushes,
 * mgcore.cu:271-305). */
mgc_status mgc_set_pull(mgc_sim* sim, int32_t min_pairs);

/* Chooses how inputs are summed (MGC_ACC_FLOAT or MGC_ACC_FIXED, see
 * above), before the handle's first step (MGC_ERR_INVALID after it, or for
 * FIXED with the pull method).  No reference counterpart. */
mgc_status mgc_set_accumulation(mgc_sim* sim, int32_t mode);

/* Steps per window of the windowed step group (mode 3 of
 * mgc_set_persistent): 1 <= steps <= min(8, minimum delay); default the
 * largest.  Windows of more than 4 steps hold their steps' inputs in eight
 * accumulator buffers (allocated for a minimum delay >= 5) instead of four;
 * the next mgc_run moves the current step's buffer between the two cycles,
 * one small kernel on the handle's stream.  Results are the same for every
 * window.  No reference counterpart. */
mgc_status mgc_set_window(mgc_sim* sim, int32_t steps);

/* ---- Step scheduler (fused deferred method: minimum delay >= 2) ----------
 * Each CUDA graph of 64 steps starts with a decision kernel that picks which
 * of two instantiations of the fused step kernel (compiled for 2 or 3
 * resident blocks per SM) runs the group, through a conditional SWITCH node:
 * the choice is made on the device, the host never waits for it, and it
 * changes no arithmetic (rasters are those of either variant alone).
 *   STATIC:    the autotuner's variant.
 *   THRESHOLD: the variant for the last group's delivered events per step
 *              (above `threshold`: hi_variant, else the other).
 *   LEARNED:   the same rule on the events per step that a small MLP
 *              (4 groups x [spikes of up to 4 trace populations, events] ->
 *              next group, 32 ReLU hidden units) predicts; trained on the
 *              GPU by the library's own forward/backward/Adam kernel on group
 *              traces the simulator recorded.
 * A decision is a miss when it differs from the rule applied to the group's
 * actual load.  No reference counterpart (fixed schedule, mgcore.cu:535-554). */
enum { MGC_SCHED_STATIC = 0, MGC_SCHED_THRESHOLD = 1, MGC_SCHED_LEARNED = 2 };

/* MLP shape: flat parameters [W1 (32x20, row-major), b1 (32), W2 (5x32), b2 (5)]. */
enum { MGC_MLP_IN = 20, MGC_MLP_HIDDEN = 32, MGC_MLP_OUT = 5, MGC_MLP_PARAMS = 837 };

typedef struct mgc_sched_stats {
    int32_t mode;
    int32_t trained;
    int64_t groups;               /* decisions scored (THRESHOLD / LEARNED groups) */
    int64_t misses;
    int64_t variant_groups[2];    /* groups run by each variant */
    double mean_abs_log_err;      /* LEARNED: mean |log1p(predicted) - log1p(actual)| events/step */
    double threshold;
    int32_t hi_variant;
    int32_t static_variant;
    int32_t recorded_groups;      /* group rows recorded for training */
    int32_t reserved;
} mgc_sched_stats;

mgc_status mgc_sched_set_mode(mgc_sim* sim, int32_t mode);

/* The load (delivered events per step) above which hi_variant runs. */
mgc_status mgc_sched_set_threshold(mgc_sim* sim, double threshold, int32_t hi_variant);

/* Runs `groups`+1 step groups alternating the two variants (real steps),
 * fits time per step = a + b * load for each and sets the threshold to the
 * crossing inside the observed load range (else: the faster variant always). */
mgc_status mgc_sched_calibrate(mgc_sim* sim, int32_t groups, double* threshold);

/* Records (on != 0) the feature row of every step group that runs from now
 * on, for training; reset drops the rows recorded so far. */
mgc_status mgc_sched_collect(mgc_sim* sim, int32_t on, int32_t reset);

/* Trains the MLP on the recorded rows (windows of 4 consecutive groups ->
 * the next), `epochs` passes of Adam, minibatches of 64, on the GPU. */
mgc_status mgc_sched_train(mgc_sim* sim, int32_t epochs, float lr, uint64_t seed, float* final_loss);

mgc_status mgc_sched_report(mgc_sim* sim, mgc_sched_stats* report, int32_t reset);

/* Loss (1/n) sum_b sum_o (y - t)^2 / 2 and its gradient at `params` for n
 * (<= 128) samples x [n][20], t [n][5], computed by the training kernel's
 * forward/backward on `device` (host arrays in and out). */
mgc_status mgc_mlp_gradient(int32_t device, const float* params, const float* x, const float* y, int32_t n,
                            float* grad, float* loss);

/* Checkpoints: the state a simulation continues from — neuron state and
 * POISSON rates, the input still in flight (delay ring or accumulators and
 * spike history), the step clock, the event counter and, with STDP, the
 * weights — copied to or from host memory.  A handle built from the same
 * network with the same method that loads a checkpoint continues exactly as
 * the saved one would have; its raster starts empty at the restored step.
 * The scheduler's state and the raster are not part of it.  No reference
 * counterpart (its test/networkio.cpp intent, survey 8f). */
mgc_status mgc_checkpoint_size(mgc_sim* sim, int64_t* bytes);
mgc_status mgc_checkpoint_save(mgc_sim* sim, void* buf, int64_t bytes);
mgc_status mgc_checkpoint_load(mgc_sim* sim, const void* buf, int64_t bytes);

/* The handle's cudaStream_t, for event timing by the caller. */
mgc_status mgc_get_stream(mgc_sim* sim, void** stream);

/* Number of steps MGSimulator::simulate runs for `steps` requested steps
 * and the network's minimum delay: cycles = steps/min_delay +
 * (steps%min_delay == 0), each cycle bounded by steps (mgsim.cpp:801-838).
 * Returns -1 when min_delay < 1. */
int64_t mgc_effective_steps(int64_t steps, int32_t min_delay);

/* Frees the handle.  Replaces MGSimulator::~MGSimulator (mgsim.cpp:364-406)
 * without its cudaDeviceReset. */
void mgc_destroy(mgc_sim* sim);

/* Text of the last error on the calling thread. */
const char* mgc_last_error(void);

/* Kernels this library launched on this handle so far. */
int64_t mgc_kernel_launches(mgc_sim* sim);

/* Measures the two ceilings of event delivery on `device`: n_events scattered
 * fp32 reductions (one per event, into n_targets accumulators, each fed by an
 * 8-byte {target, weight} record streamed from device memory, the access
 * pattern of the delivery kernels) and a plain stream of the same records.
 * Records are generated on the device; best of `reps` timed runs after one
 * warm-up, with CUDA events.  Allocates n_events*8 + n_targets*4 bytes for
 * the call.  No reference counterpart (it measures the bound of the
 * reference's event push, mgcore.cu:271-305, whose atomics set its rate). */
mgc_status mgc_measure_scatter(int32_t device, int64_t n_events, int32_t n_targets, int32_t reps,
                               double* red_events_per_s, double* read_bytes_per_s);

/* CSR row offsets of a synapse list held in DEVICE memory, computed without
 * allocating anything: row_ptr[i] = synapses whose source is below i, for
 * i = 0..n_neurons (row_ptr[n_neurons] = n_synapses) — the row_ptr that
 * mgc_create builds and mgc_export_csr returns for the same list.  src
 * (n_synapses int32) and row_ptr (n_neurons+1 int64) are device pointers on
 * the current device; the work is enqueued on `stream` (a cudaStream_t, NULL
 * for the legacy default stream), and every call waits for that stream before
 * it returns (it reads back a count of out-of-range sources).
 *
 * For callers that cannot allocate device memory at this point: a caller whose
 * memory pool owns the device (cudaMalloc can fail there although the pool
 * has room), or a loop that rebuilds offsets while the simulation runs (every
 * cudaFree synchronises the whole device).  mgc_create's own scan takes its
 * scratch from cudaMalloc; this entry point uses a fixed 256 KB static device
 * array instead, which limits it to n_neurons <= 134,217,727 (larger sizes
 * return MGC_ERR_INVALID with the limit in mgc_last_error).  row_ptr needs no
 * initial contents (the call zeroes it and its own counters).  The first call
 * on a device does a one-time set-up (it looks up the scratch array's address,
 * cudaGetSymbolAddress), so make that first call before any stream capture
 * begins.  Because every call waits for its stream, no call can be captured
 * into a CUDA graph: do not make one on a capturing stream, nor on the legacy
 * stream (NULL) while another thread runs a global-mode capture.  All calls on one device share the one scratch array, which keeps
 * the last call's contents, so calls that overlapped on the GPU would race on
 * it; the library serialises them with a lock per device, held until the
 * call's work on the stream has finished, on success and on failure alike.
 * Sources outside [0, n_neurons) are skipped and reported as
 * MGC_ERR_INVALID.  No reference counterpart (the reference computes its row
 * offsets, axon_offs, on the host: src/simulator/mgsim/adj/mgsim.cpp:115-122). */
mgc_status mgc_row_offsets_static(const int32_t* src, int64_t n_synapses, int32_t n_neurons, int64_t* row_ptr,
                                  void* stream);

#ifdef __cplusplus
}
#endif
#endif
