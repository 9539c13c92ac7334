/*
 * mgb_oracle — CPU restatement of the reference MGBrain single-GPU hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA core
 * in mgbrain_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline legs may load it.  The product never links or calls it.
 *
 * Restated reference behaviour (file:line within RAICLab-SNNGroup/MGBrain):
 *   network generation   src/model/netgen.cpp:19-38 (rand_weight/rand_delay),
 *                        :39-229 (gen_net), src/model/model.cpp:20-45 (connect)
 *   delay quantisation   src/simulator/mgsim/adj/mgsim.cpp:49, :71 (M = max+1)
 *   neuron update        src/simulator/mgsim/adj/mgcore.cu:116-234
 *   event push / ring    src/simulator/mgsim/adj/mgcore.cu:271-305, :112-115
 *   STDP                 src/simulator/mgsim/adj/mgcore.cu:346-412
 *   step count rule      src/simulator/mgsim/adj/mgsim.cpp:801-802, :821-838
 *
 * Precision: MGBO_F32 follows the reference's fp32 arithmetic operation by
 * operation (build with -ffp-contract=off); MGBO_F64 is the same algorithm
 * with fp64 state, used to state the fp32 error.
 */
#ifndef MGB_ORACLE_H
#define MGB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* NeuronType, src/macro.h:40-48 */
enum { MGBO_RAW = 0, MGBO_LIF0 = 1, MGBO_POISSON = 2, MGBO_LIF = 3, MGBO_LIFE = 4, MGBO_LIFB = 5 };
enum { MGBO_F32 = 0, MGBO_F64 = 1 };

/* ------------------------------------------------------------------ */
/* Network generation (src/model/netgen.cpp)                          */
/* ------------------------------------------------------------------ */
typedef struct {
    int32_t num;
    int32_t type;
    int32_t source;
} mgbo_pop;

typedef struct {
    int32_t src, tar;        /* population ids */
    float wmin, wmax;        /* Projection::wrange */
    float dmin, dmax;        /* Projection::drange (seconds) */
    float ctype;             /* 0 one-to-one, 1 all-to-all, (0,1) probability */
    int32_t stype;           /* 0 STATIC, 1 STDP */
} mgbo_proj;

typedef struct {
    int64_t n_syn;
    int32_t *src, *tar;
    float *weight, *delay;   /* delay in seconds, as Synapse::delay */
    int32_t *proj;           /* projection index of each synapse */
} mgbo_synlist;

/* MT19937 (Matsumoto & Nishimura 1998), the engine std::mt19937 specifies. */
typedef struct { uint32_t mt[624]; int idx; } mgbo_mt19937;
void mgbo_mt_seed(mgbo_mt19937* g, uint32_t seed);
uint32_t mgbo_mt_next(mgbo_mt19937* g);

/* Model::connect duplicate rule (model.cpp:89-110): returns the projection
 * count after adding/overwriting.  pros must have room for one more. */
int mgbo_model_connect(mgbo_proj* pros, int npro, const mgbo_pop* pops, mgbo_proj p, int* ok);

/* gen_net.  rand_seed >= 0 calls srand(rand_seed) first (glibc rand() feeds
 * rand_weight/rand_delay and the shuffle mode).  dw = Config::DW,
 * dt = Config::DT.  Returns 0 on success. */
int mgbo_netgen(const mgbo_pop* pops, int npop, const mgbo_proj* pros, int npro,
                uint32_t mt_seed, int64_t rand_seed, float dw, float dt, int shuffle_gen,
                mgbo_synlist* out);
void mgbo_synlist_free(mgbo_synlist* s);

/* ------------------------------------------------------------------ */
/* Build rules (mgsim.cpp)                                            */
/* ------------------------------------------------------------------ */
/* delay steps = round(delay / STEP) in fp32 (mgsim.cpp:49). */
void mgbo_quantize_delays(const float* delay_s, int64_t n, float step_s,
                          int32_t* out, int32_t* dmin, int32_t* dmax);
/* static_cast<int>(std::round(time / STEP)) (mgsim.cpp:801) */
int64_t mgbo_steps_for_time(float time_s, float step_s);
/* Steps simulate_sparse actually runs: cycles = steps/min_delay +
 * (steps%min_delay==0), each cycle min_delay steps bounded by steps. */
int64_t mgbo_effective_steps(int64_t steps, int32_t min_delay);

/* ------------------------------------------------------------------ */
/* Simulation                                                         */
/* ------------------------------------------------------------------ */
typedef struct mgbo_sim mgbo_sim;

/* Builds the CSR (axon, synapse-index order) and CSC (dend) like
 * build_multinet for npart=1.  delay_steps must be >= 1.
 * v0 == NULL -> V_m = lifc[1] (mgsim.cpp:97).  plastic == NULL -> every
 * synapse is plastic when stdp != 0 (Config::STDP).  nthreads > 1 uses
 * OpenMP for the neuron update and the push. */
mgbo_sim* mgbo_create(int32_t n, const int8_t* type, const float* rate, const float* v0,
                      int64_t n_syn, const int32_t* src, const int32_t* tar,
                      const float* weight, const int32_t* delay_steps,
                      const float* lifc, const float* stdpc, int32_t stdp,
                      const uint8_t* plastic, uint64_t seed, int32_t precision,
                      int32_t nthreads);

/* Procedural fixed in-degree network (the large-Brunel generator):
 * identical synapse list to the CUDA core's device generator. */
mgbo_sim* mgbo_create_fixed_indegree(const int32_t* pop_start, const int32_t* pop_num,
                                     const int32_t* pop_type, int32_t npop,
                                     const int32_t* pr_src, const int32_t* pr_tar,
                                     const int32_t* pr_k, const float* pr_w,
                                     const int32_t* pr_dmin, const int32_t* pr_dmax,
                                     int32_t npr, const float* rate, const float* v0,
                                     const float* lifc, uint64_t conn_seed, uint64_t seed,
                                     int32_t nthreads, int32_t id_offset, int32_t proj_offset);

/* Runs `steps` steps.  counts[steps] receives the spike count of each step
 * and ids the spiking neuron ids of each step in ascending order, capacity
 * ids_cap (ids may be NULL to skip recording).  Returns 0, or -1 when ids
 * overflowed (counts stay complete). */
int mgbo_run(mgbo_sim* s, int64_t steps, int64_t* counts, int32_t* ids, int64_t ids_cap,
             int64_t* n_ids);
void mgbo_set_rates(mgbo_sim* s, const float* rate);
void mgbo_set_threads(mgbo_sim* s, int32_t nthreads);  /* threads of later runs */
/* Neuron ids in the POISSON draws are offset by id_offset (a block of a
 * larger network draws as it does there). */
void mgbo_set_id_offset(mgbo_sim* s, int32_t id_offset);
/* Fixed-point accumulation, as the CUDA core's (include/mgc.h,
 * MGC_ACC_FIXED): every weight is added as llrintf(w * 2^shift) into a
 * 64-bit sum, which the neuron update reads as (float)sum * 2^-shift.  F32
 * sims, before the first step; returns 0 or -1.  Not a restatement of the
 * reference (whose fp32 atomics leave the order of unequal additions open):
 * it pins the CUDA core's order-independent arithmetic bit for bit. */
int mgbo_set_fx(mgbo_sim* s, int32_t shift);
int64_t mgbo_events(const mgbo_sim* s);      /* synaptic events delivered so far */
int64_t mgbo_step(const mgbo_sim* s);        /* steps simulated so far */
int32_t mgbo_ring_len(const mgbo_sim* s);    /* M = max_delay + 1 */
int32_t mgbo_min_delay(const mgbo_sim* s);
int64_t mgbo_n_syn(const mgbo_sim* s);
/* State readout; every pointer may be NULL.  weights in synapse-list order. */
void mgbo_read_state(const mgbo_sim* s, double* v, double* i_exc, double* i_inh,
                     int32_t* refrac, int32_t* last_fired, int32_t* fire_cnt, double* weight);
/* Raw fp32 readout (F32 sims only), bit-exact comparison against the GPU. */
void mgbo_read_state_f32(const mgbo_sim* s, float* v, float* weight);
/* CSR export (fixed in-degree sims): row_ptr[n+1], tgt[S], w[S], delay[S]. */
void mgbo_export_csr(const mgbo_sim* s, int64_t* row_ptr, int32_t* tgt, float* w, int32_t* delay);
void mgbo_destroy(mgbo_sim* s);

#ifdef __cplusplus
}
#endif
#endif
