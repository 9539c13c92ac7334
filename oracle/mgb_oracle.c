/*
 * mgb_oracle — CPU restatement of the reference MGBrain hot path.
 * TEST INFRASTRUCTURE: the checker for mgbrain_b200's CUDA core, never part
 * of the product.  See mgb_oracle.h for the reference file:line map.
 *
 * Build: see oracle/Makefile (-O2 -ffp-contract=off -fopenmp).
 */
#include "mgb_oracle.h"
#include "mgb_philox.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct mgbo_sim {
    int32_t n;
    int64_t S;
    int32_t M, dmin, dmax;
    int precision, nthreads;
    int8_t* type;
    float* rate;
    uint8_t* fired;
    int32_t *fire_cnt, *last_fired, *refrac;
    void *V, *Iexc, *Iinh, *ring_e, *ring_i, *w;
    int64_t* axon_off;
    int32_t *csr_tar, *csr_src, *csr_delay;
    int64_t* csr_syn;          /* synapse-list index of each CSR position */
    uint8_t* csr_plastic;      /* NULL: all plastic */
    int64_t* dend_off;
    int64_t* dend_pos;         /* CSR position of each incoming synapse */
    float lifc[30], stdpc[6];
    int32_t refrac_steps;
    float lifb_leak;
    int stdp;
    uint64_t seed;
    int32_t id_offset;
    int64_t step, events;
    int32_t* spk;
    /* fixed-point accumulation (mgbo_set_fx): integer rings, weights added
     * as rint(w * fx_scale), sums read as float(sum) * fx_unscale */
    int fx;
    float fx_scale, fx_unscale;
    int64_t *ring_fx_e, *ring_fx_i;
};

/* ------------------------------------------------------------------ */
/* MT19937, restated from Matsumoto & Nishimura (1998)                */
/* ------------------------------------------------------------------ */
void mgbo_mt_seed(mgbo_mt19937* g, uint32_t seed)
{
    g->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->idx = 624;
}

uint32_t mgbo_mt_next(mgbo_mt19937* g)
{
    if (g->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            uint32_t v = g->mt[(i + 397) % 624] ^ (y >> 1);
            if (y & 1u) v ^= 0x9908b0dfu;
            g->mt[i] = v;
        }
        g->idx = 0;
    }
    uint32_t y = g->mt[g->idx++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= (y >> 18);
    return y;
}

/* ------------------------------------------------------------------ */
/* Model / NetGen                                                     */
/* ------------------------------------------------------------------ */
int mgbo_model_connect(mgbo_proj* pros, int npro, const mgbo_pop* pops, mgbo_proj p, int* ok)
{
    /* model.cpp:86-111: one-to-one needs equal sizes; an existing (src,tar)
     * pair is overwritten only when its index is > 0. */
    if (p.ctype == 0.0f && pops[p.src].num != pops[p.tar].num) {
        *ok = 0;
        return npro;
    }
    *ok = 1;
    int index = -1;
    for (int i = 0; i < npro; ++i)
        if (pros[i].src == p.src && pros[i].tar == p.tar) index = i;
    if (index > 0) {
        pros[index].wmin = p.wmin; pros[index].wmax = p.wmax;
        pros[index].dmin = p.dmin; pros[index].dmax = p.dmax;
        pros[index].ctype = p.ctype; pros[index].stype = p.stype;
        return npro;
    }
    pros[npro] = p;
    return npro + 1;
}

/* netgen.cpp:19-31 */
static float rand_weight(float floor_, float ceil_, float dw)
{
    if (ceil_ == floor_) return floor_;
    int range = (int)((ceil_ - floor_) / dw) + 1;
    float tw;
    if (floor_ < 0)
        tw = floor_ + (float)(rand() % range) * dw;
    else
        tw = floor_ - (float)(rand() % range) * dw;
    return tw;
}

/* netgen.cpp:32-38 */
static float rand_delay(float floor_, float ceil_, float dt)
{
    if (ceil_ == floor_) return floor_;
    int range = (int)((ceil_ - floor_) / dt) + 1;
    return floor_ + (float)(rand() % range) * dt;
}

typedef struct {
    mgbo_synlist* o;
    int64_t cap;
} synbuf;

static int syn_push(synbuf* b, int32_t s, int32_t t, float w, float d, int32_t pr)
{
    mgbo_synlist* o = b->o;
    if (o->n_syn == b->cap) {
        int64_t nc = b->cap ? b->cap * 2 : 1024;
        int32_t* ns = realloc(o->src, nc * sizeof(int32_t));
        int32_t* nt = ns ? realloc(o->tar, nc * sizeof(int32_t)) : NULL;
        if (ns) o->src = ns;
        if (nt) o->tar = nt;
        float* nw = nt ? realloc(o->weight, nc * sizeof(float)) : NULL;
        if (nw) o->weight = nw;
        float* nd = nw ? realloc(o->delay, nc * sizeof(float)) : NULL;
        if (nd) o->delay = nd;
        int32_t* np = nd ? realloc(o->proj, nc * sizeof(int32_t)) : NULL;
        if (np) o->proj = np;
        if (!np) return -1;
        b->cap = nc;
    }
    o->src[o->n_syn] = s; o->tar[o->n_syn] = t;
    o->weight[o->n_syn] = w; o->delay[o->n_syn] = d; o->proj[o->n_syn] = pr;
    o->n_syn++;
    return 0;
}

int mgbo_netgen(const mgbo_pop* pops, int npop, const mgbo_proj* pros, int npro,
                uint32_t mt_seed, int64_t rand_seed, float dw, float dt, int shuffle_gen,
                mgbo_synlist* out)
{
    memset(out, 0, sizeof(*out));
    synbuf b = {out, 0};
    if (rand_seed >= 0) srand((unsigned)rand_seed);
    mgbo_mt19937* rng = malloc(sizeof(mgbo_mt19937));
    int32_t* start = malloc(sizeof(int32_t) * (npop + 1));
    if (!rng || !start) { free(rng); free(start); return -1; }
    mgbo_mt_seed(rng, mt_seed); /* netgen.cpp:47, one engine for the call */
    start[0] = 0;
    for (int i = 0; i < npop; ++i) start[i + 1] = start[i] + pops[i].num;

    for (int i = 0; i < npro; ++i) {
        const mgbo_proj* p = &pros[i];
        const int sn = pops[p->src].num, tn = pops[p->tar].num;
        const int32_t s0 = start[p->src], t0 = start[p->tar];
        if (p->ctype == 1.0f) {
            /* netgen.cpp:84-111 */
            for (int m = 0; m < sn; ++m)
                for (int n = 0; n < tn; ++n) {
                    float w = rand_weight(p->wmin, p->wmax, dw);
                    float d = rand_delay(p->dmin, p->dmax, dt);
                    if (syn_push(&b, s0 + m, t0 + n, w, d, i)) goto oom;
                }
        } else if (p->ctype == 0.0f) {
            /* netgen.cpp:112-126 */
            for (int k = 0; k < sn; ++k) {
                float w = rand_weight(p->wmin, p->wmax, dw);
                float d = rand_delay(p->dmin, p->dmax, dt);
                if (syn_push(&b, s0 + k, t0 + k, w, d, i)) goto oom;
            }
        } else if (p->ctype < 1.0f && p->ctype > 0.0f) {
            if (shuffle_gen) {
                /* netgen.cpp:129-163; std::random_shuffle as libstdc++
                 * implements it: for i in [1,n): j = rand() % (i+1); swap. */
                size_t len = (size_t)(int)(sn * tn);
                size_t gen_num = (size_t)roundf((float)len * p->ctype);
                uint8_t* g = calloc(len ? len : 1, 1);
                if (!g) goto oom;
                for (size_t k = 0; k < len; ++k) g[k] = k < gen_num;
                for (size_t k = 1; k < len; ++k) {
                    size_t j = (size_t)((long)rand() % (long)(k + 1));
                    if (j != k) { uint8_t t = g[k]; g[k] = g[j]; g[j] = t; }
                }
                for (int m = 0; m < sn; ++m)
                    for (int n = 0; n < tn; ++n)
                        if (g[(size_t)m * tn + n]) {
                            float w = rand_weight(p->wmin, p->wmax, dw);
                            float d = rand_delay(p->dmin, p->dmax, dt);
                            if (syn_push(&b, s0 + m, t0 + n, w, d, i)) { free(g); goto oom; }
                        }
                free(g);
            } else {
                /* netgen.cpp:164-226: Bernoulli(1.1 p) in row-major order,
                 * capped at gen_num; unfilled genlist entries stay 0 and
                 * still become synapses (m = 0, n = 0). */
                size_t max_num = (size_t)sn * (size_t)tn;
                size_t gen_num = (size_t)roundf((float)max_num * p->ctype);
                size_t count = 0;
                size_t* genlist = calloc(gen_num ? gen_num : 1, sizeof(size_t));
                if (!genlist) goto oom;
                const double lim = (double)gen_num * 1.1;
                for (size_t m = 0; m < (size_t)sn; ++m)
                    for (size_t n = 0; n < (size_t)tn; ++n)
                        if (count < gen_num &&
                            (double)((unsigned long)mgbo_mt_next(rng) % max_num) < lim)
                            genlist[count++] = m * tn + n;
                for (size_t t = 0; t < gen_num; ++t) {
                    int m = (int)(genlist[t] / tn);
                    int n = (int)(genlist[t] % tn);
                    float w = rand_weight(p->wmin, p->wmax, dw);
                    float d = rand_delay(p->dmin, p->dmax, dt);
                    if (syn_push(&b, s0 + m, t0 + n, w, d, i)) { free(genlist); goto oom; }
                }
                free(genlist);
            }
        }
    }
    free(rng);
    free(start);
    return 0;
oom:
    free(rng);
    free(start);
    mgbo_synlist_free(out);
    return -1;
}

void mgbo_synlist_free(mgbo_synlist* s)
{
    free(s->src); free(s->tar); free(s->weight); free(s->delay); free(s->proj);
    memset(s, 0, sizeof(*s));
}

/* ------------------------------------------------------------------ */
/* Build rules                                                        */
/* ------------------------------------------------------------------ */
void mgbo_quantize_delays(const float* delay_s, int64_t n, float step_s, int32_t* out,
                          int32_t* dmin, int32_t* dmax)
{
    int32_t lo = 2147483647, hi = 0; /* mgsim.cpp:42-43 */
    for (int64_t i = 0; i < n; ++i) {
        int32_t d = (int32_t)roundf(delay_s[i] / step_s);
        out[i] = d;
        if (d > hi) hi = d;
        if (d < lo) lo = d;
    }
    *dmin = lo;
    *dmax = hi;
}

int64_t mgbo_steps_for_time(float time_s, float step_s)
{
    return (int64_t)(int)roundf(time_s / step_s);
}

int64_t mgbo_effective_steps(int64_t steps, int32_t min_delay)
{
    if (min_delay <= 0) return -1;
    int64_t cycles = steps / min_delay + (steps % min_delay == 0);
    int64_t eff = cycles * (int64_t)min_delay;
    return eff < steps ? eff : steps;
}

/* ------------------------------------------------------------------ */
/* Precision-templated step core                                      */
/* ------------------------------------------------------------------ */
static inline float mgbo_exp_f32(float x) { return expf(x); }
static inline double mgbo_exp_f64(double x) { return exp(x); }

/* A neuron's input of the step from ring entry loc, and the clearing of the
 * entry: the REAL rings, or with fixed-point accumulation the integer sum
 * converted to float once (round to nearest) and scaled by 2^-shift. */
#define IN_E(loc) (s->fx ? (REAL)((float)s->ring_fx_e[loc] * s->fx_unscale) : re[loc])
#define IN_I(loc) (s->fx ? (REAL)((float)s->ring_fx_i[loc] * s->fx_unscale) : ri[loc])
#define CLEAR_IN(loc)                                         \
    do {                                                      \
        if (s->fx) {                                          \
            s->ring_fx_e[loc] = 0;                            \
            s->ring_fx_i[loc] = 0;                            \
        } else {                                              \
            re[loc] = 0;                                      \
            ri[loc] = 0;                                      \
        }                                                     \
    } while (0)

#define REAL float
#define SUFFIX(x) x##_f32
#include "oracle_core.inc"
#undef REAL
#undef SUFFIX
#define REAL double
#define SUFFIX(x) x##_f64
#include "oracle_core.inc"
#undef REAL
#undef SUFFIX

/* ------------------------------------------------------------------ */
/* Simulation object                                                  */
/* ------------------------------------------------------------------ */
static void* xcalloc(size_t n, size_t sz)
{
    return calloc(n ? n : 1, sz);
}

static mgbo_sim* sim_alloc_neurons(int32_t n, const int8_t* type, const float* rate,
                                   const float* v0, const float* lifc, int32_t precision,
                                   int32_t nthreads)
{
    mgbo_sim* s = xcalloc(1, sizeof(mgbo_sim));
    if (!s) return NULL;
    s->n = n;
    s->precision = precision;
    s->nthreads = nthreads < 1 ? 1 : nthreads;
    size_t rs = precision == MGBO_F64 ? sizeof(double) : sizeof(float);
    s->type = xcalloc(n, 1);
    s->rate = xcalloc(n, sizeof(float));
    s->fired = xcalloc(n, 1);
    s->fire_cnt = xcalloc(n, 4);
    s->last_fired = xcalloc(n, 4);
    s->refrac = xcalloc(n, 4);
    s->V = xcalloc(n, rs);
    s->Iexc = xcalloc(n, rs);
    s->Iinh = xcalloc(n, rs);
    s->spk = xcalloc(n, 4);
    memcpy(s->type, type, n);
    if (rate) memcpy(s->rate, rate, sizeof(float) * n);
    memcpy(s->lifc, lifc, sizeof(float) * 30);
    for (int32_t i = 0; i < n; ++i) {
        float v = v0 ? v0[i] : lifc[1];
        if (precision == MGBO_F64) ((double*)s->V)[i] = v;
        else ((float*)s->V)[i] = v;
    }
    /* mgcore.cu:184: Refrac_state = round(t_ref / DT) - 1, in fp32 */
    s->refrac_steps = (int32_t)roundf(lifc[8] / lifc[0]) - 1;
    /* mgcore.cu:190 hard-codes the LIFB leak 0.005f (dt/tau_m at 0.1 ms /
     * 20 ms); lifconst[9] (unused by the reference) overrides it when set. */
    s->lifb_leak = lifc[9] != 0.0f ? lifc[9] : 0.005f;
    return s;
}

static int sim_alloc_ring(mgbo_sim* s)
{
    size_t rs = s->precision == MGBO_F64 ? sizeof(double) : sizeof(float);
    s->ring_e = xcalloc((size_t)s->n * s->M, rs);
    s->ring_i = xcalloc((size_t)s->n * s->M, rs);
    return (s->ring_e && s->ring_i) ? 0 : -1;
}

mgbo_sim* mgbo_create(int32_t n, const int8_t* type, const float* rate, const float* v0,
                      int64_t n_syn, const int32_t* src, const int32_t* tar,
                      const float* weight, const int32_t* delay_steps,
                      const float* lifc, const float* stdpc, int32_t stdp,
                      const uint8_t* plastic, uint64_t seed, int32_t precision,
                      int32_t nthreads)
{
    mgbo_sim* s = sim_alloc_neurons(n, type, rate, v0, lifc, precision, nthreads);
    if (!s) return NULL;
    s->S = n_syn;
    s->seed = seed;
    s->stdp = stdp;
    memcpy(s->stdpc, stdpc, sizeof(float) * 6);
    /* mgsim.cpp:42-71 */
    int32_t dmax = 0, dmin = 2147483647;
    for (int64_t k = 0; k < n_syn; ++k) {
        if (delay_steps[k] > dmax) dmax = delay_steps[k];
        if (delay_steps[k] < dmin) dmin = delay_steps[k];
    }
    s->dmin = dmin;
    s->dmax = dmax;
    s->M = dmax + 1;
    /* CSR by source, synapse-list order inside a row (mgsim.cpp:44-70,116-131) */
    s->axon_off = xcalloc((size_t)n + 1, sizeof(int64_t));
    s->dend_off = xcalloc((size_t)n + 1, sizeof(int64_t));
    s->csr_tar = xcalloc(n_syn, 4);
    s->csr_src = xcalloc(n_syn, 4);
    s->csr_delay = xcalloc(n_syn, 4);
    s->csr_syn = xcalloc(n_syn, 8);
    s->dend_pos = xcalloc(n_syn, 8);
    s->w = xcalloc(n_syn, precision == MGBO_F64 ? 8 : 4);
    if (plastic) s->csr_plastic = xcalloc(n_syn, 1);
    if (sim_alloc_ring(s)) { mgbo_destroy(s); return NULL; }
    for (int64_t k = 0; k < n_syn; ++k) {
        s->axon_off[src[k] + 1]++;
        s->dend_off[tar[k] + 1]++;
    }
    for (int32_t i = 0; i < n; ++i) {
        s->axon_off[i + 1] += s->axon_off[i];
        s->dend_off[i + 1] += s->dend_off[i];
    }
    int64_t* fill = xcalloc((size_t)n + 1, sizeof(int64_t));
    int64_t* pos = xcalloc(n_syn, sizeof(int64_t));
    memcpy(fill, s->axon_off, sizeof(int64_t) * n);
    for (int64_t k = 0; k < n_syn; ++k) {
        int64_t p = fill[src[k]]++;
        pos[k] = p;
        s->csr_tar[p] = tar[k];
        s->csr_src[p] = src[k];
        s->csr_delay[p] = delay_steps[k];
        s->csr_syn[p] = k;
        if (precision == MGBO_F64) ((double*)s->w)[p] = weight[k];
        else ((float*)s->w)[p] = weight[k];
        if (plastic) s->csr_plastic[p] = plastic[k] ? 1 : 0;
    }
    memcpy(fill, s->dend_off, sizeof(int64_t) * n);
    for (int64_t k = 0; k < n_syn; ++k) s->dend_pos[fill[tar[k]]++] = pos[k];
    free(fill);
    free(pos);
    return s;
}

/* Fixed in-degree generator shared with the CUDA core's device generator:
 * projection r gives every target t of pop pr_tar[r] exactly pr_k[r]
 * sources drawn uniformly (with replacement) from pop pr_src[r]:
 *   x = Philox4x32-10(key = conn_seed, counter = (t + id_offset, k, r + proj_offset, "CONN"))
 *   src   = start[pr_src] + (x0 * num[pr_src]) >> 32
 *   delay = dmin + (x1 * (dmax - dmin + 1)) >> 32   (steps)
 * Synapse-list order: r, then t, then k. */
#define MGB_TAG_CONN 0x434F4E4Eu
mgbo_sim* mgbo_create_fixed_indegree(const int32_t* pop_start, const int32_t* pop_num,
                                     const int32_t* pop_type, int32_t npop,
                                     const int32_t* pr_src, const int32_t* pr_tar,
                                     const int32_t* pr_k, const float* pr_w,
                                     const int32_t* pr_dmin, const int32_t* pr_dmax,
                                     int32_t npr, const float* rate, const float* v0,
                                     const float* lifc, uint64_t conn_seed, uint64_t seed,
                                     int32_t nthreads, int32_t id_offset, int32_t proj_offset)
{
    int32_t n = 0;
    for (int p = 0; p < npop; ++p)
        if (pop_start[p] + pop_num[p] > n) n = pop_start[p] + pop_num[p];
    int8_t* type = xcalloc(n, 1);
    for (int p = 0; p < npop; ++p)
        for (int32_t i = 0; i < pop_num[p]; ++i) type[pop_start[p] + i] = (int8_t)pop_type[p];
    mgbo_sim* s = sim_alloc_neurons(n, type, rate, v0, lifc, MGBO_F32, nthreads);
    free(type);
    if (!s) return NULL;
    s->seed = seed;
    s->id_offset = id_offset;
    s->stdp = 0;
    int64_t S = 0;
    int32_t dmin = 2147483647, dmax = 0;
    for (int r = 0; r < npr; ++r) {
        S += (int64_t)pop_num[pr_tar[r]] * pr_k[r];
        if (pr_k[r] > 0) {
            if (pr_dmin[r] < dmin) dmin = pr_dmin[r];
            if (pr_dmax[r] > dmax) dmax = pr_dmax[r];
        }
    }
    s->S = S;
    s->dmin = dmin;
    s->dmax = dmax;
    s->M = dmax + 1;
    s->axon_off = xcalloc((size_t)n + 1, sizeof(int64_t));
    s->dend_off = xcalloc((size_t)n + 1, sizeof(int64_t));
    s->csr_tar = xcalloc(S, 4);
    s->csr_delay = xcalloc(S, 4);
    s->w = xcalloc(S, 4);
    if (!s->csr_tar || !s->csr_delay || !s->w || sim_alloc_ring(s)) { mgbo_destroy(s); return NULL; }
    /* Stable counting sort by source, parallel: the synapse list (r, t, k)
     * is cut into T contiguous chunks of targets per projection.  Pass 1
     * counts entries per (projection, chunk, source); the runs of a row are
     * then laid out projection-major, chunk-minor, which is synapse-list
     * order; pass 2 scatters each chunk in its own order.  Rows therefore
     * keep synapse-list order for any thread count. */
    const int T = s->nthreads > 16 ? 16 : s->nthreads;
    {
        const int64_t np1 = (int64_t)n + 1;
        int64_t* cnt = xcalloc((size_t)npr * T * np1, sizeof(int64_t));
        if (!cnt) { mgbo_destroy(s); return NULL; }
        for (int pass = 0; pass < 2; ++pass) {
#ifdef _OPENMP
#pragma omp parallel num_threads(T)
#endif
            {
#ifdef _OPENMP
                const int me = omp_get_thread_num();
#else
                const int me = 0;
#endif
                for (int r = 0; r < npr; ++r) {
                    int64_t* mine = cnt + ((size_t)r * T + me) * np1;
                    const int32_t ts = pop_start[pr_tar[r]], tnum = pop_num[pr_tar[r]];
                    const int32_t ss = pop_start[pr_src[r]], snum = pop_num[pr_src[r]];
                    const uint32_t span = (uint32_t)(pr_dmax[r] - pr_dmin[r] + 1);
                    const int32_t lo = ts + (int32_t)((int64_t)tnum * me / T);
                    const int32_t hi = ts + (int32_t)((int64_t)tnum * (me + 1) / T);
                    for (int32_t t = lo; t < hi; ++t)
                        for (int32_t k = 0; k < pr_k[r]; ++k) {
                            mgb_u32x4 x = mgb_philox4x32_10((uint32_t)(t + id_offset), (uint32_t)k, (uint32_t)(r + proj_offset), MGB_TAG_CONN,
                                                            (uint32_t)conn_seed, (uint32_t)(conn_seed >> 32));
                            int32_t src = ss + (int32_t)(((uint64_t)x.v[0] * (uint64_t)snum) >> 32);
                            if (pass == 0) {
                                mine[src]++;
                            } else {
                                int32_t d = pr_dmin[r] + (int32_t)(((uint64_t)x.v[1] * span) >> 32);
                                int64_t p = mine[src]++;
                                s->csr_tar[p] = t;
                                s->csr_delay[p] = d;
                                ((float*)s->w)[p] = pr_w[r];
                            }
                        }
                }
            }
            if (pass == 0) {
                /* row_ptr, then start of each (r, chunk) run inside a row in
                 * synapse-list order: r major, chunk minor */
                for (int32_t i = 0; i < n; ++i) {
                    int64_t tot = 0;
                    for (int64_t q = 0; q < (int64_t)npr * T; ++q) tot += cnt[q * np1 + i];
                    s->axon_off[i + 1] = s->axon_off[i] + tot;
                }
                for (int32_t i = 0; i < n; ++i) {
                    int64_t pos = s->axon_off[i];
                    for (int64_t q = 0; q < (int64_t)npr * T; ++q) {
                        int64_t c = cnt[q * np1 + i];
                        cnt[q * np1 + i] = pos;
                        pos += c;
                    }
                }
            }
        }
        free(cnt);
    }
    return s;
}

void mgbo_set_rates(mgbo_sim* s, const float* rate)
{
    memcpy(s->rate, rate, sizeof(float) * s->n);
}

int mgbo_run(mgbo_sim* s, int64_t steps, int64_t* counts, int32_t* ids, int64_t ids_cap,
             int64_t* n_ids)
{
    int overflow = 0;
    int64_t nid = 0;
    for (int64_t k = 0; k < steps; ++k) {
        const int64_t step = s->step;
        int64_t nspk;
        if (s->precision == MGBO_F64) {
            nspk = neuron_update_f64(s, step, s->spk);
            push_f64(s, step, s->spk, nspk);
            if (s->stdp) stdp_f64(s, s->spk, nspk);
        } else {
            nspk = neuron_update_f32(s, step, s->spk);
            push_f32(s, step, s->spk, nspk);
            if (s->stdp) stdp_f32(s, s->spk, nspk);
        }
        if (counts) counts[k] = nspk;
        if (ids) {
            if (nid + nspk <= ids_cap) memcpy(ids + nid, s->spk, sizeof(int32_t) * nspk);
            else overflow = 1;
        }
        nid += nspk;
        s->step++;
    }
    if (n_ids) *n_ids = nid;
    return overflow ? -1 : 0;
}

int64_t mgbo_events(const mgbo_sim* s) { return s->events; }
int64_t mgbo_step(const mgbo_sim* s) { return s->step; }
int32_t mgbo_ring_len(const mgbo_sim* s) { return s->M; }
int32_t mgbo_min_delay(const mgbo_sim* s) { return s->dmin; }
int64_t mgbo_n_syn(const mgbo_sim* s) { return s->S; }

void mgbo_read_state(const mgbo_sim* s, double* v, double* i_exc, double* i_inh,
                     int32_t* refrac, int32_t* last_fired, int32_t* fire_cnt, double* weight)
{
    const int f64 = s->precision == MGBO_F64;
    for (int32_t i = 0; i < s->n; ++i) {
        if (v) v[i] = f64 ? ((double*)s->V)[i] : ((float*)s->V)[i];
        if (i_exc) i_exc[i] = f64 ? ((double*)s->Iexc)[i] : ((float*)s->Iexc)[i];
        if (i_inh) i_inh[i] = f64 ? ((double*)s->Iinh)[i] : ((float*)s->Iinh)[i];
    }
    if (refrac) memcpy(refrac, s->refrac, 4 * (size_t)s->n);
    if (last_fired) memcpy(last_fired, s->last_fired, 4 * (size_t)s->n);
    if (fire_cnt) memcpy(fire_cnt, s->fire_cnt, 4 * (size_t)s->n);
    if (weight && s->csr_syn)
        for (int64_t p = 0; p < s->S; ++p)
            weight[s->csr_syn[p]] = f64 ? ((double*)s->w)[p] : ((float*)s->w)[p];
}

void mgbo_read_state_f32(const mgbo_sim* s, float* v, float* weight)
{
    if (s->precision != MGBO_F32) return;
    if (v) memcpy(v, s->V, 4 * (size_t)s->n);
    if (weight && s->csr_syn)
        for (int64_t p = 0; p < s->S; ++p) weight[s->csr_syn[p]] = ((float*)s->w)[p];
}

void mgbo_export_csr(const mgbo_sim* s, int64_t* row_ptr, int32_t* tgt, float* w, int32_t* delay)
{
    if (row_ptr) memcpy(row_ptr, s->axon_off, 8 * ((size_t)s->n + 1));
    if (tgt) memcpy(tgt, s->csr_tar, 4 * (size_t)s->S);
    if (delay) memcpy(delay, s->csr_delay, 4 * (size_t)s->S);
    if (w && s->precision == MGBO_F32) memcpy(w, s->w, 4 * (size_t)s->S);
}

void mgbo_destroy(mgbo_sim* s)
{
    if (!s) return;
    free(s->type); free(s->rate); free(s->fired); free(s->fire_cnt); free(s->last_fired);
    free(s->refrac); free(s->V); free(s->Iexc); free(s->Iinh); free(s->ring_e); free(s->ring_i);
    free(s->w); free(s->axon_off); free(s->csr_tar); free(s->csr_src); free(s->csr_delay);
    free(s->csr_syn); free(s->csr_plastic); free(s->dend_off); free(s->dend_pos); free(s->spk);
    free(s->ring_fx_e); free(s->ring_fx_i);
    free(s);
}

void mgbo_set_id_offset(mgbo_sim* s, int32_t id_offset) { s->id_offset = id_offset; }

int mgbo_set_fx(mgbo_sim* s, int32_t shift)
{
    if (s->precision != MGBO_F32 || s->step != 0 || s->fx) return -1;
    s->ring_fx_e = xcalloc((size_t)s->n * s->M, sizeof(int64_t));
    s->ring_fx_i = xcalloc((size_t)s->n * s->M, sizeof(int64_t));
    if (!s->ring_fx_e || !s->ring_fx_i) return -1;
    s->fx = 1;
    s->fx_scale = ldexpf(1.0f, shift);
    s->fx_unscale = ldexpf(1.0f, -shift);
    return 0;
}

void mgbo_set_threads(mgbo_sim* s, int32_t nthreads)
{
    s->nthreads = nthreads < 1 ? 1 : nthreads;
}
