/*
 * falcon_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity oracle).
 *
 * A plain-C, single-thread-per-query restatement of the Falcon FPGA traversal
 * (fpgasystems/Falcon-accelerate-graph-vector-search).  It exists so that the
 * tests, the smoke check and the bench's CPU-baseline leg can check the CUDA
 * product path bit for bit.  Nothing in the product library links or calls it.
 *
 * Parity is pinned two ways (see tests/test_oracle_pin.py):
 *   - against the reference's own HLS kernel sources compiled as plain C++
 *     with host-side stream/ap_int shims (oracle/ref_harness, built into
 *     oracle/_ref/), on seeded graphs: ids, distances, hops and visited counts
 *     must agree exactly;
 *   - against the reference's software Murmur2 (unit_tests/bloom_and_hash/
 *     sw_murmur2/murmur2.cpp) and std::sort (unit_tests/priority_queue/src/
 *     host.cpp:121-152) through golden vectors in tests/golden/.
 *
 * Semantics restated (file:line of the inter-query v1.3 kernel,
 * FPGA_multi_DDR/FPGA_inter_query_v1.3_longer_FIFO_alt_PR/src/, unless noted):
 *   scheduler            scheduler.hpp:54-172
 *   systolic queue       priority_queue.hpp:9-166 (v1.5 insert: intra
 *                        FPGA_intra_query_v1.5_support_batching_longer_FIFO/
 *                        src/priority_queue.hpp:86-90)
 *   Bloom + Murmur2      bloom_filter.hpp:43-66, 117-204
 *   adjacency fetch      DRAM_utils.hpp:198-290
 *   vector fetch         DRAM_utils.hpp:292-353
 *   L2 adder-tree order  compute.hpp:10-37, 39-282
 *   results collection   DRAM_utils.hpp:355-467 (intra: v1.5 DRAM_utils.hpp:
 *                        355-470, utils.hpp:277-347, 396-569)
 *
 * Compile with -ffp-contract=off (no FMA contraction) and without
 * -ffast-math: the float order of every operation is part of the contract.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define FO_LARGE 1e20f          /* constants.hpp:14 large_float */

/* -------------------------------------------------------------------------- */
/* Murmur2, key length 4 (bloom_filter.hpp:43-66)                              */
/* -------------------------------------------------------------------------- */
uint32_t fo_murmur2_keylen4(uint32_t key, uint32_t seed)
{
    const uint32_t m = 0x5bd1e995u;
    uint32_t k = key;
    k *= m;
    k ^= k >> 24;
    k *= m;
    uint32_t h = seed ^ 4u;
    h *= m;
    h ^= k;
    h ^= h >> 13;
    h *= m;
    h ^= h >> 15;
    return h;
}

/* -------------------------------------------------------------------------- */
/* Bloom filter: 3 hashes with seeds seed, seed+1, seed+2 (bloom_filter.hpp:   */
/* 274-288); bit index = low `bits` bits of the hash (:174-177).  A key is     */
/* valid (not yet visited) unless all three bits were already set (:168-188).  */
/* -------------------------------------------------------------------------- */
typedef struct {
    uint32_t *words;
    int bits;
    uint32_t seed;
} fo_bloom;

static void bloom_reset(fo_bloom *b) { memset(b->words, 0, ((size_t)1 << b->bits) / 8); }

static int bloom_check_update(fo_bloom *b, uint32_t key)
{
    int matched = 0;
    const uint32_t mask = (b->bits >= 32) ? 0xffffffffu : ((1u << b->bits) - 1u);
    for (int j = 0; j < 3; j++) {
        uint32_t pos = fo_murmur2_keylen4(key, b->seed + (uint32_t)j) & mask;
        uint32_t bit = 1u << (pos & 31u);
        if (b->words[pos >> 5] & bit) matched++;
        else b->words[pos >> 5] |= bit;
    }
    return matched < 3;
}

/* -------------------------------------------------------------------------- */
/* Systolic priority queue (priority_queue.hpp).  Array sorted descending by   */
/* distance; q[0] is the worst element, q[n-1] the best.                       */
/* -------------------------------------------------------------------------- */
typedef struct {
    float *d;
    int *id;
    int n;
} fo_queue;

static void q_reset(fo_queue *q)
{
    for (int i = 0; i < q->n; i++) { q->d[i] = FO_LARGE; q->id[i] = -1; }
}

static inline void q_cas(fo_queue *q, int a, int b)
{   /* compare_swap: swap iff q[a] < q[b] (priority_queue.hpp:29-39) */
    if (q->d[a] < q->d[b]) {
        float td = q->d[a]; q->d[a] = q->d[b]; q->d[b] = td;
        int ti = q->id[a]; q->id[a] = q->id[b]; q->id[b] = ti;
    }
}

static inline void q_step(fo_queue *q)
{   /* step A then step B (priority_queue.hpp:41-57); pairs touching the
       invalid tail (-1e20) never swap, so only pairs inside [0,n) matter. */
    for (int j = 0; 2 * j + 1 < q->n; j++) q_cas(q, 2 * j, 2 * j + 1);
    for (int j = 0; 2 * j + 2 < q->n; j++) q_cas(q, 2 * j + 1, 2 * j + 2);
}

static void q_sort(fo_queue *q)
{   /* sort(): ceil(n/2) rounds of A+B (priority_queue.hpp:94-105) */
    int rounds = (q->n + 1) / 2;
    for (int r = 0; r < rounds; r++) q_step(q);
}

/* v1.3 insert_only: replace q[0] if smaller, A+B after every item (:83-89) */
static void q_insert_v13(fo_queue *q, int id, float d)
{
    if (d < q->d[0]) { q->d[0] = d; q->id[0] = id; }
    q_step(q);
}

/* v1.5 insert_only: A+B only when the item replaced q[0] (v1.5 :86-90) */
static void q_insert_v15(fo_queue *q, int id, float d)
{
    if (d < q->d[0]) { q->d[0] = d; q->id[0] = id; q_step(q); }
}

static void q_pop(fo_queue *q, int *id_out)
{   /* pop_top: take q[n-1], shift right, q[0] = +large (:131-165) */
    *id_out = q->id[q->n - 1];
    for (int i = q->n - 1; i > 0; i--) { q->d[i] = q->d[i - 1]; q->id[i] = q->id[i - 1]; }
    q->d[0] = FO_LARGE; q->id[0] = -1;
}

/* -------------------------------------------------------------------------- */
/* Squared L2 in the reference adder-tree order (compute.hpp).                  */
/* Leaves are (q[j]-x[j])^2 over the dimension padded to a multiple of 16 with */
/* zeros.  Each 16-float chunk is summed by the 4-level pairwise tree (:10-37).*/
/* Chunk partials are packed 16 per pack, zero filled (:127-196), each pack is */
/* summed by the same tree, and packs are accumulated left to right (:260-267).*/
/* -------------------------------------------------------------------------- */
static inline float tree16(const float *v)
{
    float l0[8], l1[4], l2[2];
    for (int i = 0; i < 8; i++) l0[i] = v[2 * i] + v[2 * i + 1];
    for (int i = 0; i < 4; i++) l1[i] = l0[2 * i] + l0[2 * i + 1];
    for (int i = 0; i < 2; i++) l2[i] = l1[2 * i] + l1[2 * i + 1];
    return l2[0] + l2[1];
}

/* x_dec: the database vector already decoded to float (dpad entries, zero
   padded past dim); q: the query padded the same way. */
static float l2_tree(const float *q, const float *x_dec, int dpad)
{
    const int chunks = dpad / 16;
    const int packs = (chunks + 15) / 16;
    float final_dist = 0.0f;
    for (int p = 0; p < packs; p++) {
        float pack[16];
        for (int i = 0; i < 16; i++) {
            int c = p * 16 + i;
            if (c < chunks) {
                float sq[16];
                for (int s = 0; s < 16; s++) {
                    float diff = q[c * 16 + s] - x_dec[c * 16 + s];
                    sq[s] = diff * diff;
                }
                pack[i] = tree16(sq);
            } else {
                pack[i] = 0.0f;
            }
        }
        float agg = tree16(pack);
        final_dist = (p == 0) ? agg : final_dist + agg;
    }
    return final_dist;
}

float fo_l2(const float *q, const float *x, int dpad) { return l2_tree(q, x, dpad); }

/* -------------------------------------------------------------------------- */
/* Element decoders for the stored base vectors.                              */
/* -------------------------------------------------------------------------- */
enum { FO_F32 = 0, FO_BF16 = 1, FO_FP8 = 2 };

static inline float bf16_to_f32(uint16_t h)
{
    uint32_t u = ((uint32_t)h) << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

/* OCP FP8 E4M3 (the "fn" variant: no infinities, S.1111.111 is NaN). */
float fo_fp8e4m3_to_f32(uint8_t c)
{
    int s = c >> 7, e = (c >> 3) & 15, m = c & 7;
    float v;
    if (e == 15 && m == 7) return NAN;
    if (e == 0) v = ldexpf((float)m, -9);            /* m/8 * 2^-6 */
    else v = ldexpf((float)(8 + m), e - 10);          /* (1+m/8) * 2^(e-7) */
    return s ? -v : v;
}

typedef struct {
    const void *vectors;     /* base vectors, row stride vec_stride elements */
    const float *scales;     /* FP8 only: one float per vector */
    int elem;                /* FO_F32 / FO_BF16 / FO_FP8 */
    int64_t vec_stride;      /* in elements */
    const float *vectors_f32;/* FP32 copy used by the rerank (may be NULL) */
    int64_t vec_stride_f32;
    const int32_t *links;    /* adjacency rows: count at offset 0, ids at ids_offset */
    int64_t link_stride;     /* in int32 */
    int ids_offset;
    int max_degree;
    int dim;                 /* true dimension */
    int dpad;                /* dimension padded to a multiple of 16 */
    int64_t n;
} fo_graph;

static void decode_vec(const fo_graph *g, int64_t id, float *out)
{
    if (g->elem == FO_F32) {
        const float *v = (const float *)g->vectors + id * g->vec_stride;
        for (int j = 0; j < g->dpad; j++) out[j] = (j < g->dim) ? v[j] : 0.0f;
    } else if (g->elem == FO_BF16) {
        const uint16_t *v = (const uint16_t *)g->vectors + id * g->vec_stride;
        for (int j = 0; j < g->dpad; j++) out[j] = (j < g->dim) ? bf16_to_f32(v[j]) : 0.0f;
    } else {
        const uint8_t *v = (const uint8_t *)g->vectors + id * g->vec_stride;
        float sc = g->scales[id];
        for (int j = 0; j < g->dpad; j++) out[j] = (j < g->dim) ? fo_fp8e4m3_to_f32(v[j]) * sc : 0.0f;
    }
}

static float dist_to(const fo_graph *g, const float *qpad, int64_t id, float *scratch)
{
    decode_vec(g, id, scratch);
    return l2_tree(qpad, scratch, g->dpad);
}

/* -------------------------------------------------------------------------- */
/* One query.                                                                   */
/* -------------------------------------------------------------------------- */
typedef struct {
    int k, ef, mc, mg, cand_queue_size, bloom_bits;
    uint32_t hash_seed;
    int mode;        /* 0 = inter-query (v1.3), 1 = intra-query (v1.5) */
    int channels;    /* intra-query channel count (power of two) */
    int rerank;      /* reduced precision: exact FP32 rerank of the final ef */
    int max_hops;    /* 0 = unbounded; otherwise stop after this many hops */
} fo_params;

typedef struct {
    float *d; int *id;          /* result queue storage */
    float *cd; int *cid;        /* candidate queue storage */
    uint32_t *bloom_words;      /* channels * 2^bits / 32 words */
    int *fifo;                  /* mg groups * mc ids */
    int *fifo_len;
    float *qpad, *scratch;
    int *chan_ids;              /* intra: routed ids per channel */
    int *chan_len;
    int *ins_ids; float *ins_d; /* items forwarded to the candidate queue */
} fo_work;

/* Trace of one inter-query traversal (FPGA_multi_DDR/
   eval_trace_FPGA_inter_query_v1.3/src/DRAM_utils.hpp:389-474 and
   scheduler.hpp:84): per expanded candidate in FIFO order its distance (1e20
   for the entry point, which is not distance-computed) and the number of
   distances computed for its row; per computed distance in stream order the
   distance and the id.  Entries past a capacity are counted, not written. */
typedef struct {
    float *cand_d; int *cand_n; int cand_cap;
    float *d; int *id; int cap;
    int n_pop, n_exp, n_dist;
} fo_trace;

static int row_count(const fo_graph *g, int node)
{
    return g->links[(int64_t)node * g->link_stride];
}
static int row_id(const fo_graph *g, int node, int j)
{
    return g->links[(int64_t)node * g->link_stride + g->ids_offset + j];
}

/* Returns 0 on success, 1 when max_hops cut the traversal short. */
static int search_one(const fo_graph *g, const fo_params *p, const float *query, int entry,
                      fo_work *w, int *out_id, float *out_d, int *out_hops, int *out_visited, fo_trace *tr)
{
    const int ef = p->ef, mc = p->mc, mg = p->mg;
    fo_queue rq = { w->d, w->id, ef };
    fo_queue cq = { w->cd, w->cid, p->cand_queue_size };
    const int nch = (p->mode == 1) ? p->channels : 1;
    fo_bloom bl[64];
    const size_t wpc = ((size_t)1 << p->bloom_bits) / 32;
    for (int c = 0; c < nch; c++) {
        bl[c].words = w->bloom_words + c * wpc; bl[c].bits = p->bloom_bits; bl[c].seed = p->hash_seed;
        bloom_reset(&bl[c]);
    }
    for (int j = 0; j < g->dpad; j++) w->qpad[j] = (j < g->dim) ? query[j] : 0.0f;
    q_reset(&rq);
    q_reset(&cq);

    /* group FIFO: ring of mg slots, each up to mc candidate ids */
    int head = 0, inflight = 1;
    w->fifo[0] = entry; w->fifo_len[0] = 1;
    int hops = 1, visited = 0, truncated = 0;
    if (tr) {
        tr->n_pop = 1; tr->n_exp = 0; tr->n_dist = 0;
        if (tr->cand_cap > 0) tr->cand_d[0] = FO_LARGE;
    }

    while (inflight > 0) {
        const int *grp = w->fifo + head * mc;
        const int glen = w->fifo_len[head];
        if (p->mode == 0) {
            /* inter-query v1.3: per candidate, Bloom -> L2 -> result queue
               (DRAM_utils.hpp:411-439), forwarded items -> candidate queue
               (scheduler.hpp:102-110). */
            for (int b = 0; b < glen; b++) {
                const int node = grp[b];
                const int cnt = row_count(g, node);
                int nins = 0, nval = 0;
                for (int j = 0; j < cnt; j++) {
                    const int nb = row_id(g, node, j);
                    if (!bloom_check_update(&bl[0], (uint32_t)nb)) continue;
                    visited++;
                    nval++;
                    const float dd = dist_to(g, w->qpad, nb, w->scratch);
                    if (tr) {
                        if (tr->n_dist < tr->cap) { tr->d[tr->n_dist] = dd; tr->id[tr->n_dist] = nb; }
                        tr->n_dist++;
                    }
                    if (dd < rq.d[0]) {
                        rq.d[0] = dd; rq.id[0] = nb;
                        w->ins_ids[nins] = nb; w->ins_d[nins] = dd; nins++;
                    }
                    q_step(&rq);
                }
                for (int i = 0; i < nins; i++) q_insert_v13(&cq, w->ins_ids[i], w->ins_d[i]);
                if (tr) {
                    if (tr->n_exp < tr->cand_cap) tr->cand_n[tr->n_exp] = nval;
                    tr->n_exp++;
                }
            }
            q_sort(&rq);
        } else {
            /* intra-query v1.5: merge the group's rows, route ids by
               id & (channels-1) (utils.hpp:396-495), per-channel Bloom ->
               L2, merge channels in channel order (utils.hpp:497-569 picks
               readiness order; channel order is one of its schedules). */
            for (int c = 0; c < nch; c++) w->chan_len[c] = 0;
            for (int b = 0; b < glen; b++) {
                const int node = grp[b];
                const int cnt = row_count(g, node);
                for (int j = 0; j < cnt; j++) {
                    const int nb = row_id(g, node, j);
                    const int c = nb & (nch - 1);
                    w->chan_ids[c * (g->max_degree * mc) + w->chan_len[c]++] = nb;
                }
            }
            int any_insert = 0;
            for (int c = 0; c < nch; c++) {
                int nins = 0;
                for (int j = 0; j < w->chan_len[c]; j++) {
                    const int nb = w->chan_ids[c * (g->max_degree * mc) + j];
                    if (!bloom_check_update(&bl[c], (uint32_t)nb)) continue;
                    visited++;
                    const float dd = dist_to(g, w->qpad, nb, w->scratch);
                    /* v1.5 results_collection (DRAM_utils.hpp:425-437): A+B
                       only on insertion.  The stale-threshold prefilter
                       (utils.hpp:277-347) never drops an item that would be
                       inserted, so it is not restated. */
                    if (dd < rq.d[0]) {
                        rq.d[0] = dd; rq.id[0] = nb;
                        q_step(&rq);
                        w->ins_ids[nins] = nb; w->ins_d[nins] = dd; nins++;
                        any_insert = 1;
                    }
                }
                for (int i = 0; i < nins; i++) q_insert_v15(&cq, w->ins_ids[i], w->ins_d[i]);
            }
            if (any_insert) q_sort(&rq);
        }
        /* group retired: scheduler.hpp:112-155 */
        const float thr = rq.d[0];
        head = (head + 1) % mg;
        inflight--;
        q_sort(&cq);
        for (int oid = inflight; oid < mg; oid++) {
            int slot = (head + inflight) % mg;
            int n = 0;
            for (int b = 0; b < mc; b++) {
                const float best = cq.d[cq.n - 1];
                if (best <= thr && best < FO_LARGE) {
                    if (p->max_hops > 0 && hops >= p->max_hops) { truncated = 1; break; }
                    if (tr) {
                        if (tr->n_pop < tr->cand_cap) tr->cand_d[tr->n_pop] = best;
                        tr->n_pop++;
                    }
                    q_pop(&cq, &w->fifo[slot * mc + n]);
                    n++;
                    hops++;
                } else {
                    break;
                }
            }
            if (n == 0) break;
            w->fifo_len[slot] = n;
            inflight++;
        }
    }

    /* results best-first (DRAM_utils.hpp:460-464) */
    for (int i = 0; i < ef; i++) { out_id[i] = rq.id[ef - 1 - i]; out_d[i] = rq.d[ef - 1 - i]; }
    *out_hops = hops;
    *out_visited = visited;
    return truncated;
}

/* Exact FP32 rerank of the final ef candidates of a reduced-precision
   traversal: same adder tree on the FP32 vectors, stable ascending sort
   (ties keep traversal order).  Extension beyond the reference. */
static void rerank_f32(const fo_graph *g, const float *qpad, int ef, int *ids, float *ds, float *scratch)
{
    fo_graph g32 = *g;
    g32.elem = FO_F32; g32.vectors = g->vectors_f32; g32.vec_stride = g->vec_stride_f32;
    for (int i = 0; i < ef; i++) ds[i] = (ids[i] >= 0) ? dist_to(&g32, qpad, ids[i], scratch) : FO_LARGE;
    for (int i = 1; i < ef; i++) {   /* insertion sort = stable */
        float kd = ds[i]; int ki = ids[i]; int j = i - 1;
        while (j >= 0 && ds[j] > kd) { ds[j + 1] = ds[j]; ids[j + 1] = ids[j]; j--; }
        ds[j + 1] = kd; ids[j + 1] = ki;
    }
}

/* -------------------------------------------------------------------------- */
/* Batch driver (pthreads over queries).                                       */
/* -------------------------------------------------------------------------- */
typedef struct {
    const fo_graph *g;
    const fo_params *params;   /* one per query, or one shared (param_stride 0) */
    int param_stride;
    const float *queries; int64_t q_stride;
    const int32_t *entries;
    int64_t nq;
    int out_stride;            /* results per query row (>= max k) */
    int32_t *out_ids; float *out_d; int32_t *out_hops; int32_t *out_visited;
    int64_t next;
    pthread_mutex_t mu;
    int any_truncated;
    /* trace (inter-query mode; NULL = off): per query cand_cap / cap entries, counts [3] */
    float *tr_cand_d; int32_t *tr_cand_n; int tr_cand_cap;
    float *tr_d; int32_t *tr_id; int tr_cap;
    int32_t *tr_counts;
} fo_batch;

static void *batch_worker(void *arg)
{
    fo_batch *bt = (fo_batch *)arg;
    const fo_graph *g = bt->g;
    int max_ef = 0, max_mc = 0, max_mg = 0, max_cq = 0, max_bits = 0, max_ch = 1;
    for (int64_t i = 0; i < (bt->param_stride ? bt->nq : 1); i++) {
        const fo_params *p = bt->params + i * bt->param_stride;
        if (p->ef > max_ef) max_ef = p->ef;
        if (p->k > max_ef) max_ef = p->k;
        if (p->mc > max_mc) max_mc = p->mc;
        if (p->mg > max_mg) max_mg = p->mg;
        if (p->cand_queue_size > max_cq) max_cq = p->cand_queue_size;
        if (p->bloom_bits > max_bits) max_bits = p->bloom_bits;
        if (p->mode == 1 && p->channels > max_ch) max_ch = p->channels;
    }
    fo_work w;
    w.d = malloc(sizeof(float) * max_ef); w.id = malloc(sizeof(int) * max_ef);
    w.cd = malloc(sizeof(float) * max_cq); w.cid = malloc(sizeof(int) * max_cq);
    w.bloom_words = malloc(((size_t)1 << max_bits) / 8 * max_ch);
    w.fifo = malloc(sizeof(int) * max_mg * max_mc); w.fifo_len = malloc(sizeof(int) * max_mg);
    w.qpad = malloc(sizeof(float) * g->dpad); w.scratch = malloc(sizeof(float) * g->dpad);
    w.chan_ids = malloc(sizeof(int) * max_ch * g->max_degree * max_mc); w.chan_len = malloc(sizeof(int) * max_ch);
    w.ins_ids = malloc(sizeof(int) * g->max_degree * max_mc); w.ins_d = malloc(sizeof(float) * g->max_degree * max_mc);
    int *tid = malloc(sizeof(int) * max_ef); float *td = malloc(sizeof(float) * max_ef);
    for (;;) {
        pthread_mutex_lock(&bt->mu);
        int64_t qi = bt->next;
        bt->next += 8;
        pthread_mutex_unlock(&bt->mu);
        if (qi >= bt->nq) break;
        int64_t qe = qi + 8 < bt->nq ? qi + 8 : bt->nq;
        for (; qi < qe; qi++) {
            fo_params p = bt->params[qi * bt->param_stride];
            if (p.ef < p.k) p.ef = p.k;
            int hops, vis;
            fo_trace trace, *tp = NULL;
            if (bt->tr_counts) {
                trace.cand_d = bt->tr_cand_d + qi * bt->tr_cand_cap; trace.cand_n = bt->tr_cand_n + qi * bt->tr_cand_cap;
                trace.cand_cap = bt->tr_cand_cap;
                trace.d = bt->tr_d + qi * bt->tr_cap; trace.id = bt->tr_id + qi * bt->tr_cap; trace.cap = bt->tr_cap;
                tp = &trace;
            }
            int tr = search_one(g, &p, bt->queries + qi * bt->q_stride, bt->entries[qi], &w, tid, td, &hops, &vis, tp);
            if (tp) {
                bt->tr_counts[3 * qi] = trace.n_pop;
                bt->tr_counts[3 * qi + 1] = trace.n_exp;
                bt->tr_counts[3 * qi + 2] = trace.n_dist;
            }
            if (tr) { pthread_mutex_lock(&bt->mu); bt->any_truncated = 1; pthread_mutex_unlock(&bt->mu); }
            if (p.rerank && g->elem != FO_F32 && g->vectors_f32) rerank_f32(g, w.qpad, p.ef, tid, td, w.scratch);
            for (int i = 0; i < bt->out_stride; i++) {
                bt->out_ids[qi * bt->out_stride + i] = (i < p.k) ? tid[i] : -1;
                bt->out_d[qi * bt->out_stride + i] = (i < p.k) ? td[i] : FO_LARGE;
            }
            bt->out_hops[qi] = hops;
            bt->out_visited[qi] = vis;
        }
    }
    free(w.d); free(w.id); free(w.cd); free(w.cid); free(w.bloom_words); free(w.fifo); free(w.fifo_len);
    free(w.qpad); free(w.scratch); free(w.chan_ids); free(w.chan_len); free(w.ins_ids); free(w.ins_d);
    free(tid); free(td);
    return NULL;
}

/* Public entry: returns 0 ok, 1 if some query hit max_hops, <0 on bad args. */
int fo_search(const fo_graph *g, const fo_params *params, int param_stride,
              const float *queries, int64_t q_stride, const int32_t *entries, int64_t nq,
              int out_stride, int32_t *out_ids, float *out_d, int32_t *out_hops, int32_t *out_visited,
              int threads)
{
    if (!g || !params || nq < 0 || g->dpad % 16 || g->dpad < g->dim) return -1;
    for (int64_t i = 0; i < (param_stride ? nq : 1); i++) {
        const fo_params *p = params + i * param_stride;
        if (p->ef < 1 || p->k < 1 || p->k > out_stride || p->mc < 1 || p->mg < 1 ||
            p->cand_queue_size < 1 || p->bloom_bits < 10 || p->bloom_bits > 30) return -2;
        if (p->mode == 1 && (p->channels < 1 || p->channels > 64 || (p->channels & (p->channels - 1)))) return -3;
    }
    fo_batch bt;
    bt.g = g; bt.params = params; bt.param_stride = param_stride;
    bt.queries = queries; bt.q_stride = q_stride; bt.entries = entries; bt.nq = nq;
    bt.out_stride = out_stride; bt.out_ids = out_ids; bt.out_d = out_d;
    bt.out_hops = out_hops; bt.out_visited = out_visited; bt.next = 0; bt.any_truncated = 0;
    bt.tr_cand_d = NULL; bt.tr_cand_n = NULL; bt.tr_cand_cap = 0;
    bt.tr_d = NULL; bt.tr_id = NULL; bt.tr_cap = 0; bt.tr_counts = NULL;
    pthread_mutex_init(&bt.mu, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    for (int t = 0; t < threads; t++) pthread_create(&th[t], NULL, batch_worker, &bt);
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&bt.mu);
    return bt.any_truncated;
}

/* Queue kernels exposed for the unit tests (priority_queue sort check,
   unit_tests/priority_queue/src/host.cpp:49-59,121-152). */
void fo_queue_insert_sort(float *d, int *id, int n, const float *in_d, const int *in_id, int n_in, int v15)
{
    fo_queue q = { d, id, n };
    q_reset(&q);
    for (int i = 0; i < n_in; i++) {
        if (v15) q_insert_v15(&q, in_id[i], in_d[i]);
        else q_insert_v13(&q, in_id[i], in_d[i]);
    }
    q_sort(&q);
}

/* Bloom filter exposed for the unit tests: valid[i] for a key stream. */
void fo_bloom_stream(const uint32_t *keys, int n, int bits, uint32_t seed, uint8_t *valid)
{
    fo_bloom b;
    b.bits = bits; b.seed = seed;
    b.words = calloc(((size_t)1 << bits) / 32, 4);
    for (int i = 0; i < n; i++) valid[i] = (uint8_t)bloom_check_update(&b, keys[i]);
    free(b.words);
}

/* L2 of many vectors against one query, for unit tests. */
void fo_l2_batch(const fo_graph *g, const float *query, const int32_t *ids, int n, float *out)
{
    float *qpad = malloc(sizeof(float) * g->dpad), *scratch = malloc(sizeof(float) * g->dpad);
    for (int j = 0; j < g->dpad; j++) qpad[j] = (j < g->dim) ? query[j] : 0.0f;
    for (int i = 0; i < n; i++) out[i] = dist_to(g, qpad, ids[i], scratch);
    free(qpad); free(scratch);
}

/* -------------------------------------------------------------------------- */
/* HNSW upper-layer greedy descent (hnswalg.h:514-541 of the vendored hnswlib; */
/* FPGA_single_DDR/FPGA_single_DDR_multi_layer_v2.2_async/src/                  */
/* scheduler.hpp:116-144).  From the top entry, for level = max_level .. 1:     */
/* repeat { scan the current node's level row in order, moving to every       */
/* neighbour whose distance is strictly below the current one } until a scan  */
/* moves nowhere.  No visited filter.  Distances use the same adder-tree order */
/* as the base search (the FPGA computes upper and base distances in the same */
/* compute units).  The v2.2 scheduler starts one level lower (max_level - 1) */
/* because its indexes keep only the entry point on the top level, whose row  */
/* is then empty: both starts give the same entry there.                      */
/* -------------------------------------------------------------------------- */
typedef struct {
    const int32_t *rows;      /* row r at rows + r * row_stride: count, ids from ids_offset */
    int64_t row_stride;
    int ids_offset;
    const int64_t *row_start; /* node v's level-l row is row_start[v] + l - 1 */
    const int32_t *levels;    /* per node */
    int max_level;
    int entry;
} fo_upper;

int fo_descend(const fo_graph *g, const fo_upper *u, const float *queries, int64_t nq, int64_t qstride,
               int32_t *out_entry, int32_t *out_hops)
{
    float *qpad = malloc(sizeof(float) * g->dpad), *scratch = malloc(sizeof(float) * g->dpad);
    if (!qpad || !scratch) { free(qpad); free(scratch); return -1; }
    for (int64_t qi = 0; qi < nq; qi++) {
        const float *q = queries + qi * qstride;
        for (int j = 0; j < g->dpad; j++) qpad[j] = (j < g->dim) ? q[j] : 0.0f;
        int cur = u->entry, hops = 0;
        float curdist = dist_to(g, qpad, cur, scratch);
        for (int level = u->max_level; level > 0; level--) {
            int changed = 1;
            while (changed) {
                changed = 0;
                hops++;
                if (u->levels[cur] < level) break;
                const int32_t *row = u->rows + (u->row_start[cur] + level - 1) * u->row_stride;
                const int size = row[0];
                for (int i = 0; i < size; i++) {
                    const int cand = row[u->ids_offset + i];
                    const float d = dist_to(g, qpad, cand, scratch);
                    if (d < curdist) {
                        curdist = d;
                        cur = cand;
                        changed = 1;
                    }
                }
            }
        }
        out_entry[qi] = cur;
        if (out_hops) out_hops[qi] = hops;
    }
    free(qpad);
    free(scratch);
    return 0;
}

/* Inter-query search with the traversal trace (see fo_trace): per query
   cand_cap candidate entries (distance, computed count) and cap distance
   entries (distance, id); counts[3q..3q+2] = popped candidates incl. the entry,
   expanded candidates, computed distances (entries past a capacity are counted,
   not written). */
int fo_search_trace(const fo_graph *g, const fo_params *params, const float *queries, int64_t q_stride,
                    const int32_t *entries, int64_t nq, int out_stride, int32_t *out_ids, float *out_d,
                    int32_t *out_hops, int32_t *out_visited, float *tr_cand_d, int32_t *tr_cand_n, int cand_cap,
                    float *tr_d, int32_t *tr_id, int cap, int32_t *tr_counts, int threads)
{
    if (!g || !params || nq < 0 || g->dpad % 16 || g->dpad < g->dim || params->mode != 0 || !tr_counts) return -1;
    if (params->ef < 1 || params->k < 1 || params->k > out_stride || params->mc < 1 || params->mg < 1 ||
        params->cand_queue_size < 1 || params->bloom_bits < 10 || params->bloom_bits > 30 || cand_cap < 0 || cap < 0)
        return -2;
    fo_batch bt;
    bt.g = g; bt.params = params; bt.param_stride = 0;
    bt.queries = queries; bt.q_stride = q_stride; bt.entries = entries; bt.nq = nq;
    bt.out_stride = out_stride; bt.out_ids = out_ids; bt.out_d = out_d;
    bt.out_hops = out_hops; bt.out_visited = out_visited; bt.next = 0; bt.any_truncated = 0;
    bt.tr_cand_d = tr_cand_d; bt.tr_cand_n = tr_cand_n; bt.tr_cand_cap = cand_cap;
    bt.tr_d = tr_d; bt.tr_id = tr_id; bt.tr_cap = cap; bt.tr_counts = tr_counts;
    pthread_mutex_init(&bt.mu, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    for (int t = 0; t < threads; t++) pthread_create(&th[t], NULL, batch_worker, &bt);
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&bt.mu);
    return bt.any_truncated;
}
