// Graph traversal kernels for B200 (sm_100a).
//
// Inter-query mode: one warp owns one query at a time and pulls queries from a
// device work counter until the batch is drained (persistent grid sized to the
// SM count).  Per query the warp holds
//   - the result queue (ef <= 32*EPL entries, EPL per lane, registers),
//   - the candidate queue (<= 32 entries, one per lane, registers),
//   - the Bloom visited filter (2^bloom_bits bits, shared memory),
//   - the group FIFO of delayed-synchronization traversal (shared memory).
// The queues reproduce the reference's systolic odd-even priority queue
// (priority_queue.hpp:9-166) step for step, the Bloom filter its Murmur2
// 3-hash filter (bloom_filter.hpp:43-204), the distance its FP32 adder tree
// (compute.hpp:10-282), and the control loop its scheduler
// (scheduler.hpp:54-172) with the results collection of DRAM_utils.hpp:355-467.
// All reference paths are in FPGA_multi_DDR/FPGA_inter_query_v1.3_longer_FIFO_alt_PR/src.
//
// Memory traffic per hop: one adjacency row (count sector + max_degree ids) and
// one gathered vector per Bloom-accepted neighbour, loaded as 16-byte segments
// by the 32 lanes (coalesced), read-only path, no L1 allocation.
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include "falcon_internal.h"

namespace falcon {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// Murmur2 with a 4-byte key (bloom_filter.hpp:43-66)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t murmur2_keylen4(uint32_t key, uint32_t seed)
{
    const uint32_t m = 0x5bd1e995u;
    uint32_t k = key * m;
    k ^= k >> 24;
    k *= m;
    uint32_t h = (seed ^ 4u) * m;
    h ^= k;
    h ^= h >> 13;
    h *= m;
    h ^= h >> 15;
    return h;
}

// ---------------------------------------------------------------------------
// Element formats: EPS elements per 16-byte segment.
// ---------------------------------------------------------------------------
template <int ELEM> struct ET;
template <> struct ET<kF32> { static constexpr int EPS = 4; static constexpr int BYTES = 4; };
template <> struct ET<kBF16> { static constexpr int EPS = 8; static constexpr int BYTES = 2; };
template <> struct ET<kFP8> { static constexpr int EPS = 16; static constexpr int BYTES = 1; };

__device__ __forceinline__ uint4 ld_nc_v4(const void *p)
{
    uint4 r;
    asm("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
        : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
        : "l"(p));
    return r;
}

__device__ __forceinline__ int ld_nc_s32(const int32_t *p)
{
    int r;
    asm("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(r) : "l"(p));
    return r;
}

__device__ __forceinline__ float fp8_to_f32(uint32_t byte)
{
    __half_raw hr = __nv_cvt_fp8_to_halfraw((__nv_fp8_storage_t)byte, __NV_E4M3);
    return __half2float(__half(hr));
}

template <int ELEM>
__device__ __forceinline__ void decode_seg(const uint4 raw, float scale, float (&x)[ET<ELEM>::EPS])
{
    if constexpr (ELEM == kF32) {
        x[0] = __uint_as_float(raw.x);
        x[1] = __uint_as_float(raw.y);
        x[2] = __uint_as_float(raw.z);
        x[3] = __uint_as_float(raw.w);
    } else if constexpr (ELEM == kBF16) {
        const uint32_t w[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            x[2 * i] = __uint_as_float(w[i] << 16);
            x[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
        }
    } else {
        const uint32_t w[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
#pragma unroll
            for (int b = 0; b < 4; b++) x[4 * i + b] = __fmul_rn(fp8_to_f32((w[i] >> (8 * b)) & 0xffu), scale);
        }
    }
}

// Pairwise tree over the EPS squared differences of one segment: the lower
// levels of the reference's 16-leaf adder tree (compute.hpp:17-34).
template <int EPS>
__device__ __forceinline__ float seg_tree(const float (&q)[EPS], const float (&x)[EPS])
{
    float v[EPS];
#pragma unroll
    for (int i = 0; i < EPS; i++) {
        const float d = __fsub_rn(q[i], x[i]);
        v[i] = __fmul_rn(d, d);
    }
#pragma unroll
    for (int w = EPS; w > 1; w >>= 1) {
#pragma unroll
        for (int i = 0; i < w / 2; i++) v[i] = __fadd_rn(v[2 * i], v[2 * i + 1]);
    }
    return v[0];
}

// ---------------------------------------------------------------------------
// Distances of NB gathered vectors.  Lane l holds 16-byte segment l+32r of
// every vector.  The reference tree pairs adjacent leaves level by level, so
// the cross-lane levels are xor-butterflies over lane bits 0..4.  The first
// log2(NB) levels are done "transposed": at each level a lane keeps half of
// its vectors and receives the partner's partial of those, which adds the
// same operand pairs as the plain butterfly (IEEE addition is commutative)
// with fewer shuffles.  On return lane l holds the distance of vector l%NB.
// A pack is 256 leaves; packs are accumulated left to right
// (compute.hpp:260-267); zero leaves stand for the padding, which is exact.
// ---------------------------------------------------------------------------
template <int ELEM, int VROWS, int NB>
__device__ __forceinline__ float batch_distances(const float (&q)[VROWS][ET<ELEM>::EPS], const uint4 (&raw)[NB][VROWS],
                                                 const float (&scale)[NB], int lane)
{
    constexpr int EPS = ET<ELEM>::EPS;
    float rowv[VROWS];
#pragma unroll
    for (int r = 0; r < VROWS; r++) {
        float p[NB];
#pragma unroll
        for (int t = 0; t < NB; t++) {
            float x[EPS];
            decode_seg<ELEM>(raw[t][r], scale[t], x);
            p[t] = seg_tree<EPS>(q[r], x);
        }
        // transposed levels
        int level = 0;
#pragma unroll
        for (int w = NB; w > 1; w >>= 1, level++) {
            const bool hi = (lane >> level) & 1;
#pragma unroll
            for (int i = 0; i < w / 2; i++) {
                const float keep = hi ? p[2 * i + 1] : p[2 * i];
                const float send = hi ? p[2 * i] : p[2 * i + 1];
                p[i] = __fadd_rn(keep, __shfl_xor_sync(kFull, send, 1 << level));
            }
        }
        float v = p[0];
        constexpr int kLaneLevels = (ELEM == kFP8) ? 4 : 5;
#pragma unroll
        for (int lv = level; lv < kLaneLevels; lv++) v = __fadd_rn(v, __shfl_xor_sync(kFull, v, 1 << lv));
        rowv[r] = v;
    }
    float dist;
    if constexpr (ELEM == kF32) {
        // one row = 128 leaves = half a pack
#pragma unroll
        for (int pk = 0; pk < (VROWS + 1) / 2; pk++) {
            const float second = (2 * pk + 1 < VROWS) ? rowv[2 * pk + 1] : 0.0f;
            const float pack = __fadd_rn(rowv[2 * pk], second);
            dist = (pk == 0) ? pack : __fadd_rn(dist, pack);
        }
    } else if constexpr (ELEM == kBF16) {
        // one row = one pack
#pragma unroll
        for (int r = 0; r < VROWS; r++) dist = (r == 0) ? rowv[0] : __fadd_rn(dist, rowv[r]);
    } else {
        // one row = two packs: lanes 0-15 and lanes 16-31
#pragma unroll
        for (int r = 0; r < VROWS; r++) {
            const float other = __shfl_xor_sync(kFull, rowv[r], 16);
            const float lo = (lane < 16) ? rowv[r] : other;
            const float hi = (lane < 16) ? other : rowv[r];
            dist = (r == 0) ? lo : __fadd_rn(dist, lo);
            dist = __fadd_rn(dist, hi);
        }
    }
    return dist;
}

// ---------------------------------------------------------------------------
// Result queue: positions lane*EPL+e, sorted descending (position 0 = worst).
// One step = optional replacement of position 0, then step A (pairs 2j,2j+1)
// and step B (pairs 2j+1,2j+2) with swap iff q[a] < q[b]
// (priority_queue.hpp:29-57).  Returns whether this lane swapped anything.
// ---------------------------------------------------------------------------
template <int EPL>
__device__ __forceinline__ bool rq_step(float (&d)[EPL], int (&id)[EPL], int lane, bool replace, float nd, int nid)
{
    if (replace && lane == 0) { d[0] = nd; id[0] = nid; }
    bool sw = false;
#pragma unroll
    for (int e = 0; e + 1 < EPL; e += 2) {
        if (d[e] < d[e + 1]) {
            const float td = d[e]; d[e] = d[e + 1]; d[e + 1] = td;
            const int ti = id[e]; id[e] = id[e + 1]; id[e + 1] = ti;
            sw = true;
        }
    }
    // step B: lane-internal pairs (e, e+1), e odd; cross pair (last of lane, first of next lane)
    const float nb_d = __shfl_down_sync(kFull, d[0], 1);
    const int nb_i = __shfl_down_sync(kFull, id[0], 1);
    const float pv_d = __shfl_up_sync(kFull, d[EPL - 1], 1);
    const int pv_i = __shfl_up_sync(kFull, id[EPL - 1], 1);
#pragma unroll
    for (int e = 1; e + 1 < EPL; e += 2) {
        if (d[e] < d[e + 1]) {
            const float td = d[e]; d[e] = d[e + 1]; d[e + 1] = td;
            const int ti = id[e]; id[e] = id[e + 1]; id[e + 1] = ti;
            sw = true;
        }
    }
    if (lane < 31 && d[EPL - 1] < nb_d) { d[EPL - 1] = nb_d; id[EPL - 1] = nb_i; sw = true; }
    if (lane > 0 && pv_d < d[0]) { d[0] = pv_d; id[0] = pv_i; sw = true; }
    return sw;
}

// Candidate queue: position = lane (<= 32 entries).
__device__ __forceinline__ bool cq_step(float &d, int &id, int lane, bool replace, float nd, int nid)
{
    if (replace && lane == 0) { d = nd; id = nid; }
    bool sw = false;
    {   // step A: pairs (2j, 2j+1)
        const float pd = __shfl_xor_sync(kFull, d, 1);
        const int pi = __shfl_xor_sync(kFull, id, 1);
        const bool left = !(lane & 1);
        const bool swp = left ? (d < pd) : (pd < d);
        if (swp) { d = pd; id = pi; sw = true; }
    }
    {   // step B: pairs (2j+1, 2j+2)
        const float dn = __shfl_down_sync(kFull, d, 1);
        const int in = __shfl_down_sync(kFull, id, 1);
        const float du = __shfl_up_sync(kFull, d, 1);
        const int iu = __shfl_up_sync(kFull, id, 1);
        if (lane & 1) {
            if (lane < 31 && d < dn) { d = dn; id = in; sw = true; }
        } else if (lane > 0) {
            if (du < d) { d = du; id = iu; sw = true; }
        }
    }
    return sw;
}

// ---------------------------------------------------------------------------
// Bloom filter check of one 32-id chunk of the neighbour stream, with the
// sequential semantics of check_update (bloom_filter.hpp:159-200): a key is
// rejected iff all three of its bits were set by earlier keys.  Lanes read
// the filter, then set their bits with atomicOr; a bit that some other lane
// of this chunk set first is detected from the atomic's old value, and only
// then is the chunk resolved exactly by comparing against earlier lanes.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool bloom_chunk(uint32_t *words, uint32_t mask, uint32_t seed, int key, bool active, int lane)
{
    uint32_t h0 = 0, h1 = 0, h2 = 0;
    bool p0 = false, p1 = false, p2 = false;
    if (active) {
        h0 = murmur2_keylen4((uint32_t)key, seed) & mask;
        h1 = murmur2_keylen4((uint32_t)key, seed + 1u) & mask;
        h2 = murmur2_keylen4((uint32_t)key, seed + 2u) & mask;
        p0 = (words[h0 >> 5] >> (h0 & 31)) & 1u;
        p1 = (words[h1 >> 5] >> (h1 & 31)) & 1u;
        p2 = (words[h2 >> 5] >> (h2 & 31)) & 1u;
    }
    __syncwarp();
    bool coll = false;
    if (active) {
        uint32_t o;
        o = atomicOr(&words[h0 >> 5], 1u << (h0 & 31)); coll |= ((o >> (h0 & 31)) & 1u) && !p0;
        o = atomicOr(&words[h1 >> 5], 1u << (h1 & 31)); coll |= ((o >> (h1 & 31)) & 1u) && !p1;
        o = atomicOr(&words[h2 >> 5], 1u << (h2 & 31)); coll |= ((o >> (h2 & 31)) & 1u) && !p2;
    }
    if (__any_sync(kFull, coll)) {
        const unsigned act_mask = __ballot_sync(kFull, active);
        for (int src = 0; src < 31; src++) {
            const uint32_t a = __shfl_sync(kFull, h0, src);
            const uint32_t b = __shfl_sync(kFull, h1, src);
            const uint32_t c = __shfl_sync(kFull, h2, src);
            if (((act_mask >> src) & 1u) && src < lane) {
                p0 |= (h0 == a) | (h0 == b) | (h0 == c);
                p1 |= (h1 == a) | (h1 == b) | (h1 == c);
                p2 |= (h2 == a) | (h2 == b) | (h2 == c);
            }
        }
    }
    __syncwarp();
    return active && !(p0 && p1 && p2);
}

// ---------------------------------------------------------------------------
// One query, inter-query semantics (v1.3).
// ---------------------------------------------------------------------------
template <int ELEM, int EPL, int VROWS>
__device__ void search_one_inter(const SearchLaunch &A, const QParams &P, int64_t qi, uint32_t *bloom, int *fifo,
                                 int *fifo_len, int *sids, int lane)
{
    constexpr int EPS = ET<ELEM>::EPS;
    constexpr int NB = (VROWS == 1) ? 8 : 4;
    const GraphView &g = A.g;
    const int nseg = g.dpad * ET<ELEM>::BYTES / 16;

    float q[VROWS][EPS];
    {
        const float *Q = A.queries + qi * A.qstride;
#pragma unroll
        for (int r = 0; r < VROWS; r++) {
            const int seg = lane + 32 * r;
#pragma unroll
            for (int e = 0; e < EPS; e++) {
                const int j = seg * EPS + e;
                q[r][e] = (seg < nseg && j < g.dim) ? Q[j] : 0.0f;
            }
        }
    }
    {   // reset this query's Bloom filter
        const int nvec = 1 << (P.bloom_bits - 5 - 2);
        uint4 *b4 = reinterpret_cast<uint4 *>(bloom);
        for (int i = lane; i < nvec; i += 32) b4[i] = make_uint4(0, 0, 0, 0);
    }
    const uint32_t bmask = (1u << P.bloom_bits) - 1u;

    float rd[EPL];
    int ri[EPL];
#pragma unroll
    for (int e = 0; e < EPL; e++) {
        rd[e] = (lane * EPL + e < P.ef) ? kLarge : -kLarge;
        ri[e] = -1;
    }
    float cd = (lane < P.cq) ? kLarge : -kLarge;
    int ci = -1;
    bool r_sorted = true, c_sorted = true;
    float rq0 = kLarge, cq0 = kLarge;

    int entry = A.entries ? A.entries[qi] : A.default_entry;
    const int mc = P.mc, mg = P.mg;
    int head = 0, inflight = 1, hops = 1, visited = 0;
    if (entry < 0 || (int64_t)entry >= g.n) {   // bad entry from a device-memory caller: empty result
        if (lane == 0) atomicOr(A.status, 2);
        entry = 0;
        inflight = 0;
        hops = 0;
    }
    if (lane == 0) { fifo[0] = entry; fifo_len[0] = 1; }
    __syncwarp();
    bool truncated = false;

    while (inflight > 0) {
        const int glen = fifo_len[head];
        for (int b = 0; b < glen; b++) {
            const int node = fifo[head * mc + b];
            const int32_t *row = g.links + (int64_t)node * g.lstride;
            const int cnt = ld_nc_s32(row);
            for (int c0 = 0; c0 < cnt; c0 += 32) {
                const bool act = c0 + lane < cnt;
                const int nb = act ? ld_nc_s32(row + g.ids_off + c0 + lane) : -1;
                const bool valid = bloom_chunk(bloom, bmask, P.seed, nb, act, lane);
                const unsigned vm = __ballot_sync(kFull, valid);
                const int V = __popc(vm);
                visited += V;
                if (valid) sids[__popc(vm & ((1u << lane) - 1u))] = nb;
                __syncwarp();
                for (int b0 = 0; b0 < V; b0 += NB) {
                    uint4 raw[NB][VROWS];
                    float scale[NB];
#pragma unroll
                    for (int t = 0; t < NB; t++) {
                        const bool tv = b0 + t < V;
                        const int id = tv ? sids[b0 + t] : 0;
                        const unsigned char *base = g.vecs + (int64_t)id * g.vstride_bytes;
                        scale[t] = 1.0f;
                        if constexpr (ELEM == kFP8) scale[t] = tv ? g.scales[id] : 1.0f;
#pragma unroll
                        for (int r = 0; r < VROWS; r++) {
                            const int seg = lane + 32 * r;
                            raw[t][r] = (tv && seg < nseg) ? ld_nc_v4(base + 16 * seg) : make_uint4(0, 0, 0, 0);
                        }
                    }
                    const float dist = batch_distances<ELEM, VROWS, NB>(q, raw, scale, lane);
                    const int nt = min(NB, V - b0);
                    for (int t = 0; t < nt; t++) {
                        const float d = __shfl_sync(kFull, dist, t);
                        const int id = sids[b0 + t];
                        const bool ins = d < rq0;
                        if (!r_sorted || ins) {
                            const bool sw = rq_step<EPL>(rd, ri, lane, ins, d, id);
                            r_sorted = !__any_sync(kFull, sw);
                            rq0 = __shfl_sync(kFull, rd[0], 0);
                        }
                        if (ins) {   // forwarded to the scheduler's candidate queue (insert_only)
                            const bool cins = d < cq0;
                            if (!c_sorted || cins) {
                                const bool sw = cq_step(cd, ci, lane, cins, d, id);
                                c_sorted = !__any_sync(kFull, sw);
                                cq0 = __shfl_sync(kFull, cd, 0);
                            }
                        }
                    }
                }
                __syncwarp();
            }
        }
        // the oldest group is retired: sort both queues, read the threshold
        while (!r_sorted) {
            const bool sw = rq_step<EPL>(rd, ri, lane, false, 0.0f, 0);
            r_sorted = !__any_sync(kFull, sw);
        }
        rq0 = __shfl_sync(kFull, rd[0], 0);
        const float thr = rq0;
        head = (head + 1 == mg) ? 0 : head + 1;
        inflight--;
        while (!c_sorted) {
            const bool sw = cq_step(cd, ci, lane, false, 0.0f, 0);
            c_sorted = !__any_sync(kFull, sw);
        }
        // refill the pipeline with groups of up to mc candidates
        for (int oid = inflight; oid < mg && !truncated; oid++) {
            int slot = head + inflight;
            if (slot >= mg) slot -= mg;
            int n = 0;
            for (int bb = 0; bb < mc; bb++) {
                const float best = __shfl_sync(kFull, cd, P.cq - 1);
                if (!(best <= thr && best < kLarge)) break;
                if (P.max_hops > 0 && hops >= P.max_hops) { truncated = true; break; }
                const int pid = __shfl_sync(kFull, ci, P.cq - 1);
                const float ud = __shfl_up_sync(kFull, cd, 1);
                const int ui = __shfl_up_sync(kFull, ci, 1);
                if (lane < P.cq) {
                    cd = (lane == 0) ? kLarge : ud;
                    ci = (lane == 0) ? -1 : ui;
                }
                if (lane == 0) fifo[slot * mc + n] = pid;
                n++;
                hops++;
            }
            if (n == 0) break;
            if (lane == 0) fifo_len[slot] = n;
            inflight++;
        }
        cq0 = __shfl_sync(kFull, cd, 0);
        __syncwarp();
    }

    // results best-first: result i is position ef-1-i (DRAM_utils.hpp:460-464)
    const int nwrite = A.write_all_ef ? P.ef : P.k;
    int32_t *oid_row = A.out_ids + qi * A.out_stride;
    float *od_row = A.out_d + qi * A.out_stride;
#pragma unroll
    for (int e = 0; e < EPL; e++) {
        const int pos = lane * EPL + e;
        if (pos < P.ef) {
            const int i = P.ef - 1 - pos;
            if (i < nwrite) {
                int id = ri[e];
                if (!A.write_all_ef && g.labels && id >= 0) id = g.labels[id];
                oid_row[i] = id;
                od_row[i] = rd[e];
            }
        }
    }
    for (int i = nwrite + lane; i < A.out_stride; i += 32) { oid_row[i] = -1; od_row[i] = kLarge; }
    if (lane == 0) {
        if (A.out_hops) A.out_hops[qi] = hops;
        if (A.out_visited) A.out_visited[qi] = visited;
        if (truncated) atomicOr(A.status, 1);
    }
}

__device__ __forceinline__ size_t warp_smem_bytes(int bloom_bits_max, int mc_max, int mg_max)
{
    size_t b = (size_t)1 << (bloom_bits_max - 3);
    b += sizeof(int) * (size_t)(mc_max * mg_max + mg_max + 32);
    return (b + 15) & ~(size_t)15;
}

template <int ELEM, int EPL, int VROWS>
__global__ void __launch_bounds__(128) inter_kernel(const SearchLaunch A)
{
    extern __shared__ uint4 smem_u4[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t wbytes = warp_smem_bytes(A.bloom_bits_max, A.mc_max, A.mg_max);
    unsigned char *wbase = reinterpret_cast<unsigned char *>(smem_u4) + wbytes * warp;
    uint32_t *bloom = reinterpret_cast<uint32_t *>(wbase);
    int *fifo = reinterpret_cast<int *>(wbase + ((size_t)1 << (A.bloom_bits_max - 3)));
    int *fifo_len = fifo + A.mc_max * A.mg_max;
    int *sids = fifo_len + A.mg_max;
    for (;;) {
        unsigned long long qi = 0;
        if (lane == 0) qi = atomicAdd(reinterpret_cast<unsigned long long *>(A.work_counter), 1ull);
        qi = __shfl_sync(kFull, qi, 0);
        if (qi >= (unsigned long long)A.nq) break;
        const QParams P = A.params[A.per_query ? qi : 0];
        search_one_inter<ELEM, EPL, VROWS>(A, P, (int64_t)qi, bloom, fifo, fifo_len, sids, lane);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Exact FP32 rerank of the final ef candidates of a reduced-precision
// traversal (extension beyond the reference): one warp per query, the same
// adder tree on the FP32 vectors, stable ascending order (ties keep the
// traversal order), top k written with labels.
// ---------------------------------------------------------------------------
template <int VROWS>
__global__ void __launch_bounds__(128) rerank_kernel(const RerankLaunch A)
{
    __shared__ float sd[4][kMaxEf];
    __shared__ int si[4][kMaxEf];
    constexpr int NB = (VROWS == 1) ? 8 : 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const GraphView &g = A.g;
    const int nseg = g.dpad * 4 / 16;
    for (int64_t qi = (int64_t)blockIdx.x * 4 + warp; qi < A.nq; qi += (int64_t)gridDim.x * 4) {
        const QParams P = A.params[A.per_query ? qi : 0];
        float q[VROWS][4];
        const float *Q = A.queries + qi * A.qstride;
#pragma unroll
        for (int r = 0; r < VROWS; r++) {
            const int seg = lane + 32 * r;
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int j = seg * 4 + e;
                q[r][e] = (seg < nseg && j < g.dim) ? Q[j] : 0.0f;
            }
        }
        const int32_t *cand = A.cand_ids + qi * A.cand_stride;
        for (int b0 = 0; b0 < P.ef; b0 += NB) {
            uint4 raw[NB][VROWS];
            float scale[NB];
            int ids[NB];
#pragma unroll
            for (int t = 0; t < NB; t++) {
                const bool tv = b0 + t < P.ef;
                ids[t] = tv ? cand[b0 + t] : -1;
                const int id = ids[t] >= 0 ? ids[t] : 0;
                scale[t] = 1.0f;
                const unsigned char *base = g.vecs32 + (int64_t)id * g.vstride32_bytes;
#pragma unroll
                for (int r = 0; r < VROWS; r++) {
                    const int seg = lane + 32 * r;
                    raw[t][r] = (ids[t] >= 0 && seg < nseg) ? ld_nc_v4(base + 16 * seg) : make_uint4(0, 0, 0, 0);
                }
            }
            const float dist = batch_distances<kF32, VROWS, NB>(q, raw, scale, lane);
            if (lane < NB && b0 + lane < P.ef) {
                const int id = ids[lane];
                sd[warp][b0 + lane] = (id >= 0) ? dist : kLarge;
                si[warp][b0 + lane] = id;
            }
        }
        __syncwarp();
        int32_t *orow = A.out_ids + qi * A.out_stride;
        float *drow = A.out_d + qi * A.out_stride;
        for (int i = lane; i < P.ef; i += 32) {
            const float di = sd[warp][i];
            int rank = 0;
            for (int j = 0; j < P.ef; j++) {
                const float dj = sd[warp][j];
                rank += (dj < di) || (dj == di && j < i);
            }
            if (rank < P.k) {
                int id = si[warp][i];
                if (g.labels && id >= 0) id = g.labels[id];
                orow[rank] = id;
                drow[rank] = di;
            }
        }
        for (int i = P.k + lane; i < A.out_stride; i += 32) { orow[i] = -1; drow[i] = kLarge; }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Storage encoders (index creation).
// ---------------------------------------------------------------------------
__global__ void encode_bf16_kernel(const float *src, int64_t src_stride, int64_t n, int dim, int dpad, uint16_t *dst)
{
    const int64_t total = n * dpad;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = t / dpad;
        const int j = (int)(t - r * dpad);
        const float v = (j < dim) ? src[r * src_stride + j] : 0.0f;
        __nv_bfloat16 h = __float2bfloat16_rn(v);
        dst[t] = *reinterpret_cast<uint16_t *>(&h);
    }
}

// FP8 E4M3 with one scale per vector: scale = max|x| / 448 (448 = largest
// finite E4M3), code = saturating round-to-nearest of x / scale.
__global__ void encode_fp8_kernel(const float *src, int64_t src_stride, int64_t n, int dim, int dpad, uint8_t *dst,
                                  float *scales)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int64_t r = warp; r < n; r += nwarps) {
        float amax = 0.0f;
        for (int j = lane; j < dim; j += 32) amax = fmaxf(amax, fabsf(src[r * src_stride + j]));
        for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(kFull, amax, o));
        const float scale = (amax > 0.0f) ? __fdiv_rn(amax, 448.0f) : 1.0f;
        if (lane == 0) scales[r] = scale;
        for (int j = lane; j < dpad; j += 32) {
            const float v = (j < dim) ? __fdiv_rn(src[r * src_stride + j], scale) : 0.0f;
            dst[r * dpad + j] = (uint8_t)__nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
        }
    }
}

template <int ELEM, int EPL, int VROWS>
cudaError_t launch_inter(const SearchLaunch &a, size_t smem_block, int num_sms, cudaStream_t s)
{
    auto kern = inter_kernel<ELEM, EPL, VROWS>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_block);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem_block);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int64_t blocks = (int64_t)per_sm * num_sms;
    const int64_t need = (a.nq + 3) / 4;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    kern<<<(unsigned)blocks, 128, smem_block, s>>>(a);
    return cudaGetLastError();
}

template <int ELEM, int VROWS>
cudaError_t dispatch_epl(const SearchLaunch &a, size_t smem_block, int num_sms, cudaStream_t s)
{
    if (a.ef_max <= 64) return launch_inter<ELEM, 2, VROWS>(a, smem_block, num_sms, s);
    if (a.ef_max <= 128) return launch_inter<ELEM, 4, VROWS>(a, smem_block, num_sms, s);
    return launch_inter<ELEM, 8, VROWS>(a, smem_block, num_sms, s);
}

}  // namespace

cudaError_t launch_search(const SearchLaunch &a, int elem, int num_sms, cudaStream_t s)
{
    const size_t wbytes = ((((size_t)1 << (a.bloom_bits_max - 3)) +
                            sizeof(int) * (size_t)(a.mc_max * a.mg_max + a.mg_max + 32)) + 15) & ~(size_t)15;
    const size_t smem_block = wbytes * 4;
    const int seg_bytes = (elem == kF32) ? 4 : (elem == kBF16 ? 2 : 1);
    const int nseg = a.g.dpad * seg_bytes / 16;
    const int vrows = (nseg + 31) / 32;
    if (elem == kF32) {
        switch (vrows) {
            case 1: return dispatch_epl<kF32, 1>(a, smem_block, num_sms, s);
            case 2: return dispatch_epl<kF32, 2>(a, smem_block, num_sms, s);
            case 3: return dispatch_epl<kF32, 3>(a, smem_block, num_sms, s);
            case 4: return dispatch_epl<kF32, 4>(a, smem_block, num_sms, s);
        }
    } else if (elem == kBF16) {
        switch (vrows) {
            case 1: return dispatch_epl<kBF16, 1>(a, smem_block, num_sms, s);
            case 2: return dispatch_epl<kBF16, 2>(a, smem_block, num_sms, s);
        }
    } else if (elem == kFP8) {
        if (vrows == 1) return dispatch_epl<kFP8, 1>(a, smem_block, num_sms, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_rerank(const RerankLaunch &a, int ef_max, int num_sms, cudaStream_t s)
{
    (void)ef_max;
    const int vrows = (a.g.dpad * 4 / 16 + 31) / 32;
    int64_t blocks = (a.nq + 3) / 4;
    const int64_t cap = (int64_t)num_sms * 16;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    switch (vrows) {
        case 1: rerank_kernel<1><<<(unsigned)blocks, 128, 0, s>>>(a); break;
        case 2: rerank_kernel<2><<<(unsigned)blocks, 128, 0, s>>>(a); break;
        case 3: rerank_kernel<3><<<(unsigned)blocks, 128, 0, s>>>(a); break;
        case 4: rerank_kernel<4><<<(unsigned)blocks, 128, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_encode_bf16(const float *src, int64_t src_stride, int64_t n, int dim, int dpad, uint16_t *dst,
                               cudaStream_t s)
{
    encode_bf16_kernel<<<1184, 256, 0, s>>>(src, src_stride, n, dim, dpad, dst);
    return cudaGetLastError();
}

cudaError_t launch_encode_fp8(const float *src, int64_t src_stride, int64_t n, int dim, int dpad, uint8_t *dst,
                              float *scales, cudaStream_t s)
{
    encode_fp8_kernel<<<1184, 256, 0, s>>>(src, src_stride, n, dim, dpad, dst, scales);
    return cudaGetLastError();
}

}  // namespace falcon
