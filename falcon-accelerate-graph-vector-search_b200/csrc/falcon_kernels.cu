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

// Prefetch the 128-byte lines of [p, p + bytes) into L2 (one instruction per
// line from this lane; cheaper to issue than a bulk prefetch per range).
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes)
{
    const char *c = reinterpret_cast<const char *>(p);
    for (uint32_t o = 0; o < bytes; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(c + o) : "memory");
}

__device__ __forceinline__ int ld_nc_s32(const int32_t *p)
{
    int r;
    asm("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(r) : "l"(p));
    return r;
}

// Paired FP32 add and multiply (sm_100 f32x2): each half rounded to nearest
// like __fadd_rn / __fmul_rn.  The explicit .rn keeps the code generator from
// fusing a multiply into a following add, which would round once instead of
// twice and change the distance bits.
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b)
{
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

__device__ __forceinline__ float2 mul2_rn(float2 a, float2 b)
{
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
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
        // two codes per conversion (E4M3 -> f16 -> f32 is exact), then the scale
        const uint32_t w[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const __half2_raw hr =
                    __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)((w[i] >> (16 * h)) & 0xffffu), __NV_E4M3);
                const float2 f = __half22float2(__half2(hr));
                x[4 * i + 2 * h] = __fmul_rn(f.x, scale);
                x[4 * i + 2 * h + 1] = __fmul_rn(f.y, scale);
            }
        }
    }
}

// Pairwise tree over the EPS squared differences of one segment: the lower
// levels of the reference's 16-leaf adder tree (compute.hpp:17-34).  nq is
// the NEGATED query: x + (-q) is exactly -(q - x), whose square has the same
// bits as (q - x)^2, so the differences and squares of adjacent leaves run as
// paired operations.
template <int EPS>
__device__ __forceinline__ float seg_tree(const float (&nq)[EPS], const float (&x)[EPS])
{
    float v[EPS];
#pragma unroll
    for (int i = 0; i < EPS; i += 2) {
        const float2 d = add2_rn(make_float2(x[i], x[i + 1]), make_float2(nq[i], nq[i + 1]));
        const float2 s = mul2_rn(d, d);
        v[i] = s.x;
        v[i + 1] = s.y;
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
//
// Lane groups: when a vector has at most 16 segments (VROWS == 1) the warp
// holds 32/G vectors per register row, lanes [gG, gG+G) holding vector g, with
// G = 2^lg >= NB.  The levels above lane bit lg-1 would only add the zero
// leaves of the padding (every partial is a sum of squares, >= +0, so x + 0
// is x exactly), so the tree stops at bit lg-1.  lg = 5 is the plain layout.
// On return lane l holds the distance of row l%NB of group l>>lg.
// ---------------------------------------------------------------------------
template <int ELEM, int VROWS, int NB>
__device__ __forceinline__ float batch_distances(const float (&nq)[VROWS][ET<ELEM>::EPS], const uint4 (&raw)[NB][VROWS],
                                                 const float (&scale)[NB], int lane, int lg = 5)
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
            p[t] = seg_tree<EPS>(nq[r], x);
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
        const int top = min(kLaneLevels, lg);
#pragma unroll
        for (int lv = level; lv < kLaneLevels; lv++)
            if (lv < top) v = __fadd_rn(v, __shfl_xor_sync(kFull, v, 1 << lv));
        rowv[r] = v;
    }
    if (VROWS == 1 && lg < 5) return rowv[0];   // one vector per group: the rest of the tree adds zeros
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
// Queues.  The reference keeps both queues in a systolic odd-even array
// (priority_queue.hpp:9-166): an insertion replaces q[0] when the new distance
// is smaller, then runs one even and one odd compare-swap phase; sort() runs
// n phases.  That array holds its maximum in q[0] whenever an insertion is
// tested, so it behaves entry for entry like a list sorted by
// (distance, insertion age) in which an insertion happens iff d < max and
// evicts the newest of the max-valued entries, and sort() leaves equal
// distances oldest first.  Proof sketch: every operation is a min or a max,
// so by the 0/1 principle it is enough to look at 0/1 arrays; there, at the
// start of every step the zeros that precede the last 1 sit at even positions
// >= 2 with 1s on both sides, an invariant that replacement at q[0] followed
// by the two phases preserves, hence q[0] = 1 whenever any 1 is present, i.e.
// q[0] is the maximum.  Equal distances never swap, so they keep insertion
// order.  The same holds for the v1.5 variant (phases only after a
// replacement) and for pop_top (after a sort).  The kernels therefore hold the
// queues as sorted lists: a distance that is not below the current maximum
// costs one comparison.
//
// Result list: position p = lane*EPL + e in ascending order; positions >= ef
// hold evicted entries, which stay above every later insertion because the
// maximum never increases.
//
// Insertion after the entries <= x, decided per entry from local values: an
// entry <= x stays; an entry > x takes x if its predecessor is <= x (it is the
// first entry above x), else its predecessor's value.  The predecessor of a
// lane's first entry is the previous lane's last entry (one shfl_up, which
// does not depend on x); lane 0's first entry has none.
// ---------------------------------------------------------------------------
template <int EPL>
__device__ __forceinline__ void list_insert(float (&d)[EPL], int (&id)[EPL], int lane, int lim, float x, int xid)
{
    float pd = __shfl_up_sync(kFull, d[EPL - 1], 1);
    const int pi = __shfl_up_sync(kFull, id[EPL - 1], 1);
    if (lane == 0) pd = -kLarge;
#pragma unroll
    for (int e = EPL - 1; e >= 0; e--) {
        const float prev = (e == 0) ? pd : d[(e > 0) ? e - 1 : 0];
        const int previ = (e == 0) ? pi : id[(e > 0) ? e - 1 : 0];
        if (lane * EPL + e < lim && !(d[e] <= x)) {
            const bool at = prev <= x;
            d[e] = at ? x : prev;
            id[e] = at ? xid : previ;
        }
    }
}

template <int EPL>
__device__ __forceinline__ void rl_insert(float (&d)[EPL], int (&id)[EPL], int lane, float x, int xid)
{
    list_insert<EPL>(d, id, lane, 32 * EPL, x, xid);
}

// Value at warp-uniform position p of the result list.
template <int EPL>
__device__ __forceinline__ float rl_get(const float (&d)[EPL], int p)
{
    const int e0 = p % EPL;
    float v = d[0];
#pragma unroll
    for (int e = 1; e < EPL; e++) v = (e == e0) ? d[e] : v;
    return __shfl_sync(kFull, v, p / EPL);
}

// Candidate list: position p = lane*CPL + e < cq, ascending; positions >= cq
// are ignored (they may hold stale entries after pops).
template <int CPL>
__device__ __forceinline__ void cl_insert(float (&d)[CPL], int (&id)[CPL], int lane, int cq, float x, int xid)
{
    list_insert<CPL>(d, id, lane, cq, x, xid);
}

// pop_top (priority_queue.hpp:131-165): take the best entry, a +large
// placeholder enters at the worst end.
template <int CPL>
__device__ __forceinline__ int cl_pop(float (&d)[CPL], int (&id)[CPL], int lane, int cq)
{
    const int pid = __shfl_sync(kFull, id[0], 0);
    const float nd = __shfl_down_sync(kFull, d[0], 1);
    const int ni = __shfl_down_sync(kFull, id[0], 1);
#pragma unroll
    for (int e = 0; e < CPL; e++) {
        const int p = lane * CPL + e;
        const float sd = (e + 1 < CPL) ? d[(e + 1 < CPL) ? e + 1 : 0] : nd;
        const int si = (e + 1 < CPL) ? id[(e + 1 < CPL) ? e + 1 : 0] : ni;
        if (p < cq - 1) { d[e] = sd; id[e] = si; }
        else if (p == cq - 1) { d[e] = kLarge; id[e] = -1; }
    }
    return pid;
}

template <int EPL> struct CandPerLane { static constexpr int value = (EPL >= 8) ? EPL / 4 : 1; };

// For ef > 256 the result list is held in shared memory as keys
// (distance bits, insertion age) instead of 32 entries per lane in registers.
// Only the maximum matters while searching -- it is the entry the
// sorted-list model evicts: the largest distance and, among equal distances,
// the newest -- and a final sort by key gives the list order (ties oldest
// first).  Distances are >= +0, so their bit patterns order like the floats.
//
// The ef slots form 32 buckets of BSZ (= EPL) consecutive slots; lane l keeps
// bucket l's maximum key and slot in registers and the warp keeps the global
// maximum.  Replacing the maximum rewrites one slot, re-reduces that bucket
// (one slot per lane) and then the 32 bucket maxima: a handful of warp
// reductions instead of a walk down a heap.  Slots at or past ef hold key 0,
// below every real key (ages start at 1; placeholders carry 1e20).
__device__ __forceinline__ uint64_t heap_key(float d, uint32_t age)
{
    return ((uint64_t)__float_as_uint(d) << 32) | age;
}

struct BucketMax {
    uint64_t bmax;      // this lane's bucket maximum
    int bslot;          // its slot within the bucket
    uint64_t gmax;      // global maximum (warp-uniform)
    int gb, gslot;      // its bucket and slot (warp-uniform)
};

__device__ __forceinline__ void bucket_global(BucketMax &B)
{
    const uint32_t hi = (uint32_t)(B.bmax >> 32);
    const uint32_t mhi = __reduce_max_sync(kFull, hi);
    const uint32_t mlo = __reduce_max_sync(kFull, hi == mhi ? (uint32_t)B.bmax : 0u);
    B.gmax = ((uint64_t)mhi << 32) | mlo;
    B.gb = __ffs(__ballot_sync(kFull, B.bmax == B.gmax)) - 1;
    B.gslot = __shfl_sync(kFull, B.bslot, B.gb);
}

// ef placeholders (1e20, age 0), slots up to 32*BSZ cleared.
template <int BSZ>
__device__ __forceinline__ void bucket_init(BucketMax &B, uint64_t *key, int *id, int ef, int lane)
{
    for (int i = lane; i < 32 * BSZ; i += 32) { key[i] = (i < ef) ? heap_key(kLarge, 0u) : 0ull; id[i] = -1; }
    B.bmax = (BSZ * lane < ef) ? heap_key(kLarge, 0u) : 0ull;
    B.bslot = 0;
    __syncwarp();
    bucket_global(B);
}

// Replace the maximum by k < maximum; returns the new maximum's distance.
template <int BSZ>
__device__ __forceinline__ float bucket_replace_max(BucketMax &B, uint64_t *key, int *id, uint64_t k, int kid, int lane)
{
    const int slot = BSZ * B.gb + lane;
    const uint64_t old = (lane < BSZ) ? key[slot] : 0ull;
    const uint64_t ck = (lane == B.gslot) ? k : old;
    if (lane == B.gslot) { key[slot] = k; id[slot] = kid; }
    const uint32_t hi = (uint32_t)(ck >> 32);
    const uint32_t mhi = __reduce_max_sync(kFull, hi);
    const uint32_t mlo = __reduce_max_sync(kFull, hi == mhi ? (uint32_t)ck : 0u);
    const uint64_t mk = ((uint64_t)mhi << 32) | mlo;
    const int src = __ffs(__ballot_sync(kFull, ck == mk)) - 1;
    if (lane == B.gb) { B.bmax = mk; B.bslot = src; }
    bucket_global(B);
    __syncwarp();
    return __uint_as_float((uint32_t)(B.gmax >> 32));
}

// Ascending bitonic sort of the first n2 (a power of two) keys, ids alongside.
__device__ __forceinline__ void warp_bitonic_sort(uint64_t *key, int *id, int n2, int lane)
{
    for (int size = 2; size <= n2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < n2 / 2; t += 32) {
                const int lo = 2 * t - (t & (stride - 1));
                const int hi = lo + stride;
                const bool up = ((lo & size) == 0);
                const uint64_t a = key[lo], b = key[hi];
                if ((a > b) == up) {
                    key[lo] = b; key[hi] = a;
                    const int ia = id[lo]; id[lo] = id[hi]; id[hi] = ia;
                }
            }
            __syncwarp();
        }
    }
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
    if (active) {   // bits that were already set need no atomic (and dirty no line)
        uint32_t o;
        if (!p0) { o = atomicOr(&words[h0 >> 5], 1u << (h0 & 31)); coll |= (o >> (h0 & 31)) & 1u; }
        if (!p1) { o = atomicOr(&words[h1 >> 5], 1u << (h1 & 31)); coll |= (o >> (h1 & 31)) & 1u; }
        if (!p2) { o = atomicOr(&words[h2 >> 5], 1u << (h2 & 31)); coll |= (o >> (h2 & 31)) & 1u; }
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

// Bloom check of a whole adjacency row of up to 64 ids (lane l holds ids l
// and 32+l), same sequential semantics as bloom_chunk.  The filter bits of
// all ids are read first and give a provisional answer; the atomics that set
// the clear bits are issued at once but their old values are only examined by
// bloom_row_resolve, after the caller has issued its vector gathers, so the
// atomic round trip overlaps the gathers.  A collision (a bit set first by
// another id of this row) can only turn a provisional "new" into "seen".
struct BloomRow {
    uint32_t h[2][3];
    bool pre[2][3];
    uint32_t old[2][3];
    bool act[2];
};

__device__ __forceinline__ void bloom_row_begin(BloomRow &B, uint32_t *words, uint32_t mask, uint32_t seed,
                                                int k0, int k1, bool a0, bool a1, bool &prov0, bool &prov1)
{
    B.act[0] = a0;
    B.act[1] = a1;
    const int key[2] = {k0, k1};
#pragma unroll
    for (int c = 0; c < 2; c++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            B.h[c][j] = B.act[c] ? (murmur2_keylen4((uint32_t)key[c], seed + (uint32_t)j) & mask) : 0u;
            B.pre[c][j] = B.act[c] ? (((words[B.h[c][j] >> 5] >> (B.h[c][j] & 31)) & 1u) != 0) : true;
        }
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < 2; c++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            B.old[c][j] = 0u;
            if (B.act[c] && !B.pre[c][j]) B.old[c][j] = atomicOr(&words[B.h[c][j] >> 5], 1u << (B.h[c][j] & 31));
        }
    }
    prov0 = a0 && !(B.pre[0][0] && B.pre[0][1] && B.pre[0][2]);
    prov1 = a1 && !(B.pre[1][0] && B.pre[1][1] && B.pre[1][2]);
}

// Exact validity (sequential semantics) of the two ids of this lane.
__device__ __forceinline__ void bloom_row_resolve(BloomRow &B, int lane, bool &v0, bool &v1)
{
    bool coll = false;
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            coll |= B.act[c] && !B.pre[c][j] && ((B.old[c][j] >> (B.h[c][j] & 31)) & 1u);
    bool s[2][3];
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
        for (int j = 0; j < 3; j++) s[c][j] = B.pre[c][j];
    if (__any_sync(kFull, coll)) {
        const unsigned am0 = __ballot_sync(kFull, B.act[0]);
        const unsigned am1 = __ballot_sync(kFull, B.act[1]);
        for (int src = 0; src < 32; src++) {
            uint32_t t0[3], t1[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                t0[j] = __shfl_sync(kFull, B.h[0][j], src);
                t1[j] = __shfl_sync(kFull, B.h[1][j], src);
            }
            const bool src0 = (am0 >> src) & 1u, src1 = (am1 >> src) & 1u;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                // first-half id of this lane: earlier ids are first-half ids of lower lanes
                if (src0 && src < lane) s[0][j] |= (B.h[0][j] == t0[0]) | (B.h[0][j] == t0[1]) | (B.h[0][j] == t0[2]);
                // second-half id: every first-half id, and second-half ids of lower lanes
                if (src0) s[1][j] |= (B.h[1][j] == t0[0]) | (B.h[1][j] == t0[1]) | (B.h[1][j] == t0[2]);
                if (src1 && src < lane) s[1][j] |= (B.h[1][j] == t1[0]) | (B.h[1][j] == t1[1]) | (B.h[1][j] == t1[2]);
            }
        }
    }
    v0 = B.act[0] && !(s[0][0] && s[0][1] && s[0][2]);
    v1 = B.act[1] && !(s[1][0] && s[1][1] && s[1][2]);
    __syncwarp();
}

// ---------------------------------------------------------------------------
// One query, inter-query semantics (v1.3).
// ---------------------------------------------------------------------------
// Issue the gathers of stream slots b0 .. b0+(32>>lg)*NB-1 (of n) of the
// staged ids.  Slot b0 + gNB + t goes to register row t of lane group g (lanes
// [g<<lg, (g+1)<<lg)), whose lane l loads 16-byte segment (l mod 2^lg)+32r.
// Slots past n, and slots whose id was withdrawn (stored as ~id < 0), load
// nothing and read as zeros.
template <int ELEM, int VROWS, int NB>
__device__ __forceinline__ void gather_batch(const GraphView &g, const int *sids, int b0, int n, int nseg, int lane,
                                             int lg, uint4 (&raw)[NB][VROWS], float (&scale)[NB])
{
    const int s0 = b0 + (lane >> lg) * NB;
    const int lseg = lane & ((1 << lg) - 1);
#pragma unroll
    for (int t = 0; t < NB; t++) {
        const int sid = (s0 + t < n) ? sids[s0 + t] : -1;
        const bool tv = sid >= 0;
        const int id = tv ? sid : 0;
        const unsigned char *base = g.vecs + (int64_t)id * g.vstride_bytes;
        scale[t] = 1.0f;
        if constexpr (ELEM == kFP8) scale[t] = tv ? g.scales[id] : 1.0f;
#pragma unroll
        for (int r = 0; r < VROWS; r++) {
            const int seg = lseg + 32 * r;
            raw[t][r] = (tv && seg < nseg) ? ld_nc_v4(base + 16 * seg) : make_uint4(0, 0, 0, 0);
        }
    }
}

// Lane-group size (log2) for vectors of nseg 16-byte segments: the smallest
// power of two >= max(nseg, NB) when one register row holds the vector,
// otherwise the whole warp.
template <int VROWS, int NB>
__device__ __forceinline__ int lane_group_log2(int nseg)
{
    if (VROWS > 1) return 5;
    int lg = 0;
    while ((1 << lg) < nseg || (1 << lg) < NB) lg++;
    return lg;
}

// The candidate at the head of the queue is the next one expanded unless a
// closer one arrives first: its adjacency row goes to L2 when the head changes.
__device__ __forceinline__ void prefetch_head_row(const GraphView &g, int head_lane0, uint32_t rbytes, int &pf_head,
                                                  int lane)
{
    const int head = __shfl_sync(kFull, head_lane0, 0);
    if (head != pf_head) {
        if (lane == 0 && head >= 0 && rbytes) prefetch_l2(g.links + (int64_t)head * g.lstride, rbytes);
        pf_head = head;
    }
}

// Per-query inputs and outputs of search_one_inter.
struct QueryIO {
    const float *query;             // dim floats
    int entry;
    int32_t *out_ids;               // result row
    float *out_d;
    int out_stride;                 // row length (filled with -1 / large past the results)
    int write_all_ef;               // 1: write ef results, physical ids (rerank input)
    int32_t *hops;                  // per-query counters (may be null)
    int32_t *visited;
    int32_t *status;
};

// Whole-row Bloom path for vectors of one register row (FP32 dim <= 128, BF16
// <= 256, FP8 <= 512); wider vectors keep the per-32-id path, whose register
// footprint leaves room for their extra gather rows.
template <int ELEM, int VROWS>
constexpr bool kRowBloom = (VROWS == 1);

// Traversal trace of one query (the reference's trace kernel,
// FPGA_multi_DDR/eval_trace_FPGA_inter_query_v1.3/src/DRAM_utils.hpp:389-474,
// scheduler.hpp:84): per expanded candidate in FIFO order its distance (1e20
// for the entry point, which is not distance-computed) and the number of
// distances computed for its row; per computed distance in stream order the
// distance and the id.  counts = {popped incl. the entry, expanded, computed};
// entries past a capacity are counted, not written.
struct TraceIO {
    float *cand_d;
    int32_t *cand_n;
    int32_t cand_cap;
    float *d;
    int32_t *id;
    int32_t cap;
    int32_t *counts;
};

// Record the computed distances of one batch (lanes with `rec`, whose slots
// ascend with the lanes) at trace positions n.. in stream order.
__device__ __forceinline__ void trace_batch(const TraceIO *tr, int &n, bool rec, float dist, int id, int lane)
{
    const unsigned m = __ballot_sync(kFull, rec);
    if (rec) {
        const int pos = n + __popc(m & ((1u << lane) - 1u));
        if (pos < tr->cap) { tr->d[pos] = dist; tr->id[pos] = id; }
    }
    n += __popc(m);
}

// ---------------------------------------------------------------------------
// Batch merge (intra-query kernel, ef <= 256: both queues sorted in shared
// memory, merged by warp 0 while the channel warps wait for the group).
//
// In the sorted-list model above, inserting x_1..x_m one at a time (x_j kept
// iff its distance is below the result list's current maximum, then forwarded
// to the candidate list iff also below that list's maximum) has a closed
// form, because a maximum only ever decreases while results are collected:
//   * the result list afterwards holds the ef smallest keys (distance, age)
//     of the old list and x_1..x_m, and x_j is kept iff fewer than ef of
//     {old entries, x_1..x_{j-1}} have a distance <= d_j (an x_i rejected
//     earlier with d_i <= d_j implies d_j is rejected too, so counting it
//     changes nothing);
//   * x_j is forwarded iff it is kept and fewer than cq of {old candidate
//     entries, kept x_i with i < j} have a distance <= d_j (a kept x_i that
//     was not forwarded had d_i >= the candidate maximum, so again counting it
//     changes nothing);
//   * the merged order is by (distance, age): old entries before new ones of
//     equal distance, new ones in stream order.
// So a window of up to 32 stream slots (lane j = slot j) is merged at once
// (in the one-warp kernels few slots per window pass the threshold at these
// ef, and inserting them one at a time in registers measured faster):
// each lane counts the old entries <= its distance by binary search, the
// earlier slots by a ballot loop, and the lists are rewritten in place with
// every entry at its merged position.  The outcome is the one-at-a-time
// insertion's, entry for entry.
// ---------------------------------------------------------------------------
struct SmemLists {
    float *rd;    // result list distances [0, ef)
    int *ri;
    float *cd;    // candidate list distances [0, cq)
    int *ci;
};

// Entries of the ascending a[0..n) that are <= x.
__device__ __forceinline__ int count_le(const float *a, int n, float x)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Rewrite the ascending list a/ai[0..n) (PER entries per lane at p = lane +
// 32 e) merged with the lanes of mask m, each at its merged position newpos:
// an old entry moves right by the number of new entries with a smaller
// distance; entries pushed to position n or beyond drop out.
template <int PER>
__device__ __forceinline__ void list_merge_rewrite(float *a, int *ai, int n, unsigned m, float d, int id, int newpos,
                                                   int lane)
{
    float od[PER];
    int oi[PER], sh[PER];
#pragma unroll
    for (int e = 0; e < PER; e++) {
        const int p = lane + 32 * e;
        od[e] = (p < n) ? a[p] : 0.0f;
        oi[e] = (p < n) ? ai[p] : -1;
        sh[e] = 0;
    }
    for (unsigned mm = m; mm; mm &= mm - 1) {
        const float dj = __shfl_sync(kFull, d, __ffs(mm) - 1);
#pragma unroll
        for (int e = 0; e < PER; e++) sh[e] += (dj < od[e]) ? 1 : 0;
    }
    __syncwarp();
#pragma unroll
    for (int e = 0; e < PER; e++) {
        const int p = lane + 32 * e, q = p + sh[e];
        if (p < n && q < n) {
            a[q] = od[e];
            ai[q] = oi[e];
        }
    }
    if (((m >> lane) & 1u) && newpos < n) {
        a[newpos] = d;
        ai[newpos] = id;
    }
    __syncwarp();
}

// Merge the window (lane j: slot j, `valid` lanes only) into both lists.
template <int EPL, int CPL>
__device__ __forceinline__ void merge_window(const SmemLists &L, int ef, int cq, float d, int id, bool valid, int lane,
                                             float &rmax, float &cmax)
{
    const unsigned vm = __ballot_sync(kFull, valid && d < rmax);
    if (vm == 0) return;
    const bool in = (vm >> lane) & 1u;
    const int r_le = in ? count_le(L.rd, ef, d) : ef;
    int b_le = 0;
    for (unsigned m = vm; m; m &= m - 1) {
        const int i = __ffs(m) - 1;
        const float di = __shfl_sync(kFull, d, i);
        b_le += (i < lane && di <= d) ? 1 : 0;
    }
    const bool kept = in && r_le + b_le < ef;
    const unsigned km = __ballot_sync(kFull, kept);
    int k_before = 0, k_le = 0;
    for (unsigned m = km; m; m &= m - 1) {
        const int i = __ffs(m) - 1;
        const float di = __shfl_sync(kFull, d, i);
        k_before += (di < d || (di == d && i < lane)) ? 1 : 0;
        k_le += (i < lane && di <= d) ? 1 : 0;
    }
    const int c_le = kept ? count_le(L.cd, cq, d) : cq;
    const bool fwd = kept && c_le + k_le < cq;
    const unsigned fm = __ballot_sync(kFull, fwd);
    int f_before = 0;
    for (unsigned m = fm; m; m &= m - 1) {
        const int i = __ffs(m) - 1;
        const float di = __shfl_sync(kFull, d, i);
        f_before += (di < d || (di == d && i < lane)) ? 1 : 0;
    }
    list_merge_rewrite<EPL>(L.rd, L.ri, ef, km, d, id, r_le + k_before, lane);
    rmax = L.rd[ef - 1];
    if (fm) {
        list_merge_rewrite<CPL>(L.cd, L.ci, cq, fm, d, id, c_le + f_before, lane);
        cmax = L.cd[cq - 1];
    }
}

// pop_top of the candidate list in shared memory: the best entry leaves, the
// rest move up one, a +large placeholder enters at position cq - 1.
template <int CPL>
__device__ __forceinline__ int list_pop(float *cd, int *ci, int cq, int lane)
{
    const int pid = ci[0];
    float t[CPL];
    int ti[CPL];
#pragma unroll
    for (int e = 0; e < CPL; e++) {
        const int nx = lane + 32 * e + 1;
        t[e] = (nx < cq) ? cd[nx] : kLarge;
        ti[e] = (nx < cq) ? ci[nx] : -1;
    }
    __syncwarp();
#pragma unroll
    for (int e = 0; e < CPL; e++) {
        const int p = lane + 32 * e;
        if (p < cq) {
            cd[p] = t[e];
            ci[p] = ti[e];
        }
    }
    __syncwarp();
    return pid;
}

// ROW selects the whole-row Bloom path for degrees <= 64; instances whose
// vector registers leave no room for it keep the per-32-id path.
template <int ELEM, int EPL, int VROWS, bool ROW, bool TRACE = false>
__device__ void search_one_inter(const GraphView &g, const QParams &P, const QueryIO &io, uint32_t *bloom, int *fifo,
                                 int *fifo_len, int *sids, uint64_t *hkey, int *hid, int lane,
                                 const TraceIO *tr = nullptr)
{
    constexpr bool HEAP = EPL > 8;            // result list as a shared-memory heap
    constexpr int REPL = HEAP ? 1 : EPL;      // register entries per lane
    constexpr int EPS = ET<ELEM>::EPS;
    constexpr int NB = (VROWS == 1) ? 8 : 4;
    const int nseg = g.dpad * ET<ELEM>::BYTES / 16;
    // lane groups: BS = (32 >> lg) * NB stream slots per gather batch; slot
    // b0 + s lives in row s mod NB of group s / NB, read back at lane rep(s)
    const uint32_t vbytes = (uint32_t)nseg * 16u;                       // one stored vector
    const uint32_t rbytes = (uint32_t)(g.ids_off + g.max_degree) * 4u;  // count word and ids of a row
    int pf_head = -1;                                                   // last candidate head prefetched
    const int lg = lane_group_log2<VROWS, NB>(nseg);
    const int BS = (32 >> lg) * NB;
    const int gmask = (1 << lg) - 1;
    const bool rep_lane = (lane & gmask) < NB;              // one lane per slot
    const int my_slot = (lane >> lg) * NB + (lane & gmask);  // the slot that lane represents

    float nq[VROWS][EPS];   // negated query (seg_tree)
    {
        const float *Q = io.query;
#pragma unroll
        for (int r = 0; r < VROWS; r++) {
            const int seg = (lane & gmask) + 32 * r;
#pragma unroll
            for (int e = 0; e < EPS; e++) {
                const int j = seg * EPS + e;
                nq[r][e] = (seg < nseg && j < g.dim) ? -__ldcg(Q + j) : 0.0f;
            }
        }
    }
    {   // reset this query's Bloom filter
        const int nvec = 1 << (P.bloom_bits - 5 - 2);
        uint4 *b4 = reinterpret_cast<uint4 *>(bloom);
        for (int i = lane; i < nvec; i += 32) b4[i] = make_uint4(0, 0, 0, 0);
    }
    const uint32_t bmask = (1u << P.bloom_bits) - 1u;

    float rd[REPL];
    int ri[REPL];
#pragma unroll
    for (int e = 0; e < REPL; e++) {
        rd[e] = (lane * EPL + e < P.ef) ? kLarge : __int_as_float(0x7f800000);   // placeholders, then +inf
        ri[e] = -1;
    }
    uint32_t age = 0;
    BucketMax BM;
    if constexpr (HEAP) bucket_init<EPL>(BM, hkey, hid, P.ef, lane);
    constexpr int CPL = CandPerLane<EPL>::value;
    float cd[CPL];
    int ci[CPL];
#pragma unroll
    for (int e = 0; e < CPL; e++) { cd[e] = kLarge; ci[e] = -1; }
    float rmax = kLarge, cmax = kLarge;   // current maxima (warp-uniform)

    int entry = io.entry;
    const int mc = P.mc, mg = P.mg;
    int head = 0, inflight = 1, hops = 1, visited = 0;
    if (entry < 0 || (int64_t)entry >= g.n) {   // bad entry from a device-memory caller: empty result
        if (lane == 0) atomicOr(io.status, 2);
        entry = 0;
        inflight = 0;
        hops = 0;
    }
    if (lane == 0) { fifo[0] = entry; fifo_len[0] = 1; }
    __syncwarp();
    bool truncated = false;
    int t_pop = 1, t_exp = 0, t_dist = 0;   // trace counters
    if constexpr (TRACE) {
        if (lane == 0 && tr->cand_cap > 0) tr->cand_d[0] = kLarge;
    }

    while (inflight > 0) {
        const int glen = fifo_len[head];
        for (int b = 0; b < glen; b++) {
            const int node = fifo[head * mc + b];
            const int32_t *row = g.links + (int64_t)node * g.lstride;
            if (ROW && g.max_degree <= 64) {
                // count and ids in one round trip (the row always holds max_degree slots)
                const int cnt = ld_nc_s32(row);
                const int n0 = (lane < g.max_degree) ? ld_nc_s32(row + g.ids_off + lane) : -1;
                const int n1 = (32 + lane < g.max_degree) ? ld_nc_s32(row + g.ids_off + 32 + lane) : -1;
                const bool a0 = lane < cnt, a1 = 32 + lane < cnt;
                BloomRow B;
                bool p0, p1;
                bloom_row_begin(B, bloom, bmask, P.seed, n0, n1, a0, a1, p0, p1);
                // provisional candidates in stream order (first half, then second half)
                const unsigned pm0 = __ballot_sync(kFull, p0), pm1 = __ballot_sync(kFull, p1);
                const int PV0 = __popc(pm0), PV = PV0 + __popc(pm1);
                const int ps0 = __popc(pm0 & ((1u << lane) - 1u)), ps1 = PV0 + __popc(pm1 & ((1u << lane) - 1u));
                if (p0) sids[ps0] = n0;
                if (p1) sids[ps1] = n1;
                // the row's vectors go to L2 now; the batches below load them from there
                if (p0) prefetch_l2(g.vecs + (int64_t)n0 * g.vstride_bytes, vbytes);
                if (p1) prefetch_l2(g.vecs + (int64_t)n1 * g.vstride_bytes, vbytes);
                __syncwarp();
                // gathers of batch i+1 are issued as soon as batch i's distances are
                // formed, so they are in flight while batch i is inserted
                uint4 raw[NB][VROWS];
                float scale[NB];
                if (PV > 0) gather_batch<ELEM, VROWS, NB>(g, sids, 0, PV, nseg, lane, lg, raw, scale);
                bool v0, v1;
                bloom_row_resolve(B, lane, v0, v1);   // the atomics overlapped the first gathers
                const unsigned vm0 = __ballot_sync(kFull, v0), vm1 = __ballot_sync(kFull, v1);
                // a provisional id that turned out seen is withdrawn from the stream
                if (p0 && !v0) sids[ps0] = ~n0;
                if (p1 && !v1) sids[ps1] = ~n1;
                __syncwarp();
                for (int b0 = 0; b0 < PV; b0 += BS) {
                    const float dist = batch_distances<ELEM, VROWS, NB>(nq, raw, scale, lane, lg);
                    if (b0 + BS < PV) gather_batch<ELEM, VROWS, NB>(g, sids, b0 + BS, PV, nseg, lane, lg, raw, scale);
                    const int nt = min(BS, PV - b0);
                    const bool keep = rep_lane && my_slot < nt && sids[b0 + my_slot] >= 0;
                    if constexpr (TRACE) trace_batch(tr, t_dist, keep, dist, keep ? sids[b0 + my_slot] : 0, lane);
                    unsigned m = __ballot_sync(kFull, keep && dist < rmax);
                    while (m) {   // representative lanes ascend with the slots
                        const int t = __ffs(m) - 1;
                        m &= m - 1;
                        const float dd = __shfl_sync(kFull, dist, t);
                        if (dd < rmax) {
                            const int id = sids[b0 + (t >> lg) * NB + (t & gmask)];
                            if constexpr (HEAP) {
                                rmax = bucket_replace_max<EPL>(BM, hkey, hid, heap_key(dd, ++age), id, lane);
                            } else {
                                rl_insert<EPL>(rd, ri, lane, dd, id);
                                rmax = rl_get<EPL>(rd, P.ef - 1);
                            }
                            if (dd < cmax) {
                                cl_insert<CPL>(cd, ci, lane, P.cq, dd, id);
                                cmax = rl_get<CPL>(cd, P.cq - 1);
                            }
                        }
                    }
                    prefetch_head_row(g, ci[0], rbytes, pf_head, lane);
                }
                visited += __popc(vm0) + __popc(vm1);
                if constexpr (TRACE) {
                    if (lane == 0 && t_exp < tr->cand_cap) tr->cand_n[t_exp] = __popc(vm0) + __popc(vm1);
                    t_exp++;
                }
                __syncwarp();
                continue;
            }
            const int cnt = ld_nc_s32(row);
            int row_valid = 0;
            for (int c0 = 0; c0 < cnt; c0 += 32) {
                const bool act = c0 + lane < cnt;
                const int nb = act ? ld_nc_s32(row + g.ids_off + c0 + lane) : -1;
                const bool valid = bloom_chunk(bloom, bmask, P.seed, nb, act, lane);
                const unsigned vm = __ballot_sync(kFull, valid);
                const int V = __popc(vm);
                visited += V;
                row_valid += V;
                if (valid) sids[__popc(vm & ((1u << lane) - 1u))] = nb;
                if (valid) prefetch_l2(g.vecs + (int64_t)nb * g.vstride_bytes, vbytes);
                __syncwarp();
                uint4 raw[NB][VROWS];
                float scale[NB];
                if (V > 0) gather_batch<ELEM, VROWS, NB>(g, sids, 0, V, nseg, lane, lg, raw, scale);
                for (int b0 = 0; b0 < V; b0 += BS) {
                    const float dist = batch_distances<ELEM, VROWS, NB>(nq, raw, scale, lane, lg);
                    if (b0 + BS < V) gather_batch<ELEM, VROWS, NB>(g, sids, b0 + BS, V, nseg, lane, lg, raw, scale);
                    const int nt = min(BS, V - b0);
                    if constexpr (TRACE)
                        trace_batch(tr, t_dist, rep_lane && my_slot < nt, dist,
                                    (rep_lane && my_slot < nt) ? sids[b0 + my_slot] : 0, lane);
                    // results collection (DRAM_utils.hpp:421-438) in stream order; the
                    // maximum only decreases, so a distance not below it now never will be
                    unsigned m = __ballot_sync(kFull, rep_lane && my_slot < nt && dist < rmax);
                    while (m) {   // representative lanes ascend with the slots
                        const int t = __ffs(m) - 1;
                        m &= m - 1;
                        const float dd = __shfl_sync(kFull, dist, t);
                        if (dd < rmax) {
                            const int id = sids[b0 + (t >> lg) * NB + (t & gmask)];
                            if constexpr (HEAP) {
                                rmax = bucket_replace_max<EPL>(BM, hkey, hid, heap_key(dd, ++age), id, lane);
                            } else {
                                rl_insert<EPL>(rd, ri, lane, dd, id);
                                rmax = rl_get<EPL>(rd, P.ef - 1);
                            }
                            if (dd < cmax) {   // forwarded to the candidate queue (scheduler.hpp:102-110)
                                cl_insert<CPL>(cd, ci, lane, P.cq, dd, id);
                                cmax = rl_get<CPL>(cd, P.cq - 1);
                            }
                        }
                    }
                    prefetch_head_row(g, ci[0], rbytes, pf_head, lane);
                }
                __syncwarp();
            }
            if constexpr (TRACE) {
                if (lane == 0 && t_exp < tr->cand_cap) tr->cand_n[t_exp] = row_valid;
                t_exp++;
            }
        }
        // the oldest group is retired (scheduler.hpp:112-155): threshold = worst result
        const float thr = rmax;
        head = (head + 1 == mg) ? 0 : head + 1;
        inflight--;
        for (int oid = inflight; oid < mg && !truncated; oid++) {
            int slot = head + inflight;
            if (slot >= mg) slot -= mg;
            int n = 0;
            for (int bb = 0; bb < mc; bb++) {
                const float best = __shfl_sync(kFull, cd[0], 0);
                if (!(best <= thr && best < kLarge)) break;
                if (P.max_hops > 0 && hops >= P.max_hops) { truncated = true; break; }
                if constexpr (TRACE) {
                    if (lane == 0 && t_pop < tr->cand_cap) tr->cand_d[t_pop] = best;
                    t_pop++;
                }
                const int pid = cl_pop<CPL>(cd, ci, lane, P.cq);
                if (lane == 0) fifo[slot * mc + n] = pid;
                n++;
                hops++;
            }
            if (n == 0) break;
            if (lane == 0) fifo_len[slot] = n;
            inflight++;
        }
        cmax = rl_get<CPL>(cd, P.cq - 1);
        __syncwarp();
    }
    if constexpr (TRACE) {
        if (lane == 0) { tr->counts[0] = t_pop; tr->counts[1] = t_exp; tr->counts[2] = t_dist; }
    }

    // results best-first (DRAM_utils.hpp:460-464): list position i is result i
    const int nwrite = io.write_all_ef ? P.ef : P.k;
    int32_t *oid_row = io.out_ids;
    float *od_row = io.out_d;
    if constexpr (HEAP) {
        int n2 = 1;
        while (n2 < P.ef) n2 <<= 1;
        for (int i = P.ef + lane; i < n2; i += 32) { hkey[i] = ~0ull; hid[i] = -1; }
        __syncwarp();
        warp_bitonic_sort(hkey, hid, n2, lane);
        for (int i = lane; i < nwrite; i += 32) {
            int id = hid[i];
            if (!io.write_all_ef && g.labels && id >= 0) id = g.labels[id];
            oid_row[i] = id;
            od_row[i] = __uint_as_float((uint32_t)(hkey[i] >> 32));
        }
        __syncwarp();
    } else {
#pragma unroll
        for (int e = 0; e < REPL; e++) {
            const int i = lane * EPL + e;
            if (i < nwrite) {
                int id = ri[e];
                if (!io.write_all_ef && g.labels && id >= 0) id = g.labels[id];
                oid_row[i] = id;
                od_row[i] = rd[e];
            }
        }
    }
    for (int i = nwrite + lane; i < io.out_stride; i += 32) { oid_row[i] = -1; od_row[i] = kLarge; }
    if (lane == 0) {
        if (io.hops) *io.hops = hops;
        if (io.visited) *io.visited = visited;
        if (truncated) atomicOr(io.status, 1);
    }
}

// Shared memory of one warp: Bloom filter (when it fits), the bucketed
// result list (heap_cap slots) or the two sorted lists (list_r + list_c
// slots), the group FIFO and the staged neighbour ids.
__host__ __device__ __forceinline__ size_t warp_smem_bytes(int bloom_bits_max, int mc_max, int mg_max, int heap_cap,
                                                           int list_r, int list_c)
{
    size_t b = (bloom_bits_max <= kMaxSmemBloomBits) ? ((size_t)1 << (bloom_bits_max - 3)) : 0;
    b += (size_t)heap_cap * (sizeof(uint64_t) + sizeof(int));
    b += (size_t)(list_r + list_c) * (sizeof(float) + sizeof(int));
    b += sizeof(int) * (size_t)(mc_max * mg_max + mg_max + kSidsPerWarp);
    return (b + 15) & ~(size_t)15;
}

// Pointers into one warp's shared memory (layout of warp_smem_bytes).
struct WarpSmem {
    uint32_t *bloom;
    uint64_t *hkey;
    int *hid;
    SmemLists lists;
    int *fifo, *fifo_len, *sids;
};

__device__ __forceinline__ WarpSmem carve_warp_smem(unsigned char *wbase, uint32_t *bloom_global, bool smem_bloom,
                                                    size_t bloom_bytes, int heap_cap, int list_r, int list_c,
                                                    int mc_max, int mg_max)
{
    WarpSmem w;
    w.bloom = smem_bloom ? reinterpret_cast<uint32_t *>(wbase) : bloom_global;
    unsigned char *p = wbase + (smem_bloom ? bloom_bytes : 0);
    w.hkey = reinterpret_cast<uint64_t *>(p);
    p += sizeof(uint64_t) * heap_cap;
    w.hid = reinterpret_cast<int *>(p);
    p += sizeof(int) * heap_cap;
    w.lists.rd = reinterpret_cast<float *>(p);
    p += sizeof(float) * list_r;
    w.lists.ri = reinterpret_cast<int *>(p);
    p += sizeof(int) * list_r;
    w.lists.cd = reinterpret_cast<float *>(p);
    p += sizeof(float) * list_c;
    w.lists.ci = reinterpret_cast<int *>(p);
    p += sizeof(int) * list_c;
    w.fifo = reinterpret_cast<int *>(p);
    w.fifo_len = w.fifo + mc_max * mg_max;
    w.sids = w.fifo_len + mg_max;
    return w;
}

// Shared-memory list capacities: the bucketed result list for ef > 256 (all
// kernels), and the sorted lists for ef <= 256 (the intra-query kernel only;
// the one-warp traversal keeps those lists in registers).
template <int EPL, bool SORTED_LISTS = false> struct ListCaps {
    static constexpr int heap = (EPL > 8) ? 32 * EPL : 0;
    static constexpr int r = (EPL > 8 || !SORTED_LISTS) ? 0 : 32 * EPL;
    static constexpr int c = (EPL > 8 || !SORTED_LISTS) ? 0 : 32 * CandPerLane<EPL>::value;
};

// Resident blocks of 4 warps the one-warp traversal is compiled for.  3 (168
// registers) keeps the gather batch and the lists in registers without
// spilling.  FP32 rows of one 512-byte segment row (D <= 128) at ef <= 256
// run 4 (128 registers): the 16 warps per SM hide more gather latency than
// the ~100 bytes of spilled loop state cost (913.6k -> 985.5k queries/s on
// the 10M x 128 mixed-parameter workload).  FALCON_INTER_BLOCKS_SMALL_EF
// overrides that choice.
#ifndef FALCON_INTER_BLOCKS_SMALL_EF
#define FALCON_INTER_BLOCKS_SMALL_EF 4
#endif
template <int ELEM, int EPL, int VROWS> struct InterBlocks {
    static constexpr int value = (ELEM == kF32 && VROWS == 1 && EPL <= 8) ? FALCON_INTER_BLOCKS_SMALL_EF : 3;
};

template <int ELEM, int EPL, int VROWS, bool TRACE>
__global__ void __launch_bounds__(128, (InterBlocks<ELEM, EPL, VROWS>::value)) inter_kernel(const SearchLaunch A)
{
    extern __shared__ uint4 smem_u4[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    using Caps = ListCaps<EPL>;
    const size_t wbytes = warp_smem_bytes(A.bloom_bits_max, A.mc_max, A.mg_max, Caps::heap, Caps::r, Caps::c);
    unsigned char *wbase = reinterpret_cast<unsigned char *>(smem_u4) + wbytes * warp;
    const bool smem_bloom = A.bloom_bits_max <= kMaxSmemBloomBits;
    const size_t bloom_bytes = (size_t)1 << (A.bloom_bits_max - 3);
    uint32_t *gbloom = smem_bloom ? nullptr : A.bloom_global + ((size_t)blockIdx.x * 4 + warp) * (bloom_bytes / 4);
    const WarpSmem W = carve_warp_smem(wbase, gbloom, smem_bloom, bloom_bytes, Caps::heap, Caps::r, Caps::c, A.mc_max,
                                       A.mg_max);
    for (;;) {
        unsigned long long qi = 0;
        if (lane == 0) qi = atomicAdd(reinterpret_cast<unsigned long long *>(A.work_counter), 1ull);
        qi = __shfl_sync(kFull, qi, 0);
        if (qi >= (unsigned long long)A.nq) break;
        const QParams P = A.params[A.per_query ? qi : 0];
        QueryIO io;
        io.query = A.queries + (int64_t)qi * A.qstride;
        io.entry = A.entries ? A.entries[qi] : A.default_entry;
        io.out_ids = A.out_ids + (int64_t)qi * A.out_stride;
        io.out_d = A.out_d + (int64_t)qi * A.out_stride;
        io.out_stride = A.out_stride;
        io.write_all_ef = A.write_all_ef;
        io.hops = A.out_hops ? A.out_hops + qi : nullptr;
        io.visited = A.out_visited ? A.out_visited + qi : nullptr;
        io.status = A.status;
        if constexpr (TRACE) {
            TraceIO tio;
            tio.cand_d = A.trace_cand_d + (int64_t)qi * A.trace_cand_cap;
            tio.cand_n = A.trace_cand_n + (int64_t)qi * A.trace_cand_cap;
            tio.cand_cap = A.trace_cand_cap;
            tio.d = A.trace_d + (int64_t)qi * A.trace_cap;
            tio.id = A.trace_id + (int64_t)qi * A.trace_cap;
            tio.cap = A.trace_cap;
            tio.counts = A.trace_counts + 3 * (int64_t)qi;
            search_one_inter<ELEM, EPL, VROWS, kRowBloom<ELEM, VROWS>, true>(A.g, P, io, W.bloom, W.fifo, W.fifo_len,
                                                                             W.sids, W.hkey, W.hid, lane, &tio);
        } else {
            search_one_inter<ELEM, EPL, VROWS, kRowBloom<ELEM, VROWS>>(A.g, P, io, W.bloom, W.fifo, W.fifo_len, W.sids,
                                                                       W.hkey, W.hid, lane);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Intra-query mode (reference intra-query v1.5): one thread block per query,
// `channels` channels of W fetch warps each (W only spreads the work; results
// do not depend on it) and one merge warp.  Per group
//   1. the channel's first warp routes the group's neighbour ids to channel
//      id & (channels-1) keeping stream order (utils.hpp:396-495,
//      split_tasks_to_channels) and runs the channel's Bloom filter over them
//      (the reference's per-channel bloom PE), keeping the new ids in order;
//   2. the channel's W warps gather the new vectors and form their distances
//      (the per-channel fetch/compute PEs), batches dealt round robin;
//   3. the merge warp merges the channels in channel order into the queues
//      (gather_distances_from_channels, utils.hpp:497-569, merges in
//      readiness order; channel order is one of its schedules; a whole
//      group is merged before the scheduler acts, so on distinct distances
//      the order cannot change the outcome), then the scheduler refills the
//      group FIFO (v1.5 scheduler.hpp:94-146) and prefetches the rows of the
//      candidates it popped.
// Steps 1-2 of a group run while step 3 of the group before it runs (DST:
// with mg >= 2 groups in flight the fetch overlaps the merge).
// The stale-threshold prefilter of v1.5 (utils.hpp:277-347) is omitted: it
// only drops distances that the result queue would reject anyway.
// ---------------------------------------------------------------------------
struct IntraSmem {
    unsigned long long qi;
    // the group FIFO's state, published by the merge warp each step into the
    // slot of the step's parity: head, groups in flight (popped, not merged),
    // hops, truncated
    int st[2][4];
    int chan_valid[2][kMaxChannels];   // per step parity
    int chan_visited[kMaxChannels];
};

// Most warps an intra-query block uses: up to 12 fetch warps (channels x
// warps per channel) and the merge warp.  13 warps put at most 4 on each of
// the SM's four schedulers, which leaves 128 registers per thread (17 would
// leave 96 and spill).
constexpr int kIntraMaxWarps = 13;

template <int ELEM, int EPL, int VROWS>
__global__ void __launch_bounds__(32 * kIntraMaxWarps) intra_kernel(const SearchLaunch A)
{
    extern __shared__ uint4 smem_u4[];
    constexpr int EPS = ET<ELEM>::EPS;
    constexpr int NB = (VROWS == 1) ? 8 : 4;
    constexpr bool HEAP = EPL > 8;
    constexpr int HEAP_CAP = HEAP ? 32 * EPL : 0;
    const int C = A.channels;
    const int MW = (blockDim.x >> 5) - 1;                 // the merge warp; 0 .. MW-1 fetch
    const int W = MW / C;                                 // fetch warps per channel
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool merger = warp == MW;
    const int chan = merger ? 0 : warp / W, sub = merger ? 0 : warp - chan * W;
    const GraphView &g = A.g;
    const int nseg = g.dpad * ET<ELEM>::BYTES / 16;
    unsigned char *base_ptr = reinterpret_cast<unsigned char *>(smem_u4);
    IntraSmem *S = reinterpret_cast<IntraSmem *>(base_ptr);
    size_t off = (sizeof(IntraSmem) + 15) & ~(size_t)15;
    const size_t bloom_bytes = (size_t)1 << (A.bloom_bits_max - 3);
    const bool smem_bloom = A.bloom_bits_max <= kMaxSmemBloomBits;
    uint32_t *bloom = smem_bloom ? reinterpret_cast<uint32_t *>(base_ptr + off + bloom_bytes * chan)
                                 : A.bloom_global + ((size_t)blockIdx.x * C + chan) * (bloom_bytes / 4);
    if (smem_bloom) off += bloom_bytes * C;
    // channel c's ids (then its new ids and their distances) of a group: lcap
    // slots at (parity * C + c) * lcap; a step fills one parity while the
    // merge warp reads the other
    const int lcap = A.mc_max * g.max_degree;
    int *list_id = reinterpret_cast<int *>(base_ptr + off);
    off += sizeof(int) * (size_t)lcap * C * 2;
    float *list_d = reinterpret_cast<float *>(base_ptr + off);
    off += sizeof(float) * (size_t)lcap * C * 2;
    int *fifo = reinterpret_cast<int *>(base_ptr + off);
    off += sizeof(int) * (size_t)(A.mc_max * A.mg_max);
    int *fifo_len = reinterpret_cast<int *>(base_ptr + off);
    off += sizeof(int) * (size_t)A.mg_max;
    off = (off + 15) & ~(size_t)15;
    uint64_t *hkey = reinterpret_cast<uint64_t *>(base_ptr + off);
    int *hid = reinterpret_cast<int *>(base_ptr + off + sizeof(uint64_t) * HEAP_CAP);
    off += (sizeof(uint64_t) + sizeof(int)) * HEAP_CAP;
    using Caps = ListCaps<EPL, true>;
    SmemLists L;   // sorted lists for ef <= 256, used by the merge warp
    L.rd = reinterpret_cast<float *>(base_ptr + off);
    L.ri = reinterpret_cast<int *>(L.rd + Caps::r);
    L.cd = reinterpret_cast<float *>(L.ri + Caps::r);
    L.ci = reinterpret_cast<int *>(L.cd + Caps::c);
    // lane groups and gather batches as in search_one_inter
    const uint32_t vbytes = (uint32_t)nseg * 16u;
    const uint32_t rbytes = (uint32_t)(g.ids_off + g.max_degree) * 4u;
    const int lg = lane_group_log2<VROWS, NB>(nseg);
    const int BS = (32 >> lg) * NB;
    const int gmask = (1 << lg) - 1;
    const bool rep_lane = (lane & gmask) < NB;
    const int my_slot = (lane >> lg) * NB + (lane & gmask);

    for (;;) {
        if (threadIdx.x == 0) S->qi = atomicAdd(reinterpret_cast<unsigned long long *>(A.work_counter), 1ull);
        __syncthreads();
        const unsigned long long qi = S->qi;
        if (qi >= (unsigned long long)A.nq) break;
        const QParams P = A.params[A.per_query ? qi : 0];
        const int mc = P.mc, mg = P.mg;
        float nq[VROWS][EPS];   // negated query (seg_tree)
        {
            const float *Q = A.queries + qi * A.qstride;
#pragma unroll
            for (int r = 0; r < VROWS; r++) {
                const int seg = (lane & gmask) + 32 * r;
#pragma unroll
                for (int e = 0; e < EPS; e++) {
                    const int j = seg * EPS + e;
                    nq[r][e] = (seg < nseg && j < g.dim) ? -Q[j] : 0.0f;
                }
            }
        }
        if (!merger) {   // the channel's warps clear its filter
            const int nvec = 1 << (P.bloom_bits - 7);
            uint4 *b4 = reinterpret_cast<uint4 *>(bloom);
            for (int i = sub * 32 + lane; i < nvec; i += 32 * W) b4[i] = make_uint4(0, 0, 0, 0);
        }
        const uint32_t bmask = (1u << P.bloom_bits) - 1u;
        int visited = 0;
        // queues live in the merge warp: the bucketed list + register candidate
        // list for ef > 256, else the sorted lists L in shared memory
        uint32_t age = 0;
        BucketMax BM;
        constexpr int CPL = CandPerLane<EPL>::value;
        float cd[HEAP ? CPL : 1];
        int ci[HEAP ? CPL : 1];
        if constexpr (HEAP) {
            if (merger) bucket_init<EPL>(BM, hkey, hid, P.ef, lane);
#pragma unroll
            for (int e = 0; e < CPL; e++) { cd[e] = kLarge; ci[e] = -1; }
        } else if (merger) {
            for (int p = lane; p < P.ef; p += 32) { L.rd[p] = kLarge; L.ri[p] = -1; }
            for (int p = lane; p < P.cq; p += 32) { L.cd[p] = kLarge; L.ci[p] = -1; }
            __syncwarp();
        }
        float rmax = kLarge, cmax = kLarge;
        if (threadIdx.x == 0) {
            int entry = A.entries ? A.entries[qi] : A.default_entry;
            int n = 1;
            if (entry < 0 || (int64_t)entry >= g.n) {
                atomicOr(A.status, 2);
                entry = 0;
                n = 0;
            }
            fifo[0] = entry;
            fifo_len[0] = 1;
            S->st[1][0] = 0;   // head
            S->st[1][1] = n;   // groups in flight
            S->st[1][2] = n;   // hops
            S->st[1][3] = 0;   // truncated
        }
        __syncthreads();
        // Step s: the fetch warps take the oldest group not yet fetched (split,
        // Bloom, gathers, distances) into parity s & 1 while the merge warp
        // merges the group fetched in step s - 1 and refills the FIFO.  Bloom
        // filters see the groups in FIFO order and the merges happen in FIFO
        // order, each followed by its pops, so the outcome equals fetching each
        // group only after the previous one is merged; with mg >= 2 the fetch
        // of a group overlaps the merge of the one before it.
        bool hf = false;   // the head group was fetched in the previous step
        int fin = 1;       // the state slot the loop ends on
        for (int step = 0;; step++) {
            const int *st = S->st[(step + 1) & 1];
            const int head = st[0], n = st[1];
            if (n == 0) {
                fin = (step + 1) & 1;
                break;
            }
            const int par = step & 1;
            int fslot = -1;
            if (!hf) fslot = head;
            else if (n >= 2) fslot = (head + 1 == mg) ? 0 : head + 1;
            if (!merger && fslot >= 0) {
                const int glen = fifo_len[fslot];
                int *my_ids = list_id + (size_t)lcap * (par * C + chan);
                float *my_d = list_d + (size_t)lcap * (par * C + chan);
                // 1. the channel's first warp: its ids of the group's rows in
                //    stream order, then its Bloom filter; the new ids are
                //    compacted in place
                if (sub == 0) {
                    int count = 0;
                    if (g.max_degree <= 64) {
                        // counts and ids of up to 4 rows in one round trip (a row
                        // always holds max_degree slots; those past the count are masked)
                        for (int b0 = 0; b0 < glen; b0 += 4) {
                            int rc[4], r0[4], r1[4];
#pragma unroll
                            for (int u = 0; u < 4; u++) {
                                rc[u] = 0;
                                r0[u] = r1[u] = -1;
                                if (b0 + u < glen) {
                                    const int32_t *row = g.links + (int64_t)fifo[fslot * mc + b0 + u] * g.lstride;
                                    rc[u] = ld_nc_s32(row);
                                    if (lane < g.max_degree) r0[u] = ld_nc_s32(row + g.ids_off + lane);
                                    if (32 + lane < g.max_degree) r1[u] = ld_nc_s32(row + g.ids_off + 32 + lane);
                                }
                            }
#pragma unroll
                            for (int u = 0; u < 4; u++) {
#pragma unroll
                                for (int hf2 = 0; hf2 < 2; hf2++) {
                                    const int nb = hf2 ? r1[u] : r0[u];
                                    const bool mine = 32 * hf2 + lane < rc[u] && nb >= 0 && (nb & (C - 1)) == chan;
                                    const unsigned mm = __ballot_sync(kFull, mine);
                                    if (mine) my_ids[count + __popc(mm & ((1u << lane) - 1u))] = nb;
                                    count += __popc(mm);
                                }
                            }
                        }
                    } else {
                        for (int b = 0; b < glen; b++) {
                            const int32_t *row = g.links + (int64_t)fifo[fslot * mc + b] * g.lstride;
                            const int cnt = ld_nc_s32(row);
                            for (int c0 = 0; c0 < cnt; c0 += 32) {
                                const int nb = (c0 + lane < cnt) ? ld_nc_s32(row + g.ids_off + c0 + lane) : -1;
                                const bool mine = nb >= 0 && (nb & (C - 1)) == chan;
                                const unsigned mm = __ballot_sync(kFull, mine);
                                if (mine) my_ids[count + __popc(mm & ((1u << lane) - 1u))] = nb;
                                count += __popc(mm);
                            }
                        }
                    }
                    __syncwarp();
                    int nvalid = 0;
                    for (int c0 = 0; c0 < count; c0 += 32) {
                        const bool act = c0 + lane < count;
                        const int nb = act ? my_ids[c0 + lane] : -1;
                        const bool valid = bloom_chunk(bloom, bmask, P.seed, nb, act, lane);
                        const unsigned vm = __ballot_sync(kFull, valid);
                        // written at or below the chunk just read: the in-place compaction is safe
                        if (valid) {
                            my_ids[nvalid + __popc(vm & ((1u << lane) - 1u))] = nb;
                            prefetch_l2(g.vecs + (int64_t)nb * g.vstride_bytes, vbytes);
                        }
                        nvalid += __popc(vm);
                        __syncwarp();
                    }
                    visited += nvalid;
                    if (lane == 0) S->chan_valid[par][chan] = nvalid;
                }
                // the channel's warps wait for its first warp (named barrier 1 + chan)
                asm volatile("bar.sync %0, %1;" ::"r"(1 + chan), "r"(32 * W) : "memory");
                // 2. the channel's warps: gathers and distances, batch b by warp b mod W
                const int nvalid = S->chan_valid[par][chan];
                const int stp = BS * W;
                int b0 = BS * sub;
                uint4 raw[NB][VROWS];
                float scale[NB];
                if (b0 < nvalid) gather_batch<ELEM, VROWS, NB>(g, my_ids, b0, nvalid, nseg, lane, lg, raw, scale);
                for (; b0 < nvalid; b0 += stp) {
                    const float dist = batch_distances<ELEM, VROWS, NB>(nq, raw, scale, lane, lg);
                    if (b0 + stp < nvalid)
                        gather_batch<ELEM, VROWS, NB>(g, my_ids, b0 + stp, nvalid, nseg, lane, lg, raw, scale);
                    if (rep_lane && b0 + my_slot < nvalid) my_d[b0 + my_slot] = dist;
                }
            }
            if (merger) {
                int h = head, inflight = n, hops = st[2];
                bool truncated = st[3] != 0;
                if (hf) {
                    // 3. merge the group fetched in the previous step, channels in
                    //    order; the windows of 32 run over the channel lists laid
                    //    end to end, so a window spans channel boundaries
                    const int mp = par ^ 1;
                    int *lid = list_id + (size_t)lcap * mp * C;
                    float *ld = list_d + (size_t)lcap * mp * C;
                    int total = 0;
                    for (int c = 0; c < C; c++) total += S->chan_valid[mp][c];
                    if constexpr (!HEAP) {
                        // Only ids below the worst result can be kept (the maximum only
                        // decreases during the merge): they are packed in sequence order
                        // to the front of this parity's lists, so that every window but
                        // the last is full.  A packed slot never lies beyond its source
                        // (channel c's lists start after all earlier channels' ids).
                        int np = 0;
                        for (int j0 = 0; j0 < total; j0 += 32) {
                            const int p = j0 + lane;
                            const bool v = p < total;
                            int src = 0;
                            if (v) {
                                int rem = p, c = 0;
                                while (rem >= S->chan_valid[mp][c]) rem -= S->chan_valid[mp][c++];
                                src = c * lcap + rem;
                            }
                            const float dl = v ? ld[src] : kLarge;
                            const int il = v ? lid[src] : -1;
                            const bool keep = v && dl < rmax;
                            const unsigned km = __ballot_sync(kFull, keep);
                            __syncwarp();
                            if (keep) {
                                const int t = np + __popc(km & ((1u << lane) - 1u));
                                ld[t] = dl;
                                lid[t] = il;
                            }
                            np += __popc(km);
                            __syncwarp();
                        }
                        for (int j0 = 0; j0 < np; j0 += 32) {
                            const bool v = j0 + lane < np;
                            const float dl = v ? ld[j0 + lane] : kLarge;
                            const int idl = v ? lid[j0 + lane] : -1;
                            merge_window<EPL, CPL>(L, P.ef, P.cq, dl, idl, v, lane, rmax, cmax);
                        }
                        total = 0;
                    }
                    for (int j0 = 0; j0 < total; j0 += 32) {
                        const int p = j0 + lane;
                        const bool v = p < total;
                        int src = 0;
                        if (v) {
                            int rem = p, c = 0;
                            while (rem >= S->chan_valid[mp][c]) rem -= S->chan_valid[mp][c++];
                            src = c * lcap + rem;
                        }
                        const float dl = v ? ld[src] : kLarge;
                        if constexpr (HEAP) {
                            unsigned m = __ballot_sync(kFull, v && dl < rmax);
                            while (m) {
                                const int t = __ffs(m) - 1;
                                m &= m - 1;
                                const float dd = __shfl_sync(kFull, dl, t);
                                const int sr = __shfl_sync(kFull, src, t);
                                if (dd < rmax) {
                                    const int id = lid[sr];
                                    rmax = bucket_replace_max<EPL>(BM, hkey, hid, heap_key(dd, ++age), id, lane);
                                    if (dd < cmax) {
                                        cl_insert<CPL>(cd, ci, lane, P.cq, dd, id);
                                        cmax = rl_get<CPL>(cd, P.cq - 1);
                                    }
                                }
                            }
                        }
                    }
                    // 4. the scheduler retires the group and refills the free
                    //    group slots (threshold = worst result)
                    const float thr = rmax;
                    h = (h + 1 == mg) ? 0 : h + 1;
                    inflight--;
                    for (int oid = inflight; oid < mg && !truncated; oid++) {
                        int slot = h + inflight;
                        if (slot >= mg) slot -= mg;
                        int cnt = 0;
                        for (int bb = 0; bb < mc; bb++) {
                            float best;
                            if constexpr (HEAP) best = __shfl_sync(kFull, cd[0], 0);
                            else best = L.cd[0];
                            if (!(best <= thr && best < kLarge)) break;
                            if (P.max_hops > 0 && hops >= P.max_hops) { truncated = true; break; }
                            int pid;
                            if constexpr (HEAP) pid = cl_pop<CPL>(cd, ci, lane, P.cq);
                            else pid = list_pop<CPL>(L.cd, L.ci, P.cq, lane);
                            // the popped candidate's row is read when its group is fetched
                            if (lane == cnt) prefetch_l2(g.links + (int64_t)pid * g.lstride, rbytes);
                            if (lane == 0) fifo[slot * mc + cnt] = pid;
                            cnt++;
                            hops++;
                        }
                        if (cnt == 0) break;
                        if (lane == 0) fifo_len[slot] = cnt;
                        inflight++;
                    }
                    if constexpr (HEAP) cmax = rl_get<CPL>(cd, P.cq - 1);
                    else cmax = L.cd[P.cq - 1];
                }
                if (lane == 0) {
                    int *nst = S->st[step & 1];
                    nst[0] = h;
                    nst[1] = inflight;
                    nst[2] = hops;
                    nst[3] = truncated ? 1 : 0;
                }
            }
            hf = fslot >= 0;
            __syncthreads();
        }
        if (!merger && sub == 0 && lane == 0) S->chan_visited[chan] = visited;
        __syncthreads();
        if (merger) {
            const int nwrite = A.write_all_ef ? P.ef : P.k;
            int32_t *oid_row = A.out_ids + qi * A.out_stride;
            float *od_row = A.out_d + qi * A.out_stride;
            if constexpr (HEAP) {
                int n2 = 1;
                while (n2 < P.ef) n2 <<= 1;
                for (int i = P.ef + lane; i < n2; i += 32) { hkey[i] = ~0ull; hid[i] = -1; }
                __syncwarp();
                warp_bitonic_sort(hkey, hid, n2, lane);
                for (int i = lane; i < nwrite; i += 32) {
                    int id = hid[i];
                    if (!A.write_all_ef && g.labels && id >= 0) id = g.labels[id];
                    oid_row[i] = id;
                    od_row[i] = __uint_as_float((uint32_t)(hkey[i] >> 32));
                }
                __syncwarp();
            } else {
                for (int i = lane; i < nwrite; i += 32) {
                    int id = L.ri[i];
                    if (!A.write_all_ef && g.labels && id >= 0) id = g.labels[id];
                    oid_row[i] = id;
                    od_row[i] = L.rd[i];
                }
            }
            for (int i = nwrite + lane; i < A.out_stride; i += 32) { oid_row[i] = -1; od_row[i] = kLarge; }
            if (lane == 0) {
                int vis = 0;
                for (int c = 0; c < C; c++) vis += S->chan_visited[c];
                if (A.out_hops) A.out_hops[qi] = S->st[fin][2];
                if (A.out_visited) A.out_visited[qi] = vis;
                if (S->st[fin][3]) atomicOr(A.status, 1);
            }
        }
        __syncthreads();
    }
}

size_t intra_smem_bytes(const SearchLaunch &a, int channels, int heap_cap, int list_r, int list_c)
{
    size_t b = (sizeof(IntraSmem) + 15) & ~(size_t)15;
    if (a.bloom_bits_max <= kMaxSmemBloomBits) b += ((size_t)1 << (a.bloom_bits_max - 3)) * channels;
    b += 2 * 2 * sizeof(int) * (size_t)a.mc_max * a.g.max_degree * channels;
    b += sizeof(int) * (size_t)(a.mc_max * a.mg_max + a.mg_max);
    b = (b + 15) & ~(size_t)15;
    b += (size_t)heap_cap * (sizeof(uint64_t) + sizeof(int));
    b += (size_t)(list_r + list_c) * (sizeof(float) + sizeof(int));
    return (b + 15) & ~(size_t)15;
}

// ---------------------------------------------------------------------------
// HNSW upper-layer greedy descent (hnswalg.h:514-541 of the reference's
// vendored hnswlib; the FPGA multi-layer scheduler, FPGA_single_DDR/
// FPGA_single_DDR_multi_layer_v2.2_async/src/scheduler.hpp:116-144): from the
// top entry, at every level from the top down to 1, expand the current node's
// row and move to a neighbour whenever its distance is strictly below the
// current one, scanning the row in order, until a row brings no improvement.
// The result of one row scan is the first neighbour with the smallest
// distance, if that is below the current distance.  No visited filter; FP32
// distances in the adder-tree order of the base-layer search.  One warp per
// query; its row's ids are staged in shared memory.
// ---------------------------------------------------------------------------
template <int VROWS>
__global__ void __launch_bounds__(128) descend_kernel(const DescendLaunch A)
{
    __shared__ int s_ids[4][kMaxDegree];
    constexpr int NB = (VROWS == 1) ? 8 : 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *sids = s_ids[warp];
    const GraphView &g = A.g;
    const UpperView &u = A.u;
    const int nseg = g.dpad * 4 / 16;
    const int lg = lane_group_log2<VROWS, NB>(nseg);
    const int BS = (32 >> lg) * NB;
    const int gmask = (1 << lg) - 1;
    const bool rep_lane = (lane & gmask) < NB;
    const int my_slot = (lane >> lg) * NB + (lane & gmask);
    const int64_t nwarps = (int64_t)gridDim.x * 4;
    for (int64_t qn = (int64_t)blockIdx.x * 4 + warp; qn < A.nq; qn += nwarps) {
        const int64_t qi = A.rows ? (int64_t)A.rows[qn] : qn;   // the query's row
        float nq[VROWS][4];   // negated query (seg_tree)
        const float *Q = A.queries + qi * A.qstride;
#pragma unroll
        for (int r = 0; r < VROWS; r++) {
            const int seg = (lane & gmask) + 32 * r;
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int j = seg * 4 + e;
                nq[r][e] = (seg < nseg && j < g.dim) ? -__ldg(Q + j) : 0.0f;
            }
        }
        int cur = u.entry, hops = 0;
        float curd;
        {   // distance to the top entry
            if (lane == 0) sids[0] = cur;
            __syncwarp();
            uint4 raw[NB][VROWS];
            float scale[NB];
            gather_batch<kF32, VROWS, NB>(g, sids, 0, 1, nseg, lane, lg, raw, scale);
            curd = __shfl_sync(kFull, batch_distances<kF32, VROWS, NB>(nq, raw, scale, lane, lg), 0);
            __syncwarp();
        }
        for (int level = u.max_level; level > 0; level--) {
            for (;;) {
                int cnt = 0;
                const int32_t *row = nullptr;
                if (__ldg(u.levels + cur) >= level) {
                    row = u.rows + (__ldg(u.row_start + cur) + level - 1) * u.stride;
                    cnt = __ldg(row);
                }
                hops++;
                for (int i = lane; i < cnt; i += 32) sids[i] = __ldg(row + 16 + i);
                __syncwarp();
                float bestd = curd;
                int best = -1;   // first slot with the smallest distance below curd
                uint4 raw[NB][VROWS];
                float scale[NB];
                if (cnt > 0) gather_batch<kF32, VROWS, NB>(g, sids, 0, cnt, nseg, lane, lg, raw, scale);
                for (int b0 = 0; b0 < cnt; b0 += BS) {
                    const float dist = batch_distances<kF32, VROWS, NB>(nq, raw, scale, lane, lg);
                    if (b0 + BS < cnt) gather_batch<kF32, VROWS, NB>(g, sids, b0 + BS, cnt, nseg, lane, lg, raw, scale);
                    const bool in = rep_lane && b0 + my_slot < cnt;
                    // distances are >= +0: their bit patterns order like the floats
                    const uint32_t mb = __reduce_min_sync(kFull, in ? __float_as_uint(dist) : 0xffffffffu);
                    const float md = __uint_as_float(mb);
                    if (md < bestd) {   // strictly better than every earlier slot
                        const unsigned at = __ballot_sync(kFull, in && __float_as_uint(dist) == mb);
                        const int t = __ffs(at) - 1;   // representative lanes ascend with the slots
                        bestd = md;
                        best = b0 + (t >> lg) * NB + (t & gmask);
                    }
                }
                if (best >= 0) { cur = sids[best]; curd = bestd; }
                __syncwarp();
                if (best < 0) break;
            }
        }
        if (lane == 0) {
            A.out_entry[qi * (A.out_entry_stride > 0 ? A.out_entry_stride : 1)] = cur;
            if (A.out_hops) A.out_hops[qn] = hops;
        }
    }
}

// The same descent with one block of four warps per query, for small batches
// (at batch 1 the warp-per-query kernel pays one gather round trip per batch
// of BS slots, four per 32-id row).  Warp w takes the slots [w*BS, (w+1)*BS)
// of every 4*BS, so a row of up to 4*BS ids costs one gather round trip; each
// warp reduces its slots to (smallest distance bits, first slot) and the four
// pairs are combined in the same lexicographic order, which picks the row's
// first slot with the smallest distance, as the one-warp scan does.  Every
// warp reads the node's level and row itself (the same addresses), so a hop
// takes one block barrier.
template <int VROWS>
__global__ void __launch_bounds__(128) descend_block_kernel(const DescendLaunch A)
{
    __shared__ int s_ids[4][kMaxDegree];
    __shared__ unsigned long long s_best[2][4];   // per hop parity: (distance bits << 32) | slot
    constexpr int NB = (VROWS == 1) ? 8 : 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *sids = s_ids[warp];
    const GraphView &g = A.g;
    const UpperView &u = A.u;
    const int nseg = g.dpad * 4 / 16;
    const int lg = lane_group_log2<VROWS, NB>(nseg);
    const int BS = (32 >> lg) * NB;
    const int gmask = (1 << lg) - 1;
    const bool rep_lane = (lane & gmask) < NB;
    const int my_slot = (lane >> lg) * NB + (lane & gmask);
    for (int64_t qn = blockIdx.x; qn < A.nq; qn += gridDim.x) {
        const int64_t qi = A.rows ? (int64_t)A.rows[qn] : qn;
        float nq[VROWS][4];   // negated query (seg_tree)
        const float *Q = A.queries + qi * A.qstride;
#pragma unroll
        for (int r = 0; r < VROWS; r++) {
            const int seg = (lane & gmask) + 32 * r;
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int j = seg * 4 + e;
                nq[r][e] = (seg < nseg && j < g.dim) ? -__ldg(Q + j) : 0.0f;
            }
        }
        int cur = u.entry, hops = 0;
        float curd;
        {   // distance to the top entry (every warp, the same value)
            if (lane == 0) sids[0] = cur;
            __syncwarp();
            uint4 raw[NB][VROWS];
            float scale[NB];
            gather_batch<kF32, VROWS, NB>(g, sids, 0, 1, nseg, lane, lg, raw, scale);
            curd = __shfl_sync(kFull, batch_distances<kF32, VROWS, NB>(nq, raw, scale, lane, lg), 0);
            __syncwarp();
        }
        int par = 0;
        for (int level = u.max_level; level > 0; level--) {
            for (;;) {
                int cnt = 0;
                const int32_t *row = nullptr;
                if (__ldg(u.levels + cur) >= level) {
                    row = u.rows + (__ldg(u.row_start + cur) + level - 1) * u.stride;
                    cnt = __ldg(row);
                }
                hops++;
                // this warp's slots: [b*BS, (b+1)*BS) for b = warp, warp + 4, ...
                uint32_t mbits = 0xffffffffu;
                int mslot = 0x7fffffff;
                for (int base = warp * BS; base < cnt; base += 4 * BS) {
                    const int n = min(BS, cnt - base);
                    for (int i = lane; i < n; i += 32) sids[i] = __ldg(row + 16 + base + i);
                    __syncwarp();
                    uint4 raw[NB][VROWS];
                    float scale[NB];
                    gather_batch<kF32, VROWS, NB>(g, sids, 0, n, nseg, lane, lg, raw, scale);
                    const float dist = batch_distances<kF32, VROWS, NB>(nq, raw, scale, lane, lg);
                    const bool in = rep_lane && my_slot < n;
                    // distances are >= +0: their bit patterns order like the floats
                    const uint32_t mb = __reduce_min_sync(kFull, in ? __float_as_uint(dist) : 0xffffffffu);
                    const unsigned at = __ballot_sync(kFull, in && __float_as_uint(dist) == mb);
                    if (at && mb < mbits) {   // earlier batches of this warp hold lower slots
                        const int t = __ffs(at) - 1;
                        mbits = mb;
                        mslot = base + (t >> lg) * NB + (t & gmask);
                    }
                    __syncwarp();
                }
                if (lane == 0) s_best[par][warp] = ((unsigned long long)mbits << 32) | (unsigned)mslot;
                __syncthreads();
                unsigned long long b = s_best[par][0];
#pragma unroll
                for (int w = 1; w < 4; w++) b = min(b, s_best[par][w]);
                par ^= 1;
                const uint32_t bb = (uint32_t)(b >> 32);
                if (bb == 0xffffffffu || !(__uint_as_float(bb) < curd)) break;
                cur = __ldg(row + 16 + (int)(b & 0xffffffffu));
                curd = __uint_as_float(bb);
            }
        }
        if (threadIdx.x == 0) {
            A.out_entry[qi * (A.out_entry_stride > 0 ? A.out_entry_stride : 1)] = cur;
            if (A.out_hops) A.out_hops[qn] = hops;
        }
    }
}

// ---------------------------------------------------------------------------
// Exact FP32 rerank of the final ef candidates of a reduced-precision
// traversal (extension beyond the reference): one warp per query, the same
// adder tree on the FP32 vectors, stable ascending order (ties keep the
// traversal order), top k written with labels.
// ---------------------------------------------------------------------------
// One query's rerank: FP32 tree distances of its ef candidates (physical ids,
// best-first, -1 = empty), stable ascending order, top k written with labels.
// sd/si: ef floats/ints of per-warp scratch (shared memory).
template <int VROWS>
__device__ void rerank_one(const GraphView &g, const QParams &P, const float *Q, const int32_t *cand, int32_t *orow,
                           float *drow, int out_stride, float *sd, int *si, int lane)
{
    constexpr int NB = (VROWS == 1) ? 8 : 4;
    const int nseg = g.dpad * 4 / 16;
    float nq[VROWS][4];   // negated query (seg_tree)
#pragma unroll
    for (int r = 0; r < VROWS; r++) {
        const int seg = lane + 32 * r;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int j = seg * 4 + e;
            nq[r][e] = (seg < nseg && j < g.dim) ? -__ldcg(Q + j) : 0.0f;
        }
    }
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
        const float dist = batch_distances<kF32, VROWS, NB>(nq, raw, scale, lane);
        if (lane < NB && b0 + lane < P.ef) {
            const int id = ids[lane];
            sd[b0 + lane] = (id >= 0) ? dist : kLarge;
            si[b0 + lane] = id;
        }
    }
    __syncwarp();
    for (int i = lane; i < P.ef; i += 32) {
        const float di = sd[i];
        int rank = 0;
        for (int j = 0; j < P.ef; j++) {
            const float dj = sd[j];
            rank += (dj < di) || (dj == di && j < i);
        }
        if (rank < P.k) {
            int id = si[i];
            if (g.labels && id >= 0) id = g.labels[id];
            orow[rank] = id;
            drow[rank] = di;
        }
    }
    for (int i = P.k + lane; i < out_stride; i += 32) { orow[i] = -1; drow[i] = kLarge; }
    __syncwarp();
}

template <int VROWS>
__global__ void __launch_bounds__(128) rerank_kernel(const RerankLaunch A)
{
    __shared__ float sd[4][kMaxEf];
    __shared__ int si[4][kMaxEf];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t qi = (int64_t)blockIdx.x * 4 + warp; qi < A.nq; qi += (int64_t)gridDim.x * 4) {
        const QParams P = A.params[A.per_query ? qi : 0];
        rerank_one<VROWS>(A.g, P, A.queries + qi * A.qstride, A.cand_ids + qi * A.cand_stride,
                          A.out_ids + qi * A.out_stride, A.out_d + qi * A.out_stride, A.out_stride, sd[warp],
                          si[warp], lane);
    }
}

// ---------------------------------------------------------------------------
// Serving kernel: a persistent grid whose warps pull requests one at a time
// from the claim queue of one request class (precision x register rows),
// which the host keeps appending to while the kernel runs (continuous
// batching: a request admitted while others are in flight starts as soon as
// a warp is free).  A request names a resident index, its precision and its
// own k/ef/mc/mg; results, hops and visited go to host-mapped memory, then a
// per-entry done word (seq + 1) is released to the host.  Claiming uses
// compare-and-swap so no request is ever claimed before it is published.
// Every wait is bounded: a warp that finds no work sleeps and leaves after
// its class has had no claim or completion for `idle_ns` (or at once when
// `stop` is set), and every warp leaves between requests once the host sets
// its class's yield_epoch to this launch's epoch (the host re-partitions the
// SMs between the classes with work); the host relaunches a class kernel when
// its class has work waiting.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long load_acquire_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ long long global_ns()
{
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Exact FP32 rerank of a served request's ef candidates (the warp's scratch
// row).  Everything it needs is reloaded from the ring entry, so nothing of
// the request stays live in registers through the traversal.  FP32 rows:
// BF16 one row -> 1..2, BF16 two rows -> 3..4, FP8 -> 1..4.
template <int ELEM, int VROWS>
__device__ __forceinline__ void serve_rerank(const ServeLaunch &S, int e, float *rsd, int *rsi, int lane)
{
    ServeDesc D;
    {
        const int *src = reinterpret_cast<const int *>(S.ring + e);
        int *dst = reinterpret_cast<int *>(&D);
#pragma unroll
        for (int w = 0; w < (int)(sizeof(ServeDesc) / sizeof(int)); w++) dst[w] = __ldcg(src + w);
    }
    const GraphView &v = S.views[D.index];
    const int32_t *cand_ids = S.cand_ids + ((size_t)S.warp_base + (size_t)blockIdx.x * 4 + (threadIdx.x >> 5)) * S.ef_max;
    const float *query = S.qpool + (int64_t)e * S.qstride;
    int32_t *orow = S.out_ids + (int64_t)e * S.out_stride;
    float *drow = S.out_d + (int64_t)e * S.out_stride;
    const int vr32 = serve_vrows(v.dpad, kF32);
    if ((ELEM == kFP8 || VROWS == 1) && vr32 <= 1)
        rerank_one<1>(v, D.p, query, cand_ids, orow, drow, S.out_stride, rsd, rsi, lane);
    else if ((ELEM == kFP8 || VROWS == 1) && vr32 == 2)
        rerank_one<2>(v, D.p, query, cand_ids, orow, drow, S.out_stride, rsd, rsi, lane);
    else if ((ELEM == kFP8 || VROWS == 2) && vr32 == 3)
        rerank_one<3>(v, D.p, query, cand_ids, orow, drow, S.out_stride, rsd, rsi, lane);
    else if (ELEM == kFP8 || VROWS == 2)
        rerank_one<4>(v, D.p, query, cand_ids, orow, drow, S.out_stride, rsd, rsi, lane);
}

// One serving kernel per request class (precision ELEM, VROWS register rows):
// a single traversal variant per kernel keeps the hop loop free of spills.
template <int ELEM, int EPL, int VROWS>
__global__ void __launch_bounds__(128, 3) serve_kernel(const ServeLaunch S)
{
    extern __shared__ uint4 smem_u4[];
    constexpr int CLS = serve_class(ELEM, VROWS);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    using Caps = ListCaps<EPL>;
    const size_t wbytes =
        serve_warp_smem_bytes(S.bloom_bits_max, S.mc_max, S.mg_max, Caps::heap, Caps::r, Caps::c, S.ef_max);
    unsigned char *wbase = reinterpret_cast<unsigned char *>(smem_u4) + wbytes * warp;
    const bool smem_bloom = S.bloom_bits_max <= kMaxSmemBloomBits;
    const size_t bloom_bytes = (size_t)1 << (S.bloom_bits_max - 3);
    const size_t gw = (size_t)S.warp_base + (size_t)blockIdx.x * 4 + warp;   // this warp's scratch slot
    uint32_t *gbloom = smem_bloom ? nullptr : S.bloom_global + gw * (bloom_bytes / 4);
    const WarpSmem W = carve_warp_smem(wbase, gbloom, smem_bloom, bloom_bytes, Caps::heap, Caps::r, Caps::c, S.mc_max,
                                       S.mg_max);
    // rerank scratch: the bucketed list's space once the traversal has written
    // its results, else ef_max slots after the warp's traversal state
    float *rsd = Caps::heap ? reinterpret_cast<float *>(W.hkey)
                            : reinterpret_cast<float *>(wbase + wbytes - serve_rerank_bytes(S.ef_max));
    int *rsi = Caps::heap ? reinterpret_cast<int *>(W.hkey) + S.ef_max : reinterpret_cast<int *>(rsd + S.ef_max);
    int32_t *cand_ids = S.cand_ids + gw * S.ef_max;
    float *cand_d = S.cand_d + gw * S.ef_max;
    const int32_t *slots = S.class_slots + (size_t)CLS * S.ring_cap;
    uint32_t epoch = 0;
    long long t_start = 0;   // a launch counts its own start as activity of its class
    if (lane == 0) {
        epoch = reinterpret_cast<const volatile uint32_t *>(S.run_epoch)[CLS];
        t_start = global_ns();
    }

    for (;;) {
        unsigned long long h = ~0ull;
        int yielded = 0;
        if (lane == 0) {
            // the host hands the GPU to another class: leave between requests
            yielded = *reinterpret_cast<volatile uint32_t *>(&S.ctl->yield_epoch[CLS]) == epoch;
            for (int tries = 0; !yielded && tries < 256; tries++) {
                const unsigned long long hd = atomicAdd(&S.ctl->head[CLS], 0ull);
                const unsigned long long tl = load_acquire_u64(&S.ctl->tail[CLS]);
                if (hd >= tl) break;
                if (atomicCAS(&S.ctl->head[CLS], hd, hd + 1) == hd) { h = hd; break; }
            }
            if (h != ~0ull) atomicMax(&S.ctl->last_active_ns[CLS], global_ns());
        }
        if (__shfl_sync(kFull, yielded, 0)) break;
        h = __shfl_sync(kFull, h, 0);
        if (h == ~0ull) {
            // leave only when this class has been idle for idle_ns
            int leave = 0;
            if (lane == 0) {
                const int stop = *reinterpret_cast<volatile int *>(&S.ctl->stop);
                long long last = *reinterpret_cast<volatile long long *>(&S.ctl->last_active_ns[CLS]);
                if (last < t_start) last = t_start;
                leave = stop || (global_ns() - last > S.idle_ns);
            }
            if (__shfl_sync(kFull, leave, 0)) break;
            __nanosleep(1000);
            continue;
        }
        const int e = __ldcg(slots + (int)(h % (unsigned long long)S.ring_cap));
        ServeDesc D;
        {
            const int *src = reinterpret_cast<const int *>(S.ring + e);
            int *dst = reinterpret_cast<int *>(&D);
#pragma unroll
            for (int w = 0; w < (int)(sizeof(ServeDesc) / sizeof(int)); w++) dst[w] = __ldcg(src + w);
        }
        const GraphView &v = S.views[D.index];
        const bool rerank = ELEM != kF32 && D.p.rerank != 0;
        QueryIO io;
        io.query = S.qpool + (int64_t)e * S.qstride;
        io.entry = D.entry;
        io.out_ids = rerank ? cand_ids : S.out_ids + (int64_t)e * S.out_stride;
        io.out_d = rerank ? cand_d : S.out_d + (int64_t)e * S.out_stride;
        io.out_stride = rerank ? S.ef_max : S.out_stride;
        io.write_all_ef = rerank ? 1 : 0;
        io.hops = S.out_hops + e;
        io.visited = S.out_visited + e;
        io.status = S.status;
        search_one_inter<ELEM, EPL, VROWS, kRowBloom<ELEM, VROWS>>(v, D.p, io, W.bloom, W.fifo, W.fifo_len, W.sids,
                                                                   W.hkey, W.hid, lane);
        if constexpr (ELEM != kF32) {
            if (rerank) {
                __syncwarp();
                serve_rerank<ELEM, VROWS>(S, e, rsd, rsi, lane);
            }
        }
        __syncwarp();
        if (lane == 0) {
            __threadfence_system();
            *reinterpret_cast<volatile unsigned long long *>(S.done + e) = D.seq + 1;
            atomicMax(&S.ctl->last_active_ns[CLS], global_ns());
        }
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
cudaError_t launch_inter(const SearchLaunch &a, size_t, int num_sms, cudaStream_t s, int64_t *slots)
{
    // the trace variant (a.trace_counts set) exists for FP32 only
    constexpr bool kTrace = (ELEM == kF32);
    auto kern = (kTrace && a.trace_counts) ? inter_kernel<ELEM, EPL, VROWS, kTrace> : inter_kernel<ELEM, EPL, VROWS, false>;
    if (a.trace_counts && !kTrace) return cudaErrorInvalidValue;
    using Caps = ListCaps<EPL>;
    const size_t smem_block = warp_smem_bytes(a.bloom_bits_max, a.mc_max, a.mg_max, Caps::heap, Caps::r, Caps::c) * 4;
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
    if (slots) {
        *slots = blocks * 4;
        return cudaSuccess;
    }
    kern<<<(unsigned)blocks, 128, smem_block, s>>>(a);
    return cudaGetLastError();
}

template <int ELEM, int EPL, int VROWS>
cudaError_t launch_intra(const SearchLaunch &a, int channels, int num_sms, cudaStream_t s, int64_t *slots)
{
    auto kern = intra_kernel<ELEM, EPL, VROWS>;
    using Caps = ListCaps<EPL, true>;
    const size_t smem = intra_smem_bytes(a, channels, Caps::heap, Caps::r, Caps::c);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    // warps per channel: a batch smaller than the SMs gets up to 16 warps per
    // query (latency), a larger one a warp per channel (throughput)
    int wpc = 1;
    if (a.nq <= num_sms) wpc = (kIntraMaxWarps - 1) / channels;
    if (wpc < 1) wpc = 1;
    const int threads = 32 * (channels * wpc + 1);   // fetch warps and the merge warp
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int64_t blocks = (int64_t)per_sm * num_sms;
    if (blocks > a.nq) blocks = a.nq;
    if (blocks < 1) blocks = 1;
    if (slots) {
        *slots = blocks * channels;
        return cudaSuccess;
    }
    kern<<<(unsigned)blocks, threads, smem, s>>>(a);
    return cudaGetLastError();
}

// Entries per lane: the result list needs ef <= 32*EPL, the candidate list
// cq <= 32*CPL with CPL = EPL/4 for EPL >= 8.
inline int pick_epl(int ef_max, int cq_max)
{
    int epl = 2;
    while (32 * epl < ef_max) epl *= 2;
    if (cq_max > 32) {
        int cpl = 2;
        while (32 * cpl < cq_max) cpl *= 2;
        if (4 * cpl > epl) epl = 4 * cpl;
    }
    return epl;
}

template <int ELEM, int VROWS>
cudaError_t dispatch_epl(const SearchLaunch &a, size_t smem_block, int num_sms, cudaStream_t s, int64_t *slots)
{
    const int epl = pick_epl(a.ef_max, a.cq_max);
    if (a.channels > 0) {
        switch (epl) {
            case 2: return launch_intra<ELEM, 2, VROWS>(a, a.channels, num_sms, s, slots);
            case 4: return launch_intra<ELEM, 4, VROWS>(a, a.channels, num_sms, s, slots);
            case 8: return launch_intra<ELEM, 8, VROWS>(a, a.channels, num_sms, s, slots);
            case 16: return launch_intra<ELEM, 16, VROWS>(a, a.channels, num_sms, s, slots);
            case 32: return launch_intra<ELEM, 32, VROWS>(a, a.channels, num_sms, s, slots);
        }
        return cudaErrorInvalidValue;
    }
    switch (epl) {
        case 2: return launch_inter<ELEM, 2, VROWS>(a, smem_block, num_sms, s, slots);
        case 4: return launch_inter<ELEM, 4, VROWS>(a, smem_block, num_sms, s, slots);
        case 8: return launch_inter<ELEM, 8, VROWS>(a, smem_block, num_sms, s, slots);
        case 16: return launch_inter<ELEM, 16, VROWS>(a, smem_block, num_sms, s, slots);
        case 32: return launch_inter<ELEM, 32, VROWS>(a, smem_block, num_sms, s, slots);
    }
    return cudaErrorInvalidValue;
}

}  // namespace

static cudaError_t search_dispatch(const SearchLaunch &a, int elem, int num_sms, cudaStream_t s, int64_t *slots)
{
    const size_t smem_block = 0;   // each launcher sizes its own shared memory
    const int seg_bytes = (elem == kF32) ? 4 : (elem == kBF16 ? 2 : 1);
    const int nseg = a.g.dpad * seg_bytes / 16;
    const int vrows = (nseg + 31) / 32;
    if (elem == kF32) {
        switch (vrows) {
            case 1: return dispatch_epl<kF32, 1>(a, smem_block, num_sms, s, slots);
            case 2: return dispatch_epl<kF32, 2>(a, smem_block, num_sms, s, slots);
            case 3: return dispatch_epl<kF32, 3>(a, smem_block, num_sms, s, slots);
            case 4: return dispatch_epl<kF32, 4>(a, smem_block, num_sms, s, slots);
        }
    } else if (elem == kBF16) {
        switch (vrows) {
            case 1: return dispatch_epl<kBF16, 1>(a, smem_block, num_sms, s, slots);
            case 2: return dispatch_epl<kBF16, 2>(a, smem_block, num_sms, s, slots);
        }
    } else if (elem == kFP8) {
        if (vrows == 1) return dispatch_epl<kFP8, 1>(a, smem_block, num_sms, s, slots);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_descend(const DescendLaunch &a, int num_sms, cudaStream_t s)
{
    if (a.nq <= 0) return cudaSuccess;
    const int vrows = (a.g.dpad * 4 / 16 + 31) / 32;
    if (a.nq <= (int64_t)num_sms * 4) {   // small batches: a block per query
        const unsigned nb = (unsigned)a.nq;
        switch (vrows) {
            case 1: descend_block_kernel<1><<<nb, 128, 0, s>>>(a); break;
            case 2: descend_block_kernel<2><<<nb, 128, 0, s>>>(a); break;
            case 3: descend_block_kernel<3><<<nb, 128, 0, s>>>(a); break;
            case 4: descend_block_kernel<4><<<nb, 128, 0, s>>>(a); break;
            default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
    int64_t blocks = (a.nq + 3) / 4;
    const int64_t cap = (int64_t)num_sms * 8;
    if (blocks > cap) blocks = cap;
    switch (vrows) {
        case 1: descend_kernel<1><<<(unsigned)blocks, 128, 0, s>>>(a); break;
        case 2: descend_kernel<2><<<(unsigned)blocks, 128, 0, s>>>(a); break;
        case 3: descend_kernel<3><<<(unsigned)blocks, 128, 0, s>>>(a); break;
        case 4: descend_kernel<4><<<(unsigned)blocks, 128, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_search(const SearchLaunch &a, int elem, int num_sms, cudaStream_t s)
{
    return search_dispatch(a, elem, num_sms, s, nullptr);
}

cudaError_t search_bloom_slots(const SearchLaunch &a, int elem, int num_sms, int64_t *slots)
{
    return search_dispatch(a, elem, num_sms, nullptr, slots);
}

template <int ELEM, int EPL, int VROWS>
static cudaError_t serve_config_t(const ServeLaunch &sv, int num_sms, int *grid, size_t *smem)
{
    const int heap_cap = (EPL > 8) ? 32 * EPL : 0;
    using Caps = ListCaps<EPL>;
    (void)heap_cap;
    *smem = serve_warp_smem_bytes(sv.bloom_bits_max, sv.mc_max, sv.mg_max, Caps::heap, Caps::r, Caps::c, sv.ef_max) * 4;
    cudaError_t e = cudaFuncSetAttribute(serve_kernel<ELEM, EPL, VROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)*smem);
    int per_sm = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_kernel<ELEM, EPL, VROWS>, 128, *smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    *grid = per_sm * num_sms;
    return cudaSuccess;
}

template <int EPL>
static cudaError_t serve_config_c(const ServeLaunch &sv, int cls, int num_sms, int *grid, size_t *smem)
{
    switch (cls) {
        case serve_class(kF32, 1): return serve_config_t<kF32, EPL, 1>(sv, num_sms, grid, smem);
        case serve_class(kF32, 2): return serve_config_t<kF32, EPL, 2>(sv, num_sms, grid, smem);
        case serve_class(kF32, 3): return serve_config_t<kF32, EPL, 3>(sv, num_sms, grid, smem);
        case serve_class(kF32, 4): return serve_config_t<kF32, EPL, 4>(sv, num_sms, grid, smem);
        case serve_class(kBF16, 1): return serve_config_t<kBF16, EPL, 1>(sv, num_sms, grid, smem);
        case serve_class(kBF16, 2): return serve_config_t<kBF16, EPL, 2>(sv, num_sms, grid, smem);
        case serve_class(kFP8, 1): return serve_config_t<kFP8, EPL, 1>(sv, num_sms, grid, smem);
    }
    return cudaErrorInvalidValue;
}

cudaError_t serve_config(const ServeLaunch &sv, int epl, int cls, int num_sms, int *grid, size_t *smem)
{
    if (epl == 8) return serve_config_c<8>(sv, cls, num_sms, grid, smem);
    if (epl == 32) return serve_config_c<32>(sv, cls, num_sms, grid, smem);
    return cudaErrorInvalidValue;
}

template <int EPL>
static cudaError_t launch_serve_c(const ServeLaunch &sv, int cls, int grid, size_t smem, cudaStream_t st)
{
    switch (cls) {
        case serve_class(kF32, 1): serve_kernel<kF32, EPL, 1><<<grid, 128, smem, st>>>(sv); break;
        case serve_class(kF32, 2): serve_kernel<kF32, EPL, 2><<<grid, 128, smem, st>>>(sv); break;
        case serve_class(kF32, 3): serve_kernel<kF32, EPL, 3><<<grid, 128, smem, st>>>(sv); break;
        case serve_class(kF32, 4): serve_kernel<kF32, EPL, 4><<<grid, 128, smem, st>>>(sv); break;
        case serve_class(kBF16, 1): serve_kernel<kBF16, EPL, 1><<<grid, 128, smem, st>>>(sv); break;
        case serve_class(kBF16, 2): serve_kernel<kBF16, EPL, 2><<<grid, 128, smem, st>>>(sv); break;
        case serve_class(kFP8, 1): serve_kernel<kFP8, EPL, 1><<<grid, 128, smem, st>>>(sv); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_serve(const ServeLaunch &sv, int epl, int cls, int grid, size_t smem, cudaStream_t st)
{
    if (epl == 8) return launch_serve_c<8>(sv, cls, grid, smem, st);
    if (epl == 32) return launch_serve_c<32>(sv, cls, grid, smem, st);
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
