// Internal structures shared by the traversal kernels and the C-ABI layer.
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace falcon {

constexpr float kLarge = 1e20f;   // constants.hpp:14 large_float

enum Elem { kF32 = 0, kBF16 = 1, kFP8 = 2 };

// Limits of the built kernels.
constexpr int kMaxEf = 1024;
constexpr int kMaxCandQueue = 256;
constexpr int kMaxMc = 8;
constexpr int kMaxMg = 16;
constexpr int kMaxDegree = 128;
constexpr int kMaxBloomBits = 24;
constexpr int kMaxSmemBloomBits = 18;   // larger filters live in global memory, one slot per warp/channel
constexpr int kMinBloomBits = 10;
constexpr int kMaxDimPadded = 512;
constexpr int kMaxChannels = 8;
// Neighbour ids staged per warp: a whole adjacency row of up to 64 ids.
constexpr int kSidsPerWarp = 64;

// Device view of one resident graph.
struct GraphView {
    const unsigned char *vecs;      // traversal storage (f32 / bf16 / fp8 codes)
    int64_t vstride_bytes;
    const float *scales;            // fp8: one scale per vector
    const unsigned char *vecs32;    // FP32 storage (rerank), may equal vecs
    int64_t vstride32_bytes;
    const int32_t *links;           // count at row*lstride, ids at row*lstride+ids_off
    int64_t lstride;
    int32_t ids_off;
    int32_t max_degree;
    int32_t dim;
    int32_t dpad;
    int64_t n;
    const int32_t *labels;          // may be null
};

// HNSW upper layers on the device: node v's level-l row (1 <= l <= levels[v])
// is rows + (row_start[v] + l - 1) * stride, count at [0], ids from [16].
struct UpperView {
    const int32_t *rows;
    int64_t stride;                 // int32 per row (16 * (1 + ceil(max_degree / 16)))
    const int64_t *row_start;       // per node
    const int32_t *levels;          // per node (0 = base layer only)
    int32_t max_level;              // top level (>= 1)
    int32_t max_degree;             // ids per upper row
    int32_t entry;                  // top-level entry node
};

// Greedy descent of the upper layers for nq queries: the base-layer entry of
// each query (and the number of upper rows expanded).
struct DescendLaunch {
    GraphView g;                    // FP32 vectors (vecs = vecs32)
    UpperView u;
    const float *queries;
    int64_t qstride;
    int64_t nq;
    int32_t *out_entry;
    int64_t out_entry_stride;       // int32 units between queries' entries (0: contiguous)
    int32_t *out_hops;              // may be null
    const int32_t *rows;            // may be null: query i is row rows[i] of queries and of out_entry
};

// Per-query search parameters as the kernels read them.
struct QParams {
    int32_t k, ef, mc, mg, cq, bloom_bits;
    uint32_t seed;
    int32_t mode, channels, precision, rerank, max_hops;
};

struct SearchLaunch {
    GraphView g;
    const float *queries;
    int64_t qstride;
    const int32_t *entries;         // may be null
    int32_t default_entry;
    int64_t nq;
    const QParams *params;          // device array (1 or nq)
    int32_t per_query;
    // result rows: out_ids[q*out_stride + i] for i < (rerank ? ef : k)
    int32_t *out_ids;
    float *out_d;
    int32_t out_stride;
    int32_t write_all_ef;           // 1: write ef results (rerank input), physical ids
    int32_t *out_hops;
    int32_t *out_visited;
    int32_t *work_counter;          // zeroed before launch
    int32_t *status;                // bit 0: some query hit max_hops
    int32_t bloom_bits_max;         // shared-memory Bloom size per warp/channel
    int32_t ef_max;
    int32_t mc_max, mg_max;
    int32_t channels;               // 0: inter-query (warp per query); else intra-query block of `channels` warps
    int32_t cq_max;                 // largest candidate queue of the call
    uint32_t *bloom_global;         // bloom_bits_max > kMaxSmemBloomBits: per-warp filters in global memory
    // traversal trace (FP32 inter-query only; null = off): per query trace_cand_cap
    // (distance, computed count) and trace_cap (distance, id) entries, 3 counts
    float *trace_cand_d;
    int32_t *trace_cand_n;
    int32_t trace_cand_cap;
    float *trace_d;
    int32_t *trace_id;
    int32_t trace_cap;
    int32_t *trace_counts;
};

struct RerankLaunch {
    GraphView g;
    const float *queries;
    int64_t qstride;
    int64_t nq;
    const QParams *params;
    int32_t per_query;
    const int32_t *cand_ids;        // nq x cand_stride physical ids (best-first)
    int32_t cand_stride;
    int32_t *out_ids;
    float *out_d;
    int32_t out_stride;
};

// Serving: one published request (device ring entry).
struct ServeDesc {
    int32_t index;                  // registered index
    int32_t precision;              // kF32 / kBF16 / kFP8
    int32_t entry;                  // entry point
    int32_t pad;
    unsigned long long seq;         // request sequence number
    QParams p;
};

// Serving kernels are specialised per request class, the traversal precision
// and the 16-byte register rows per lane its vectors take: FP32 1..4, BF16
// 1..2, FP8 1.  One kernel holding several traversal variants (called or
// inlined) spills inside the hop loop, so each class has its own kernel and
// its own claim queue; the kernels of the classes with work run at the same
// time, each on its own stream over a share of the SMs.
constexpr int kServeClasses = 7;

__host__ __device__ constexpr int serve_class(int precision, int vrows)
{
    return precision == kF32 ? vrows - 1 : (precision == kBF16 ? 3 + vrows : 6);
}

// 16-byte register rows per lane of a padded dimension at a precision.
__host__ __device__ constexpr int serve_vrows(int dpad, int precision)
{
    return (dpad * (precision == kF32 ? 4 : (precision == kBF16 ? 2 : 1)) / 16 + 31) / 32;
}

struct ServeCtl {
    unsigned long long head[kServeClasses];   // per class queue: requests claimed by warps
    unsigned long long tail[kServeClasses];   // per class queue: requests published by the host
    long long last_active_ns[kServeClasses];  // per class: last claim or completion (globaltimer)
    uint32_t yield_epoch[kServeClasses];      // host: class c's launch with this epoch leaves between requests
    int32_t stop;                   // host: leave when idle
    int32_t error;
};

struct ServeLaunch {
    const GraphView *views;
    int32_t nviews;
    const ServeDesc *ring;
    int32_t ring_cap;
    const int32_t *class_slots;     // kServeClasses x ring_cap: ring entries in each class's claim order
    const uint32_t *run_epoch;      // host-mapped, per class: epoch of its current launch, read once at start
    const float *qpool;             // ring_cap x qstride (device)
    int32_t qstride;
    int32_t *out_ids;               // ring_cap x out_stride (host-mapped)
    float *out_d;
    int32_t out_stride;
    int32_t *out_hops;              // ring_cap (host-mapped)
    int32_t *out_visited;
    unsigned long long *done;       // ring_cap (host-mapped): seq + 1 when the entry's result is complete
    ServeCtl *ctl;
    int32_t *status;
    uint32_t *bloom_global;
    int32_t bloom_bits_max, mc_max, mg_max, ef_max, cq_max;
    int32_t *cand_ids;              // per warp ef_max (rerank candidates)
    float *cand_d;
    long long idle_ns;
    int32_t warp_base;              // first per-warp scratch slot (Bloom, rerank) of this launch
};

// Rerank scratch of a serving warp without the bucketed list: ef_max
// distances and ids.
__host__ __device__ inline size_t serve_rerank_bytes(int ef_max)
{
    return ((size_t)ef_max * (sizeof(float) + sizeof(int)) + 15) & ~(size_t)15;
}

// Shared memory of one serving warp: the traversal's (Bloom filter when it
// fits, bucketed result list of heap_cap slots or sorted lists of list_r +
// list_c slots, group FIFO, staged ids), then the rerank scratch unless the
// rerank reuses the bucketed list's space.
__host__ __device__ inline size_t serve_warp_smem_bytes(int bloom_bits_max, int mc_max, int mg_max, int heap_cap,
                                                        int list_r, int list_c, int ef_max)
{
    size_t b = (bloom_bits_max <= kMaxSmemBloomBits) ? ((size_t)1 << (bloom_bits_max - 3)) : 0;
    b += (size_t)heap_cap * (sizeof(uint64_t) + sizeof(int));
    b += (size_t)(list_r + list_c) * (sizeof(float) + sizeof(int));
    b += sizeof(int) * (size_t)(mc_max * mg_max + mg_max + kSidsPerWarp);
    b = (b + 15) & ~(size_t)15;
    if (heap_cap == 0) b += serve_rerank_bytes(ef_max);
    return b;
}

// Serving kernel of request class `cls` for entries-per-lane `epl` (8 or 32).
cudaError_t serve_config(const ServeLaunch &s, int epl, int cls, int num_sms, int *grid, size_t *smem);
cudaError_t launch_serve(const ServeLaunch &s, int epl, int cls, int grid, size_t smem, cudaStream_t st);

// A validated search request (host side), used by falcon_search_noalloc.
struct SearchPlan {
    int64_t np = 0;                 // number of parameter structs (1 or nq)
    int ef_max = 0, k_max = 0, mc_max = 1, mg_max = 1, bits_max = 10, cq_max = 1;
    int prec = 0, mode = 0, channels = 0;
    bool any_rerank = false;
    bool per_query = false;
};

// Launchers (falcon_kernels.cu).  Return cudaError_t of the launch.
cudaError_t launch_search(const SearchLaunch &a, int elem, int num_sms, cudaStream_t s);
// Number of Bloom-filter slots (warps or channel warps) launch_search will
// use for this launch; the global filter buffer must hold that many filters.
cudaError_t search_bloom_slots(const SearchLaunch &a, int elem, int num_sms, int64_t *slots);
cudaError_t launch_rerank(const RerankLaunch &a, int ef_max, int num_sms, cudaStream_t s);
cudaError_t launch_encode_bf16(const float *src, int64_t src_stride, int64_t n, int dim, int dpad, uint16_t *dst,
                               cudaStream_t s);
cudaError_t launch_encode_fp8(const float *src, int64_t src_stride, int64_t n, int dim, int dpad, uint8_t *dst,
                              float *scales, cudaStream_t s);
cudaError_t launch_descend(const DescendLaunch &a, int num_sms, cudaStream_t s);
// Number of kernel launches the last launch_search issued (for accounting).
int search_kernel_count();

}  // namespace falcon
