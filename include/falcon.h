/*
 * falcon.h -- C ABI of the B200 graph vector search library (libfalcon_b200.so).
 *
 * The library is a drop-in for the Falcon FPGA search path of
 * fpgasystems/Falcon-accelerate-graph-vector-search: best-first traversal of
 * an HNSW base layer or an NSG graph with delayed-synchronization traversal
 * (mc candidates per group, mg groups in flight), in inter-query mode (one
 * warp per query) and intra-query mode (one thread block per query, the
 * neighbour list split over channel warps, a merge warp merging one group
 * while the channel warps fetch the next).  Results, hop counts and visited
 * counts are bit-identical to the reference kernel's when distances are FP32.
 *
 * Conventions: every function returns an int status (FALCON_OK == 0, negative
 * on error, never aborts); falcon_last_error() gives a thread-local message.
 * Pointers are plain host or device pointers as flagged; no torch types.
 */
#ifndef FALCON_H
#define FALCON_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FALCON_OK 0
#define FALCON_WARN_TRUNCATED 1     /* some query stopped at max_hops */
#define FALCON_ERR_ARG (-1)         /* invalid argument */
#define FALCON_ERR_OOM (-2)         /* device or host allocation failed */
#define FALCON_ERR_CUDA (-3)        /* CUDA runtime error */
#define FALCON_ERR_IO (-4)          /* index file missing or malformed */
#define FALCON_ERR_GRAPH (-5)       /* graph invalid: id out of range, degree > max */
#define FALCON_ERR_UNSUPPORTED (-6) /* parameter combination not built */

/* base-vector storage formats (bit mask in falcon_index_desc.storage) */
#define FALCON_STORE_F32 1
#define FALCON_STORE_BF16 2
#define FALCON_STORE_FP8 4          /* OCP E4M3 codes + one FP32 scale per vector */

/* traversal precision (falcon_search_params.precision) */
#define FALCON_PREC_F32 0
#define FALCON_PREC_BF16 1
#define FALCON_PREC_FP8 2

/* search modes (falcon_search_params.mode) */
#define FALCON_MODE_INTER 0         /* one warp per query (reference inter-query v1.3) */
#define FALCON_MODE_INTRA 1         /* one block per query, `channels` warps (intra-query v1.5) */

/* memory flags for falcon_search */
#define FALCON_MEM_HOST 0
#define FALCON_MEM_DEVICE 1

typedef struct falcon_index falcon_index;

/*
 * Index description.  Replaces the buffers the reference host loads and
 * hands to its kernel (FPGA_multi_DDR/FPGA_inter_query_v1.3_longer_FIFO_alt_PR/
 * src/host.cpp:201-713 and vadd.cpp:11-95):
 *   links: adjacency rows; row r holds its neighbour count at
 *          links[r*link_stride] and the ids at links[r*link_stride+ids_offset+j].
 *          The reference file layout (64-byte header line, then the ids) is
 *          link_stride = 16*(1+ceil(max_degree/16)), ids_offset = 16.
 *   vectors: FP32, row r at vectors[r*vector_stride]; the first `dim` values
 *          are used (the reference layout has vector_stride = pad16(dim)+16).
 *   labels: optional physical-id -> label map applied to returned ids
 *          (host.cpp:1002-1007); NULL returns physical ids.
 * All pointers are host memory; the index copies what it needs to the device.
 */
typedef struct falcon_index_desc {
    int64_t num_vectors;
    int32_t dim;
    int32_t max_degree;
    const float *vectors;
    int64_t vector_stride;
    const int32_t *links;
    int64_t link_stride;
    int32_t ids_offset;
    int32_t entry_point;
    const int32_t *labels;
    int32_t storage;                /* FALCON_STORE_* mask; 0 = FP32 only */
    int32_t device;                 /* CUDA device ordinal */
} falcon_index_desc;

typedef struct falcon_index_info {
    int64_t num_vectors;
    int32_t dim, dim_padded, max_degree, entry_point, storage, device;
    int64_t device_bytes;           /* HBM held by the index */
} falcon_index_info;

/*
 * Search parameters.  Names follow the reference host (host.cpp:34-96):
 * mc = max_cand_per_group, mg = max_group_num_in_pipe,
 * cand_queue_size = candidate_queue_runtime_size (32 in the reference),
 * bloom_bits = runtime_n_bucket_addr_bits (16 for the 4-channel builds),
 * hash_seed = 1 in the reference.  k <= ef; k > ef raises ef to k.
 */
typedef struct falcon_search_params {
    int32_t k;
    int32_t ef;                     /* result queue size, 1..1024 (the reference hardware: <= 64) */
    int32_t mc;                     /* candidates per group, 1..8 */
    int32_t mg;                     /* groups in flight, 1..16 */
    int32_t cand_queue_size;        /* 1..256 (the reference hardware: <= 32) */
    int32_t bloom_bits;             /* 10..24; above 18 the filters live in global memory */
    uint32_t hash_seed;
    int32_t mode;                   /* FALCON_MODE_* */
    int32_t channels;               /* intra mode: 1,2,4,8 */
    int32_t precision;              /* FALCON_PREC_* (storage must hold it) */
    int32_t rerank;                 /* reduced precision: exact FP32 rerank of the final ef */
    int32_t max_hops;               /* 0 = unbounded; else traversal stops, status 1 */
} falcon_search_params;

/* Reference defaults: k=10, ef=64, mc=1, mg=1, cand_queue_size=32,
   bloom_bits=16, hash_seed=1, inter mode, FP32. */
void falcon_default_params(falcon_search_params *p);

/* Build a device-resident index from host arrays.  Replaces the host's file
   loading + buffer migration (host.cpp:201-713, 927). */
int falcon_index_create(const falcon_index_desc *desc, falcon_index **out);

/* Load the reference's FPGA index files (meta.bin, ground_links_{nc}_chan_{i}.bin,
   ground_vectors_{nc}_chan_{i}.bin, ground_labels.bin written by
   vector_search_baselines/scripts_hnsw/hnsw.py:264-377 and
   scripts_nsg/nsg_to_FPGA.py:56-137; read as host.cpp:201-278 reads them).
   The single-channel set is used when present, else the first complete set
   of nc = 2, 4, 8 or 16 channel files, whose rows (node i is row i / nc of
   channel i % nc, the writers' round robin) are put back in node order, as
   the multi-channel hosts read them (intra v1.5 host.cpp:242-260).
   graph_type is "HNSW" or "NSG". */
int falcon_index_load_fpga(const char *index_dir, const char *graph_type, int32_t dim, int32_t storage,
                           int32_t device, falcon_index **out);

int falcon_index_info_get(const falcon_index *ix, falcon_index_info *info);

/* Copy one resident storage array of the index back to host memory (for
   checkpointing the device-ready index, and for checking the encoders):
   which = FALCON_STORE_F32 (n x dim_padded floats), FALCON_STORE_BF16
   (n x dim_padded uint16 codes), FALCON_STORE_FP8 (n x dim_padded uint8 codes
   followed by n float scales).  `bytes` must equal the array size.  The
   reference keeps its index only in host files (hnsw.py:264-377); this has no
   kernel-side counterpart there. */
int falcon_index_copy_storage(const falcon_index *ix, int32_t which, void *dst, int64_t bytes);
/* Fails (FALCON_ERR_ARG) while a server holds the index: free the server first. */
int falcon_index_free(falcon_index *ix);

/*
 * HNSW upper layers (levels >= 1) for an index whose graph is an HNSW base
 * layer, in hnswlib's own arrangement (hnswalg.h:371-384, 588-616 of the
 * reference's vendored hnswlib; hnsw.py:230-262): node v lives on levels
 * 0..levels[v]; for 1 <= l <= levels[v] its level-l list is row
 * row_start[v] + l - 1 of `rows`, a row being row_stride int32: the count at
 * [0], the ids at [ids_offset ..].  Host arrays; copied to the device.
 * Replaces the reference multi-layer FPGA inputs meta.bin (max_level, entry),
 * upper_links.bin and upper_links_pointers.bin (FPGA_single_DDR/
 * FPGA_single_DDR_multi_layer_v2.2_async/src/host.cpp:66-161,
 * vadd.cpp ptr_to_upper_links/links_upper).
 *   max_level:   hnswlib maxlevel_ (>= 1)
 *   max_degree:  hnswlib maxM_ (ids per upper row, <= 128)
 *   entry_point: hnswlib enterpoint_node_ (a node with levels[v] == max_level)
 * Every id on level l must itself be on level l.  Errors: FALCON_ERR_GRAPH.
 */
typedef struct falcon_upper_layers_desc {
    int32_t max_level;
    int32_t max_degree;
    int32_t entry_point;
    int32_t ids_offset;
    int64_t num_rows;
    int64_t row_stride;
    const int32_t *levels;          /* num_vectors */
    const int64_t *row_start;       /* num_vectors (ignored where levels[v] == 0) */
    const int32_t *rows;            /* num_rows x row_stride */
} falcon_upper_layers_desc;

/* Fails (FALCON_ERR_ARG) once the index is registered with a server. */
int falcon_index_set_upper_layers(falcon_index *ix, const falcon_upper_layers_desc *desc);

/*
 * Greedy descent of the upper layers (hnswalg.h:514-541; the multi-layer
 * scheduler FPGA_single_DDR_multi_layer_v2.2_async/src/scheduler.hpp:116-144):
 * for each query, the base-layer entry point (mem_debug[2q] of the
 * multi-layer kernel) and the number of upper rows expanded.  FP32 distances
 * in the base search's order; requires FP32 storage and upper layers.
 * falcon_search and falcon_search_noalloc run this descent themselves when
 * the index has upper layers and entry_points is NULL.
 * memory as for falcon_search.
 */
int falcon_descend(falcon_index *ix, const float *queries, int64_t nq, int64_t query_stride,
                   int32_t *out_entry_points, int32_t *out_upper_hops, int32_t memory, void *stream);

/*
 * Search nq queries.  Replaces the kernel launch + result migration of the
 * reference host (host.cpp:852-993, vadd.cpp:11-95).
 *   queries:      nq rows of `dim` floats, row stride query_stride floats
 *   entry_points: per-query entry ids, or NULL: the upper-layer descent's
 *                 entry when the index has HNSW upper layers
 *                 (falcon_index_set_upper_layers), else the index entry
 *                 point (the reference's multi-DDR host sets every query to
 *                 the global entry, host.cpp:711-713)
 *   params:       one falcon_search_params, or nq of them when
 *                 per_query_params != 0 (mixed k/ef/mc in one launch);
 *                 always host memory (validated on the host, then copied to
 *                 the device on `stream`), whatever `memory` says
 *   out_ids/out_dists: nq rows of out_stride (>= every k); the first k of a
 *                 row are the results best-first, the rest -1 / 1e20
 *   out_hops/out_visited: per query (may be NULL); hops = 1 + popped
 *                 candidates, visited = Bloom-accepted neighbours
 *                 (the reference's mem_debug[2q], [2q+1])
 *   memory:       FALCON_MEM_HOST (pageable or pinned host buffers; copies are
 *                 made on `stream`) or FALCON_MEM_DEVICE (all buffers on the
 *                 index's device)
 *   stream:       cudaStream_t (NULL = the legacy default stream); the call
 *                 returns after the results are in place for host memory and
 *                 after enqueueing for device memory.
 */
int falcon_search(falcon_index *ix, const float *queries, int64_t nq, int64_t query_stride,
                  const int32_t *entry_points, const falcon_search_params *params, int32_t per_query_params,
                  int32_t *out_ids, float *out_dists, int32_t out_stride, int32_t *out_hops,
                  int32_t *out_visited, int32_t memory, void *stream);

/*
 * Search with the traversal trace: the reference's trace kernel
 * (FPGA_multi_DDR/eval_trace_FPGA_inter_query_v1.3: vadd's
 * debug_out_per_query_{cand_dists, cand_num_neighbors, dists, ids}, written by
 * DRAM_utils.hpp:389-474) as per-query arrays instead of -1/-2-delimited
 * streams.  Results as falcon_search (one params struct: FP32, inter-query
 * mode, no rerank).  Per query q:
 *   trace_cand_dists/counts [q * cand_capacity + i]: the i-th expanded
 *       candidate's distance (1e20 for the entry point, which is not
 *       distance-computed) and the number of distances computed for its row;
 *   trace_dists/ids [q * capacity + j]: the j-th computed distance and its id,
 *       in the order the traversal computed them;
 *   trace_counts[3q .. 3q+2]: popped candidates including the entry,
 *       expanded candidates, computed distances (= hops, hops, visited).
 * Entries past a capacity are counted but not written; array slots past a
 * query's counts are unspecified.  memory/stream as for falcon_search.
 */
int falcon_search_trace(falcon_index *ix, const float *queries, int64_t nq, int64_t query_stride,
                        const int32_t *entry_points, const falcon_search_params *params, int32_t *out_ids,
                        float *out_dists, int32_t out_stride, int32_t *out_hops, int32_t *out_visited,
                        float *trace_cand_dists, int32_t *trace_cand_counts, int32_t cand_capacity,
                        float *trace_dists, int32_t *trace_ids, int32_t capacity, int32_t *trace_counts,
                        int32_t memory, void *stream);

/*
 * Search without allocating: for callers that cannot allocate device memory
 * on their query path -- serving threads with a fixed, pre-reserved
 * device-memory budget, hosts embedding this library inside a runtime that
 * owns every device allocation, and latency-critical loops that cannot take
 * the implicit synchronisation of cudaMalloc/cudaFree.  It has no counterpart
 * in the reference (whose host migrates buffers before each kernel call).
 * Same results as falcon_search with FALCON_MEM_DEVICE; every data pointer is
 * a device pointer on the index's device and `params` are host structs, each
 * with ef >= k.  Scratch lives in one static 4 MiB device array per GPU (held
 * until the process exits); a call needing more (256 B + 48 B per params
 * struct + 8 B x nq x ef_max for a reduced-precision search with rerank
 * + 4 B x nq for upper-layer entries) fails with FALCON_ERR_ARG.  The first call on a device looks the array up with
 * cudaGetSymbolAddress and should come before any stream capture.  All calls
 * share the array: calls whose kernels overlap on the GPU race and must be
 * serialised by the caller.  Nothing is allocated by this call.
 */
int falcon_search_noalloc(falcon_index *ix, const float *queries, int64_t nq, int64_t query_stride,
                          const int32_t *entry_points, const falcon_search_params *params,
                          int32_t per_query_params, int32_t *out_ids, float *out_dists, int32_t out_stride,
                          int32_t *out_hops, int32_t *out_visited, void *stream);

/*
 * The reference kernel's own argument list (vadd.cpp:11-95, one channel),
 * on host buffers in the reference layout, for hosts that bind `vadd`
 * directly: query_vectors nq x pad16(dim) floats, db_vectors and links_base
 * in the FPGA file layout, out_id/out_dist nq x ef, mem_debug nq x 2
 * (hops, visited).  query_batch_size and max_bloom_out_burst_size only shape
 * the FPGA pipeline and do not change results; they are validated and
 * otherwise ignored.
 */
int falcon_vadd(int32_t query_num, int32_t query_batch_size, int32_t ef, int32_t candidate_queue_runtime_size,
                int32_t max_cand_batch_size, int32_t max_async_stage_num, int32_t runtime_n_bucket_addr_bits,
                uint32_t hash_seed, int32_t max_bloom_out_burst_size, int32_t max_link_num_base, int32_t dim,
                int64_t num_db_vec, const int32_t *entry_point_ids, const float *query_vectors,
                const void *db_vectors, const void *links_base, int32_t *out_id, float *out_dist,
                int32_t *mem_debug, int32_t device);

/*
 * Graph construction: neighbour selection for one set of nodes, the step the
 * reference's offline builders run per node -- hnswlib's
 * getNeighborsByHeuristic2 (networked_FPGA/CPU_programs_oldest/hnswlib/
 * hnswalg.h:328-369) and NSG's occlusion prune behind
 * vector_search_baselines/scripts_nsg (the NSG tool itself is not vendored).
 * For every node in `nodes` (or 0..num_nodes-1 when NULL), in that order:
 * its num_candidates ids at candidates[node * cand_stride ..] (any order;
 * -1, out-of-range ids, the node itself and repeats are skipped) are sorted by
 * (FP32 squared distance to the node, id), then scanned nearest first; a
 * candidate c is kept unless an already kept neighbour i has
 * alpha * d(i, c) < d(c, node) (alpha = 1 is hnswlib's and NSG's rule),
 * until max_degree are kept.  out_neighbors[node * out_stride ..] receives
 * the kept ids nearest first, then -1; out_counts[node] (may be NULL) their
 * number.  Distances sum the dimensions in ascending order with every product
 * and sum rounded separately.  All pointers are device pointers on `device`;
 * vectors are FP32 rows of vector_stride floats.  Limits: num_candidates
 * <= 256, max_degree <= 128, alpha in [1, 4], and num_candidates x
 * (round4(dim) + 4) x 4 bytes within shared memory (227 KB).  Enqueued on
 * `stream` (cudaStream_t); returns after the launch.
 */
int falcon_graph_prune(const float *vectors, int64_t num_vectors, int32_t dim, int64_t vector_stride,
                       const int32_t *candidates, int64_t cand_stride, int32_t num_candidates,
                       const int32_t *nodes, int64_t num_nodes, float alpha, int32_t max_degree,
                       int32_t *out_neighbors, int64_t out_stride, int32_t *out_counts, int32_t device,
                       void *stream);

/*
 * Serving: continuous batching of single-query requests against several
 * device-resident indexes.  Extends the reference's networked serving path
 * (networked_FPGA/CPU_programs/README.md:50-72, CPU_client.cpp:455-612: a
 * client streams query batches to the FPGA and collects per-query results)
 * with on-device admission.  A persistent kernel, launched from a captured
 * CUDA graph, pulls requests from a device ring while the host keeps
 * appending, so requests that arrive while others run start as soon as a warp
 * is free; each request has its own index, precision, k, ef, mc, mg.  The ring
 * is sized from free device memory (memory_fraction); falcon_server_submit
 * admits requests in order while ring entries are free and the requests in
 * flight stay within memory_fraction of the free device memory (read every
 * few milliseconds by the server's monitor thread) plus the server's own, and
 * returns how many it admitted (the caller keeps the rest and retries after
 * collecting results).  Requests of different classes (traversal precision x
 * vector width) run in concurrent persistent kernels that share the SMs.
 * Results are collected with falcon_server_poll / falcon_server_wait.
 * Only inter-query mode is served.
 */
typedef struct falcon_server falcon_server;

typedef struct falcon_server_config {
    int32_t device;
    int32_t ring_capacity;          /* most requests admitted and not yet collected */
    int32_t max_k;                  /* largest k of any request */
    int32_t ef_max;                 /* largest ef (1..1024) */
    int32_t cand_queue_max;         /* largest cand_queue_size (1..256) */
    int32_t bloom_bits_max;         /* largest bloom_bits (10..24) */
    int32_t mc_max, mg_max;
    int32_t dim_max;                /* largest dimension of a registered index */
    int64_t idle_exit_us;           /* the kernel leaves after this long without work */
    double memory_fraction;         /* share of free device memory for per-request state */
} falcon_server_config;

typedef struct falcon_server_info {
    int64_t ring_entries, in_flight, submitted, kernel_launches, warps, device_bytes;
    int64_t concurrent_classes_max; /* most request classes whose kernels ran at the same time */
} falcon_server_info;

void falcon_server_default_config(falcon_server_config *c);
int falcon_server_create(const falcon_server_config *c, falcon_server **out);
/* Register a resident index (same device); *index_id names it in requests. */
int falcon_server_add_index(falcon_server *sv, falcon_index *ix, int32_t *index_id);
/* Submit n requests (host queries, row stride query_stride floats; one params
   struct or n of them).  Returns the number admitted (>= 0; the first ones in
   order) and their ids in request_ids, or a negative error. */
int falcon_server_submit(falcon_server *sv, int32_t n, const int32_t *index_ids, const float *queries,
                         int64_t query_stride, const falcon_search_params *params, int32_t per_request_params,
                         int64_t *request_ids);
/* 1 and the k results if done (the request is then collected), 0 if pending. */
int falcon_server_poll(falcon_server *sv, int64_t request_id, int32_t *out_ids, float *out_dists, int32_t *hops,
                       int32_t *visited);
/* Poll until done or timeout_us; FALCON_OK when done. */
int falcon_server_wait(falcon_server *sv, int64_t request_id, int64_t timeout_us, int32_t *out_ids,
                       float *out_dists, int32_t *hops, int32_t *visited);
/* Load driver: replay an arrival schedule (microsecond offsets from the call,
   ascending) from the calling thread.  Each request is submitted when it has
   arrived and a ring entry is free (with an index that has upper layers in
   the server, arrivals are gathered for up to 200 us or 512 requests per
   submit, since each submit launches one descent), completions are detected
   by polling, and latency_us[i] = completion - arrival (queueing included).  Results go to
   out_ids / out_dists (n x out_stride, may be NULL), hops, visited. */
int falcon_server_replay(falcon_server *sv, int32_t n, const int32_t *index_ids, const float *queries,
                         int64_t query_stride, const falcon_search_params *params, int32_t per_request_params,
                         const double *arrival_us, double *latency_us, int32_t *out_ids, int32_t out_stride,
                         float *out_dists, int32_t *hops, int32_t *visited, double *elapsed_us);
int falcon_server_info_get(falcon_server *sv, falcon_server_info *info);
int falcon_server_free(falcon_server *sv);

/* Thread-local description of the last error on this thread. */
const char *falcon_last_error(void);

/* Library build information (architecture, version). */
const char *falcon_build_info(void);

#ifdef __cplusplus
}
#endif
#endif /* FALCON_H */
