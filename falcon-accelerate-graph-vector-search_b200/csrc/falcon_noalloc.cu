// falcon_search_noalloc: the batched search for callers that must not
// allocate device memory while they run.
//
// falcon_search obtains its per-call scratch (the work counter the persistent
// kernel pulls queries from, the status word, the device copy of the search
// parameters and, for a reduced-precision search with rerank, the list of
// traversal candidates) from cudaMallocAsync and returns it with
// cudaFreeAsync.  Some callers cannot do that: serving threads with a fixed,
// pre-reserved device-memory budget, hosts embedding the library inside
// another runtime that owns all device allocations, and real-time loops that
// cannot afford an allocator call (or the implicit device synchronisation of
// cudaMalloc/cudaFree) on the query path.  For them this entry point takes
// every buffer from the caller and keeps its scratch in one file-scope device
// array, g_noalloc_scratch, of kNoAllocScratchBytes (4 MiB), which every GPU
// that loads the library holds until the process exits.
//
// Rules of use:
//  - queries, entry points and all outputs are device pointers on the index's
//    device; the parameters are host structs, copied unchanged into the
//    scratch array, so every struct must have ef >= k.
//  - The scratch needed by one call is 256 bytes of header, plus 48 bytes per
//    parameter struct, plus 8 * nq * ef_max bytes when a reduced-precision
//    search asks for the FP32 rerank, plus 4 * nq bytes for the upper-layer
//    descent's entries when the index has HNSW upper layers and no entry
//    points are given; a call needing more than 4 MiB is rejected with
//    FALCON_ERR_ARG before any device work.
//  - The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make that
//    first call before any stream capture.
//  - All calls share the one array and it keeps the previous call's
//    contents; the header is cleared on the caller's stream at the start of
//    each call.  Calls whose kernels overlap on the GPU (different streams,
//    or different host threads without ordering) race on the array and must
//    be serialised by the caller.
//  - Nothing here calls cudaMalloc, cudaMallocAsync, cudaFree, cudaFreeAsync
//    or any other allocating routine, and the successful path makes no host
//    heap allocation either.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/falcon.h"
#include "falcon_internal.h"

using namespace falcon;

namespace {

constexpr size_t kNoAllocScratchBytes = 4u << 20;   // 4 MiB per device
constexpr size_t kHeaderBytes = 256;                 // work counter (8 B) + status (4 B), padded
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (looked up once per device,
// with that device current).  Returns nullptr and sets *err on failure.
void *scratch_address(int device, cudaError_t *err)
{
    *err = cudaSuccess;
    if (device < 0 || device >= kMaxDevices) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            *err = e;
            return nullptr;
        }
        g_scratch_addr[device] = p;
    }
    return g_scratch_addr[device];
}

}  // namespace

// Defined in falcon_capi.cu: validation and the launch shared with falcon_search.
namespace falcon {
int prepare_search(const falcon_index *ix, int64_t nq, int64_t query_stride, const falcon_search_params *params,
                   int32_t per_query_params, int32_t out_stride, SearchPlan *plan);
int run_search_plan(const falcon_index *ix, const SearchPlan &plan, int64_t nq, const float *queries,
                    int64_t query_stride, const int32_t *entry_points, QParams *d_params, int32_t *d_scratch,
                    int32_t *d_cand_ids, float *d_cand_d, int32_t *out_ids, float *out_dists, int32_t out_stride,
                    int32_t *out_hops, int32_t *out_visited, int32_t *d_entry_scratch, cudaStream_t s);
int set_error_code(int code, const char *msg);
int index_device(const falcon_index *ix);
bool index_has_upper(const falcon_index *ix);
}  // namespace falcon

extern "C" int falcon_search_noalloc(falcon_index *ix, const float *queries, int64_t nq, int64_t query_stride,
                                     const int32_t *entry_points, const falcon_search_params *params,
                                     int32_t per_query_params, int32_t *out_ids, float *out_dists,
                                     int32_t out_stride, int32_t *out_hops, int32_t *out_visited, void *stream_v)
{
    if (!ix || !params || !out_ids || !out_dists || (nq > 0 && !queries))
        return set_error_code(FALCON_ERR_ARG, "falcon_search_noalloc: null argument");
    if (nq < 0) return set_error_code(FALCON_ERR_ARG, "falcon_search_noalloc: nq < 0");
    if (nq == 0) return FALCON_OK;
    SearchPlan plan;
    int rc = prepare_search(ix, nq, query_stride, params, per_query_params, out_stride, &plan);
    if (rc != FALCON_OK) return rc;
    const size_t param_bytes = sizeof(QParams) * (size_t)plan.np;
    const size_t param_off = kHeaderBytes;
    const size_t cand_off = (param_off + param_bytes + 255) & ~(size_t)255;
    const size_t cand_bytes = plan.any_rerank ? (size_t)nq * plan.ef_max * (sizeof(int32_t) + sizeof(float)) : 0;
    // per-query entries of the upper-layer descent, when the index has upper layers and none are given
    const size_t entry_off = (cand_off + cand_bytes + 255) & ~(size_t)255;
    const size_t entry_bytes = (!entry_points && index_has_upper(ix)) ? (size_t)nq * sizeof(int32_t) : 0;
    if (entry_off + entry_bytes > kNoAllocScratchBytes)
        return set_error_code(FALCON_ERR_ARG,
                              "falcon_search_noalloc: this call needs more than the 4 MiB static scratch "
                              "(48 B per parameter struct + 8 B per query per ef with rerank + 4 B per query "
                              "for upper-layer entries); split the batch or use falcon_search");
    const int device = index_device(ix);
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (cudaSetDevice(device) != cudaSuccess)
        return set_error_code(FALCON_ERR_CUDA, "falcon_search_noalloc: cannot select the index's device");
    cudaError_t err;
    unsigned char *base = static_cast<unsigned char *>(scratch_address(device, &err));
    if (!base) {
        if (prev >= 0) cudaSetDevice(prev);
        return set_error_code(FALCON_ERR_CUDA, "falcon_search_noalloc: cudaGetSymbolAddress failed");
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream_v);
    int32_t *d_header = reinterpret_cast<int32_t *>(base);
    QParams *d_params = reinterpret_cast<QParams *>(base + param_off);
    int32_t *d_cand_ids = nullptr;
    float *d_cand_d = nullptr;
    if (plan.any_rerank) {
        d_cand_ids = reinterpret_cast<int32_t *>(base + cand_off);
        d_cand_d = reinterpret_cast<float *>(base + cand_off + (size_t)nq * plan.ef_max * sizeof(int32_t));
    }
    int32_t *d_entry = entry_bytes ? reinterpret_cast<int32_t *>(base + entry_off) : nullptr;
    rc = FALCON_OK;
    if (cudaMemsetAsync(d_header, 0, 16, s) != cudaSuccess ||
        cudaMemcpyAsync(d_params, params, param_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        rc = set_error_code(FALCON_ERR_CUDA, "falcon_search_noalloc: scratch initialisation failed");
    if (rc == FALCON_OK)
        rc = run_search_plan(ix, plan, nq, queries, query_stride, entry_points, d_params, d_header, d_cand_ids,
                             d_cand_d, out_ids, out_dists, out_stride, out_hops, out_visited, d_entry, s);
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}
