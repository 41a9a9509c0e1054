// Graph construction on the GPU: the neighbour-selection step of the graph
// builders the reference uses offline (hnswlib's getNeighborsByHeuristic2,
// networked_FPGA/CPU_programs_oldest/hnswlib/hnswalg.h:328-369, and the MRNG
// occlusion rule of NSG, which vector_search_baselines/scripts_nsg drives
// through the un-vendored NSG tool).
//
// One thread block per node.  The node's candidate ids (any order, with -1,
// the node itself and repeats allowed) are gathered into shared memory with
// asynchronous 16-byte (or 4-byte) copies, their distances to the node are
// formed, the candidates are sorted by (distance, id) and scanned in that
// order: a candidate is kept unless some already kept neighbour i has
// alpha * d(i, c) < d(c, node) (hnswlib's rule is alpha = 1), until
// max_degree are kept.  Distances are FP32 sums over the dimensions in
// ascending order (no FMA contraction), so results are deterministic and equal
// to a sequential FP32 restatement.  Nodes are taken in the caller's order:
// passing them grouped by cluster keeps the candidate vectors of the blocks in
// flight resident in L2.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../include/falcon.h"
#include "falcon_internal.h"

namespace falcon {
int set_error_code(int code, const char *msg);
}

using namespace falcon;

namespace {

constexpr int kPruneThreads = 128;
constexpr int kMaxPruneCand = 256;
constexpr int kMaxPruneDegree = 128;
constexpr size_t kMaxPruneSmem = 227 * 1024;

struct PruneArgs {
    const float *vecs;
    int64_t vstride;        // floats between rows
    int64_t n;
    int dim;
    int dpad4;              // dim rounded up to 4
    int rowp;               // shared-memory row stride in floats (dpad4 + 4)
    bool vec16;             // 16-byte copies are aligned
    const int32_t *cand;
    int64_t cstride;
    int K, Kp;              // candidates per node, next power of two
    const int32_t *nodes;   // processing order (null: 0 .. nn-1)
    int64_t nn;
    float alpha;
    int R;
    int32_t *out;
    int64_t ostride;
    int32_t *out_count;
};

__host__ __device__ inline size_t prune_smem_bytes(int K, int Kp, int rowp, int R)
{
    size_t b = sizeof(float) * (size_t)rowp * (K + 1);   // candidate rows, then the node's row
    b = (b + 7) & ~(size_t)7;
    b += sizeof(uint64_t) * Kp;                           // sort keys (distance bits, id)
    b += sizeof(int) * Kp;                                // key payload: candidate slot
    b += sizeof(int) * K;                                 // candidate ids
    b += sizeof(int) * R;                                 // kept slots
    return b;
}

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// Squared L2 distance of two shared-memory rows, dimensions in ascending
// order, every product and sum rounded on its own.
__device__ __forceinline__ float row_dist(const float *a, const float *b, int dpad4)
{
    float s = 0.0f;
    for (int j = 0; j < dpad4; j += 4) {
        const float4 x = *reinterpret_cast<const float4 *>(a + j);
        const float4 y = *reinterpret_cast<const float4 *>(b + j);
        float d = __fsub_rn(x.x, y.x);
        s = __fadd_rn(s, __fmul_rn(d, d));
        d = __fsub_rn(x.y, y.y);
        s = __fadd_rn(s, __fmul_rn(d, d));
        d = __fsub_rn(x.z, y.z);
        s = __fadd_rn(s, __fmul_rn(d, d));
        d = __fsub_rn(x.w, y.w);
        s = __fadd_rn(s, __fmul_rn(d, d));
    }
    return s;
}

__global__ void __launch_bounds__(kPruneThreads) prune_kernel(const PruneArgs A)
{
    extern __shared__ uint4 smem_u4[];
    unsigned char *base = reinterpret_cast<unsigned char *>(smem_u4);
    float *cv = reinterpret_cast<float *>(base);
    float *qv = cv + (size_t)A.rowp * A.K;
    size_t off = (sizeof(float) * (size_t)A.rowp * (A.K + 1) + 7) & ~(size_t)7;
    uint64_t *key = reinterpret_cast<uint64_t *>(base + off);
    off += sizeof(uint64_t) * A.Kp;
    int *pay = reinterpret_cast<int *>(base + off);
    off += sizeof(int) * A.Kp;
    int *cid = reinterpret_cast<int *>(base + off);
    off += sizeof(int) * A.K;
    int *kept = reinterpret_cast<int *>(base + off);
    const int tid = threadIdx.x;
    const int nseg4 = A.dpad4 / 4;

    for (int64_t t = blockIdx.x; t < A.nn; t += gridDim.x) {
        const int64_t node = A.nodes ? (int64_t)A.nodes[t] : t;
        // 1. candidate ids; the node's own row is the extra row
        for (int k = tid; k < A.K; k += kPruneThreads) {
            const int c = A.cand[node * A.cstride + k];
            cid[k] = (c >= 0 && (int64_t)c < A.n && (int64_t)c != node) ? c : -1;
        }
        __syncthreads();
        // 2. gather the rows (the node's row and every valid candidate's)
        if (A.vec16) {
            const int total = (A.K + 1) * nseg4;
            for (int e = tid; e < total; e += kPruneThreads) {
                const int k = e / nseg4, s = e - k * nseg4;
                const int64_t id = (k == A.K) ? node : (int64_t)cid[k];
                float *dst = cv + (size_t)k * A.rowp + 4 * s;
                if (id >= 0) cp_async16(dst, A.vecs + id * A.vstride + 4 * s);
            }
        } else {
            const int total = (A.K + 1) * A.dim;
            for (int e = tid; e < total; e += kPruneThreads) {
                const int k = e / A.dim, j = e - k * A.dim;
                const int64_t id = (k == A.K) ? node : (int64_t)cid[k];
                if (id >= 0) cp_async4(cv + (size_t)k * A.rowp + j, A.vecs + id * A.vstride + j);
            }
            // padding columns of every row read as zeros
            for (int e = tid; e < (A.K + 1) * (A.dpad4 - A.dim); e += kPruneThreads) {
                const int pw = A.dpad4 - A.dim;
                const int k = e / pw, j = A.dim + (e - k * pw);
                cv[(size_t)k * A.rowp + j] = 0.0f;
            }
        }
        cp_async_wait_all();
        __syncthreads();
        // 3. distance to the node; key = (distance bits, id): distances are
        //    >= +0, so the bits order like the floats, and repeats of one id
        //    end up next to each other
        for (int k = tid; k < A.Kp; k += kPruneThreads) {
            uint64_t kk = ~0ull;
            if (k < A.K && cid[k] >= 0) {
                const float d = row_dist(cv + (size_t)k * A.rowp, qv, A.dpad4);
                kk = ((uint64_t)__float_as_uint(d) << 32) | (uint32_t)cid[k];
            }
            key[k] = kk;
            pay[k] = k;
        }
        __syncthreads();
        // 4. ascending bitonic sort of the Kp keys
        for (int size = 2; size <= A.Kp; size <<= 1) {
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int p = tid; p < A.Kp / 2; p += kPruneThreads) {
                    const int lo = 2 * p - (p & (stride - 1));
                    const int hi = lo + stride;
                    const bool up = (lo & size) == 0;
                    const uint64_t a = key[lo], b = key[hi];
                    if ((a > b) == up) {
                        key[lo] = b;
                        key[hi] = a;
                        const int pa = pay[lo];
                        pay[lo] = pay[hi];
                        pay[hi] = pa;
                    }
                }
                __syncthreads();
            }
        }
        // 5. occlusion scan in ascending distance order
        int nk = 0;
        for (int s = 0; s < A.K && nk < A.R; s++) {
            const uint64_t ks = key[s];
            if (ks == ~0ull) break;
            if (s > 0 && ks == key[s - 1]) continue;   // the same id again
            const int k = pay[s];
            const float dk = __uint_as_float((uint32_t)(ks >> 32));
            bool rej = false;
            if (tid < nk) {
                const float dik = row_dist(cv + (size_t)kept[tid] * A.rowp, cv + (size_t)k * A.rowp, A.dpad4);
                rej = __fmul_rn(A.alpha, dik) < dk;
            }
            // slot nk is read by no thread before the barrier below
            if (tid == 0) kept[nk] = k;
            if (!__syncthreads_or(rej)) nk++;
        }
        // 6. the kept ids, nearest first, then -1
        int32_t *orow = A.out + node * A.ostride;
        for (int r = tid; r < A.R; r += kPruneThreads) orow[r] = (r < nk) ? cid[kept[r]] : -1;
        if (tid == 0 && A.out_count) A.out_count[node] = nk;
        __syncthreads();
    }
}

}  // namespace

extern "C" int falcon_graph_prune(const float *vectors, int64_t num_vectors, int32_t dim, int64_t vector_stride,
                                  const int32_t *candidates, int64_t cand_stride, int32_t num_candidates,
                                  const int32_t *nodes, int64_t num_nodes, float alpha, int32_t max_degree,
                                  int32_t *out_neighbors, int64_t out_stride, int32_t *out_counts, int32_t device,
                                  void *stream)
{
    if (!vectors || !candidates || !out_neighbors || num_vectors <= 0 || num_nodes < 0)
        return set_error_code(FALCON_ERR_ARG, "falcon_graph_prune: null pointer or empty vector set");
    if (dim < 1 || vector_stride < dim)
        return set_error_code(FALCON_ERR_ARG, "falcon_graph_prune: dim < 1 or vector_stride < dim");
    if (num_candidates < 1 || num_candidates > kMaxPruneCand || cand_stride < num_candidates)
        return set_error_code(FALCON_ERR_ARG, "falcon_graph_prune: num_candidates must be 1..256 and <= cand_stride");
    if (max_degree < 1 || max_degree > kMaxPruneDegree || out_stride < max_degree)
        return set_error_code(FALCON_ERR_ARG, "falcon_graph_prune: max_degree must be 1..128 and <= out_stride");
    if (!(alpha >= 1.0f) || alpha > 4.0f)
        return set_error_code(FALCON_ERR_ARG, "falcon_graph_prune: alpha must be in [1, 4]");
    if (num_nodes == 0) return FALCON_OK;
    PruneArgs a;
    memset(&a, 0, sizeof(a));
    a.vecs = vectors;
    a.vstride = vector_stride;
    a.n = num_vectors;
    a.dim = dim;
    a.dpad4 = (dim + 3) & ~3;
    a.rowp = a.dpad4 + 4;
    a.vec16 = (dim % 4 == 0) && (vector_stride % 4 == 0) && ((reinterpret_cast<uintptr_t>(vectors) & 15) == 0);
    a.cand = candidates;
    a.cstride = cand_stride;
    a.K = num_candidates;
    a.Kp = 2;
    while (a.Kp < a.K) a.Kp <<= 1;
    a.nodes = nodes;
    a.nn = num_nodes;
    a.alpha = alpha;
    a.R = max_degree;
    a.out = out_neighbors;
    a.ostride = out_stride;
    a.out_count = out_counts;
    const size_t smem = prune_smem_bytes(a.K, a.Kp, a.rowp, a.R);
    if (smem > kMaxPruneSmem)
        return set_error_code(FALCON_ERR_UNSUPPORTED,
                              "falcon_graph_prune: num_candidates x (dim + 8) x 4 bytes exceed shared memory");
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (cudaSetDevice(device) != cudaSuccess)
        return set_error_code(FALCON_ERR_CUDA, "falcon_graph_prune: cannot select the device");
    int rc = FALCON_OK;
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(prune_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, prune_kernel, kPruneThreads, smem);
    if (e == cudaSuccess && per_sm < 1) e = cudaErrorInvalidConfiguration;
    if (e == cudaSuccess) {
        int64_t blocks = (int64_t)sms * per_sm;
        if (blocks > num_nodes) blocks = num_nodes;
        prune_kernel<<<(unsigned)blocks, kPruneThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(a);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) rc = set_error_code(FALCON_ERR_CUDA, cudaGetErrorString(e));
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}
