// C ABI of libfalcon_b200.so: index management, search entry points and the
// reference-kernel-compatible falcon_vadd.  Host code; all device work is
// issued on the caller's stream.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/falcon.h"
#include "falcon_internal.h"

using namespace falcon;

struct falcon_index {
    std::atomic<int> server_refs{0};   // servers holding device pointers into this index
    int device = 0;
    int num_sms = 0;
    int64_t n = 0;
    int dim = 0, dpad = 0, max_degree = 0, entry = 0, storage = 0;
    int64_t link_stride = 0;
    int ids_offset = 0;
    float *d_f32 = nullptr;        // n x dpad
    uint16_t *d_bf16 = nullptr;    // n x dpad
    uint8_t *d_fp8 = nullptr;      // n x dpad
    float *d_scales = nullptr;     // n
    int32_t *d_links = nullptr;    // n x link_stride
    int32_t *d_labels = nullptr;   // n or null
    int64_t device_bytes = 0;
    // HNSW upper layers (falcon_index_set_upper_layers); max_level 0 = none
    int32_t *d_upper_rows = nullptr;
    int64_t *d_upper_start = nullptr;
    int32_t *d_upper_levels = nullptr;
    int64_t upper_stride = 0;
    int upper_max_level = 0, upper_max_degree = 0, upper_entry = 0;
};

namespace {

thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

#define FALCON_CUDA(call)                                                                               \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) {                                                                        \
            rc = set_error(e_ == cudaErrorMemoryAllocation ? FALCON_ERR_OOM : FALCON_ERR_CUDA, "%s: %s", \
                           #call, cudaGetErrorString(e_));                                              \
            goto done;                                                                                  \
        }                                                                                               \
    } while (0)

int pad16(int d) { return (d + 15) / 16 * 16; }

void free_upper(falcon_index *ix)
{
    cudaFree(ix->d_upper_rows);
    cudaFree(ix->d_upper_start);
    cudaFree(ix->d_upper_levels);
    ix->d_upper_rows = nullptr; ix->d_upper_start = nullptr; ix->d_upper_levels = nullptr;
    ix->upper_max_level = 0;
}

// Device view of the upper layers and the FP32 vectors for the descent.
DescendLaunch descend_launch(const falcon_index *ix)
{
    DescendLaunch a;
    memset(&a, 0, sizeof(a));
    a.g.vecs = reinterpret_cast<const unsigned char *>(ix->d_f32);
    a.g.vstride_bytes = (int64_t)ix->dpad * 4;
    a.g.vecs32 = a.g.vecs;
    a.g.vstride32_bytes = a.g.vstride_bytes;
    a.g.dim = ix->dim;
    a.g.dpad = ix->dpad;
    a.g.n = ix->n;
    a.u.rows = ix->d_upper_rows;
    a.u.stride = ix->upper_stride;
    a.u.row_start = ix->d_upper_start;
    a.u.levels = ix->d_upper_levels;
    a.u.max_level = ix->upper_max_level;
    a.u.max_degree = ix->upper_max_degree;
    a.u.entry = ix->upper_entry;
    return a;
}

void free_index_buffers(falcon_index *ix)
{
    cudaFree(ix->d_f32);
    cudaFree(ix->d_bf16);
    cudaFree(ix->d_fp8);
    cudaFree(ix->d_scales);
    cudaFree(ix->d_links);
    cudaFree(ix->d_labels);
    ix->d_f32 = nullptr; ix->d_bf16 = nullptr; ix->d_fp8 = nullptr;
    ix->d_scales = nullptr; ix->d_links = nullptr; ix->d_labels = nullptr;
    free_upper(ix);
}

// Host-side validation of the adjacency rows: count in [0, max_degree], ids in [0, n).
int validate_graph(const falcon_index_desc *d)
{
    for (int64_t r = 0; r < d->num_vectors; r++) {
        const int32_t *row = d->links + r * d->link_stride;
        const int32_t c = row[0];
        if (c < 0 || c > d->max_degree)
            return set_error(FALCON_ERR_GRAPH, "row %lld: neighbour count %d outside [0, %d]", (long long)r, c,
                             d->max_degree);
        for (int j = 0; j < c; j++) {
            const int32_t v = row[d->ids_offset + j];
            if (v < 0 || v >= d->num_vectors)
                return set_error(FALCON_ERR_GRAPH, "row %lld: neighbour id %d outside [0, %lld)", (long long)r, v,
                                 (long long)d->num_vectors);
        }
    }
    return FALCON_OK;
}

int check_params(const falcon_search_params &p, const falcon_index *ix, int64_t qi)
{
    int ef = p.ef < p.k ? p.k : p.ef;
    if (p.k < 1 || ef < 1 || ef > kMaxEf)
        return set_error(FALCON_ERR_ARG, "query %lld: k=%d ef=%d (need 1 <= k, ef <= %d)", (long long)qi, p.k, p.ef, kMaxEf);
    if (p.mc < 1 || p.mc > kMaxMc) return set_error(FALCON_ERR_ARG, "query %lld: mc=%d outside [1,%d]", (long long)qi, p.mc, kMaxMc);
    if (p.mg < 1 || p.mg > kMaxMg) return set_error(FALCON_ERR_ARG, "query %lld: mg=%d outside [1,%d]", (long long)qi, p.mg, kMaxMg);
    if (p.cand_queue_size < 1 || p.cand_queue_size > kMaxCandQueue)
        return set_error(FALCON_ERR_ARG, "query %lld: cand_queue_size=%d outside [1,%d]", (long long)qi, p.cand_queue_size, kMaxCandQueue);
    if (p.bloom_bits < kMinBloomBits || p.bloom_bits > kMaxBloomBits)
        return set_error(FALCON_ERR_ARG, "query %lld: bloom_bits=%d outside [%d,%d]", (long long)qi, p.bloom_bits, kMinBloomBits, kMaxBloomBits);
    if (p.max_hops < 0) return set_error(FALCON_ERR_ARG, "query %lld: max_hops < 0", (long long)qi);
    if (p.mode != FALCON_MODE_INTER && p.mode != FALCON_MODE_INTRA)
        return set_error(FALCON_ERR_ARG, "query %lld: unknown mode %d", (long long)qi, p.mode);
    if (p.mode == FALCON_MODE_INTRA &&
        (p.channels < 1 || p.channels > kMaxChannels || (p.channels & (p.channels - 1))))
        return set_error(FALCON_ERR_ARG, "query %lld: channels=%d must be a power of two <= %d", (long long)qi, p.channels, kMaxChannels);
    if (p.precision == FALCON_PREC_BF16 && !(ix->storage & FALCON_STORE_BF16))
        return set_error(FALCON_ERR_ARG, "BF16 traversal needs FALCON_STORE_BF16 in the index");
    if (p.precision == FALCON_PREC_FP8 && !(ix->storage & FALCON_STORE_FP8))
        return set_error(FALCON_ERR_ARG, "FP8 traversal needs FALCON_STORE_FP8 in the index");
    if (p.precision < 0 || p.precision > 2) return set_error(FALCON_ERR_ARG, "unknown precision %d", p.precision);
    return FALCON_OK;
}

QParams to_qparams(const falcon_search_params &p)
{
    QParams q;
    q.k = p.k;
    q.ef = p.ef < p.k ? p.k : p.ef;
    q.mc = p.mc;
    q.mg = p.mg;
    q.cq = p.cand_queue_size;
    q.bloom_bits = p.bloom_bits;
    q.seed = p.hash_seed;
    q.mode = p.mode;
    q.channels = p.channels;
    q.precision = p.precision;
    q.rerank = p.rerank;
    q.max_hops = p.max_hops;
    return q;
}

}  // namespace

extern "C" {

const char *falcon_last_error(void) { return g_last_error.c_str(); }

const char *falcon_build_info(void) { return "libfalcon_b200 sm_100a (inter-query + intra-query DST traversal)"; }

void falcon_default_params(falcon_search_params *p)
{
    if (!p) return;
    p->k = 10;
    p->ef = 64;
    p->mc = 1;
    p->mg = 1;
    p->cand_queue_size = 32;
    p->bloom_bits = 16;
    p->hash_seed = 1;
    p->mode = FALCON_MODE_INTER;
    p->channels = 4;
    p->precision = FALCON_PREC_F32;
    p->rerank = 0;
    p->max_hops = 0;
}

int falcon_index_create(const falcon_index_desc *d, falcon_index **out)
{
    if (!d || !out) return set_error(FALCON_ERR_ARG, "null argument");
    *out = nullptr;
    if (d->num_vectors < 1 || d->dim < 1 || pad16(d->dim) > kMaxDimPadded || d->max_degree < 1 ||
        d->max_degree > kMaxDegree || !d->vectors || !d->links || d->vector_stride < d->dim ||
        d->link_stride < d->ids_offset + d->max_degree || d->ids_offset < 1)
        return set_error(FALCON_ERR_ARG, "invalid index description (n=%lld dim=%d max_degree=%d)",
                         (long long)d->num_vectors, d->dim, d->max_degree);
    if (d->num_vectors > 0x7fffffffLL) return set_error(FALCON_ERR_ARG, "more than 2^31-1 vectors");
    if (d->entry_point < 0 || d->entry_point >= d->num_vectors)
        return set_error(FALCON_ERR_GRAPH, "entry point %d outside [0, %lld)", d->entry_point, (long long)d->num_vectors);
    int rc = validate_graph(d);
    if (rc != FALCON_OK) return rc;

    DeviceGuard guard(d->device);
    if (!guard.ok) return set_error(FALCON_ERR_CUDA, "cannot select device %d", d->device);
    falcon_index *ix = new falcon_index;
    ix->device = d->device;
    ix->n = d->num_vectors;
    ix->dim = d->dim;
    ix->dpad = pad16(d->dim);
    ix->max_degree = d->max_degree;
    ix->entry = d->entry_point;
    ix->storage = d->storage | FALCON_STORE_F32;
    ix->link_stride = d->link_stride;
    ix->ids_offset = d->ids_offset;
    {
        rc = FALCON_OK;
        const size_t nvec = (size_t)ix->n;
        const size_t f32_bytes = nvec * ix->dpad * sizeof(float);
        cudaDeviceProp prop;
        FALCON_CUDA(cudaGetDeviceProperties(&prop, ix->device));
        ix->num_sms = prop.multiProcessorCount;
        {   // keep freed per-call scratch in the device's default pool instead of
            // returning it to the driver at every synchronisation
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, ix->device) == cudaSuccess) {
                uint64_t keep = ~0ull;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            }
        }
        FALCON_CUDA(cudaMalloc(&ix->d_f32, f32_bytes));
        FALCON_CUDA(cudaMemset(ix->d_f32, 0, f32_bytes));
        FALCON_CUDA(cudaMemcpy2D(ix->d_f32, ix->dpad * sizeof(float), d->vectors, d->vector_stride * sizeof(float),
                                 ix->dim * sizeof(float), nvec, cudaMemcpyHostToDevice));
        ix->device_bytes += f32_bytes;
        const size_t link_bytes = nvec * ix->link_stride * sizeof(int32_t);
        FALCON_CUDA(cudaMalloc(&ix->d_links, link_bytes));
        FALCON_CUDA(cudaMemcpy(ix->d_links, d->links, link_bytes, cudaMemcpyHostToDevice));
        ix->device_bytes += link_bytes;
        if (d->labels) {
            FALCON_CUDA(cudaMalloc(&ix->d_labels, nvec * sizeof(int32_t)));
            FALCON_CUDA(cudaMemcpy(ix->d_labels, d->labels, nvec * sizeof(int32_t), cudaMemcpyHostToDevice));
            ix->device_bytes += nvec * sizeof(int32_t);
        }
        if (ix->storage & FALCON_STORE_BF16) {
            FALCON_CUDA(cudaMalloc(&ix->d_bf16, nvec * ix->dpad * sizeof(uint16_t)));
            FALCON_CUDA(launch_encode_bf16(ix->d_f32, ix->dpad, ix->n, ix->dim, ix->dpad, ix->d_bf16, 0));
            ix->device_bytes += nvec * ix->dpad * sizeof(uint16_t);
        }
        if (ix->storage & FALCON_STORE_FP8) {
            FALCON_CUDA(cudaMalloc(&ix->d_fp8, nvec * ix->dpad));
            FALCON_CUDA(cudaMalloc(&ix->d_scales, nvec * sizeof(float)));
            FALCON_CUDA(launch_encode_fp8(ix->d_f32, ix->dpad, ix->n, ix->dim, ix->dpad, ix->d_fp8, ix->d_scales, 0));
            ix->device_bytes += nvec * ix->dpad + nvec * sizeof(float);
        }
        FALCON_CUDA(cudaDeviceSynchronize());
    }
done:
    if (rc != FALCON_OK) {
        free_index_buffers(ix);
        delete ix;
        return rc;
    }
    *out = ix;
    return FALCON_OK;
}

int falcon_index_free(falcon_index *ix)
{
    if (!ix) return FALCON_OK;
    if (ix->server_refs.load() > 0)
        return set_error(FALCON_ERR_ARG, "the index is registered with a server: free the server first");
    DeviceGuard guard(ix->device);
    free_index_buffers(ix);
    delete ix;
    return FALCON_OK;
}

int falcon_index_info_get(const falcon_index *ix, falcon_index_info *info)
{
    if (!ix || !info) return set_error(FALCON_ERR_ARG, "null argument");
    info->num_vectors = ix->n;
    info->dim = ix->dim;
    info->dim_padded = ix->dpad;
    info->max_degree = ix->max_degree;
    info->entry_point = ix->entry;
    info->storage = ix->storage;
    info->device = ix->device;
    info->device_bytes = ix->device_bytes;
    return FALCON_OK;
}

int falcon_index_copy_storage(const falcon_index *ix, int32_t which, void *dst, int64_t bytes)
{
    if (!ix || !dst) return set_error(FALCON_ERR_ARG, "null argument");
    const int64_t nd = ix->n * (int64_t)ix->dpad;
    DeviceGuard guard(ix->device);
    cudaError_t e = cudaSuccess;
    if (which == FALCON_STORE_F32) {
        if (bytes != nd * 4) return set_error(FALCON_ERR_ARG, "F32 storage is %lld bytes", (long long)(nd * 4));
        e = cudaMemcpy(dst, ix->d_f32, bytes, cudaMemcpyDeviceToHost);
    } else if (which == FALCON_STORE_BF16) {
        if (!ix->d_bf16) return set_error(FALCON_ERR_ARG, "index holds no BF16 storage");
        if (bytes != nd * 2) return set_error(FALCON_ERR_ARG, "BF16 storage is %lld bytes", (long long)(nd * 2));
        e = cudaMemcpy(dst, ix->d_bf16, bytes, cudaMemcpyDeviceToHost);
    } else if (which == FALCON_STORE_FP8) {
        if (!ix->d_fp8) return set_error(FALCON_ERR_ARG, "index holds no FP8 storage");
        if (bytes != nd + ix->n * 4) return set_error(FALCON_ERR_ARG, "FP8 storage is %lld bytes", (long long)(nd + ix->n * 4));
        e = cudaMemcpy(dst, ix->d_fp8, nd, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy((char *)dst + nd, ix->d_scales, ix->n * 4, cudaMemcpyDeviceToHost);
    } else {
        return set_error(FALCON_ERR_ARG, "unknown storage %d", which);
    }
    if (e != cudaSuccess) return set_error(FALCON_ERR_CUDA, "copy storage: %s", cudaGetErrorString(e));
    return FALCON_OK;
}

static bool read_file(const std::string &path, std::vector<char> &buf)
{
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    buf.resize(sz > 0 ? (size_t)sz : 0);
    const bool ok = sz <= 0 || fread(buf.data(), 1, (size_t)sz, f) == (size_t)sz;
    fclose(f);
    return ok;
}

int falcon_index_load_fpga(const char *index_dir, const char *graph_type, int32_t dim, int32_t storage,
                           int32_t device, falcon_index **out)
{
    if (!index_dir || !graph_type || !out || dim < 1) return set_error(FALCON_ERR_ARG, "null argument or dim < 1");
    const std::string dir(index_dir), gt(graph_type);
    if (gt != "HNSW" && gt != "NSG") return set_error(FALCON_ERR_ARG, "graph_type must be HNSW or NSG");
    std::vector<char> meta, links, vecs, labels;
    if (!read_file(dir + "/meta.bin", meta)) return set_error(FALCON_ERR_IO, "cannot read %s/meta.bin", index_dir);
    const int32_t *m = reinterpret_cast<const int32_t *>(meta.data());
    int32_t n, entry, md;
    if (gt == "HNSW") {   // cur_element_count, maxlevel_, enterpoint_node_, maxM_, maxM0_ (hnsw.py:270-275)
        if (meta.size() < 20) return set_error(FALCON_ERR_IO, "meta.bin too short for HNSW");
        n = m[0]; entry = m[2]; md = m[4];
    } else {              // num_nodes, entry point, width (nsg_to_FPGA.py)
        if (meta.size() < 12) return set_error(FALCON_ERR_IO, "meta.bin too short for NSG");
        n = m[0]; entry = m[1]; md = m[2];
    }
    if (n < 1 || md < 1 || md > kMaxDegree) return set_error(FALCON_ERR_IO, "meta.bin: n=%d max_degree=%d", n, md);
    const int64_t lstride = 16LL * (1 + (md + 15) / 16);
    const int64_t vstride = pad16(dim) + 16;
    // The reference writes the rows round robin over nc channel files, node i
    // as row i / nc of channel i % nc (hnsw.py:324-335, nsg_to_FPGA.py:124-135);
    // its hosts read the set their kernel was built for (intra v1.5
    // host.cpp:242-260).  The single-channel set is used when present, else
    // the first complete set of 2, 4, 8 or 16 channels, de-interleaved.
    int nc = 0;
    for (int c : {1, 2, 4, 8, 16}) {
        FILE *f = fopen((dir + "/ground_links_" + std::to_string(c) + "_chan_0.bin").c_str(), "rb");
        if (f) {
            fclose(f);
            nc = c;
            break;
        }
    }
    if (nc == 0) return set_error(FALCON_ERR_IO, "no ground_links_{1,2,4,8,16}_chan_0.bin in %s", index_dir);
    links.resize((size_t)n * lstride * 4);
    vecs.resize((size_t)n * vstride * 4);
    for (int c = 0; c < nc; c++) {
        const int64_t rows = (n - c + nc - 1) / nc;   // nodes c, c + nc, ...
        const std::string suffix = std::to_string(nc) + "_chan_" + std::to_string(c) + ".bin";
        std::vector<char> lc, vc;
        if (!read_file(dir + "/ground_links_" + suffix, lc) || (int64_t)lc.size() != rows * lstride * 4)
            return set_error(FALCON_ERR_IO, "ground_links_%s missing or not %lld bytes", suffix.c_str(),
                             (long long)(rows * lstride * 4));
        if (!read_file(dir + "/ground_vectors_" + suffix, vc) || (int64_t)vc.size() != rows * vstride * 4)
            return set_error(FALCON_ERR_IO, "ground_vectors_%s missing or not %lld bytes for dim %d", suffix.c_str(),
                             (long long)(rows * vstride * 4), dim);
        for (int64_t r = 0; r < rows; r++) {
            const int64_t node = r * nc + c;
            memcpy(links.data() + node * lstride * 4, lc.data() + r * lstride * 4, (size_t)lstride * 4);
            memcpy(vecs.data() + node * vstride * 4, vc.data() + r * vstride * 4, (size_t)vstride * 4);
        }
    }
    const bool have_labels = read_file(dir + "/ground_labels.bin", labels) && (int64_t)labels.size() == (int64_t)n * 4;
    falcon_index_desc d;
    memset(&d, 0, sizeof(d));
    d.num_vectors = n;
    d.dim = dim;
    d.max_degree = md;
    d.vectors = reinterpret_cast<const float *>(vecs.data());
    d.vector_stride = vstride;
    d.links = reinterpret_cast<const int32_t *>(links.data());
    d.link_stride = lstride;
    d.ids_offset = 16;
    d.entry_point = entry;
    d.labels = (gt == "HNSW" && have_labels) ? reinterpret_cast<const int32_t *>(labels.data()) : nullptr;
    d.storage = storage;
    d.device = device;
    return falcon_index_create(&d, out);
}

int falcon_index_set_upper_layers(falcon_index *ix, const falcon_upper_layers_desc *d)
{
    if (!ix || !d || !d->levels || !d->row_start || (d->num_rows > 0 && !d->rows))
        return set_error(FALCON_ERR_ARG, "null argument");
    if (ix->server_refs.load() > 0)
        return set_error(FALCON_ERR_ARG, "the index is registered with a server: set its upper layers before "
                                         "falcon_server_add_index");
    if (d->max_level < 1 || d->max_degree < 1 || d->max_degree > kMaxDegree || d->ids_offset < 1 ||
        d->row_stride < d->ids_offset + d->max_degree || d->num_rows < 0)
        return set_error(FALCON_ERR_ARG, "bad upper-layer shape (max_level=%d, max_degree=%d, ids_offset=%d, "
                         "row_stride=%lld)", d->max_level, d->max_degree, d->ids_offset, (long long)d->row_stride);
    const int64_t n = ix->n;
    if (d->entry_point < 0 || d->entry_point >= n || d->levels[d->entry_point] != d->max_level)
        return set_error(FALCON_ERR_GRAPH, "upper-layer entry point %d is not on level %d", d->entry_point,
                         d->max_level);
    for (int64_t v = 0; v < n; v++) {
        const int lv = d->levels[v];
        if (lv < 0 || lv > d->max_level)
            return set_error(FALCON_ERR_GRAPH, "node %lld: level %d outside [0, %d]", (long long)v, lv, d->max_level);
        if (lv == 0) continue;
        const int64_t r0 = d->row_start[v];
        if (r0 < 0 || r0 + lv > d->num_rows)
            return set_error(FALCON_ERR_GRAPH, "node %lld: rows [%lld, %lld) outside %lld rows", (long long)v,
                             (long long)r0, (long long)(r0 + lv), (long long)d->num_rows);
        for (int l = 1; l <= lv; l++) {
            const int32_t *row = d->rows + (r0 + l - 1) * d->row_stride;
            const int c = row[0];
            if (c < 0 || c > d->max_degree)
                return set_error(FALCON_ERR_GRAPH, "node %lld level %d: count %d outside [0, %d]", (long long)v, l, c,
                                 d->max_degree);
            for (int j = 0; j < c; j++) {
                const int32_t u = row[d->ids_offset + j];
                if (u < 0 || u >= n || d->levels[u] < l)
                    return set_error(FALCON_ERR_GRAPH, "node %lld level %d: neighbour %d is not on that level",
                                     (long long)v, l, u);
            }
        }
    }
    // device layout: rows of 16 * (1 + ceil(max_degree / 16)) int32, count at 0, ids at 16; rows of a node consecutive
    const int64_t stride = 16LL * (1 + (d->max_degree + 15) / 16);
    std::vector<int64_t> start((size_t)n, 0);
    int64_t nrows = 0;
    for (int64_t v = 0; v < n; v++) {
        start[(size_t)v] = nrows;
        nrows += d->levels[v];
    }
    std::vector<int32_t> rows((size_t)(nrows > 0 ? nrows : 1) * stride, 0);
    for (int64_t v = 0; v < n; v++)
        for (int l = 1; l <= d->levels[v]; l++) {
            const int32_t *src = d->rows + (d->row_start[v] + l - 1) * d->row_stride;
            int32_t *dst = rows.data() + (start[(size_t)v] + l - 1) * stride;
            dst[0] = src[0];
            for (int j = 0; j < src[0]; j++) dst[16 + j] = src[d->ids_offset + j];
        }
    DeviceGuard guard(ix->device);
    if (!guard.ok) return set_error(FALCON_ERR_CUDA, "cannot select device %d", ix->device);
    free_upper(ix);
    int rc = FALCON_OK;
    cudaStream_t s = nullptr;
    FALCON_CUDA(cudaMalloc((void **)&ix->d_upper_rows, rows.size() * sizeof(int32_t)));
    FALCON_CUDA(cudaMalloc((void **)&ix->d_upper_start, (size_t)n * sizeof(int64_t)));
    FALCON_CUDA(cudaMalloc((void **)&ix->d_upper_levels, (size_t)n * sizeof(int32_t)));
    FALCON_CUDA(cudaMemcpyAsync(ix->d_upper_rows, rows.data(), rows.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    FALCON_CUDA(cudaMemcpyAsync(ix->d_upper_start, start.data(), (size_t)n * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    FALCON_CUDA(cudaMemcpyAsync(ix->d_upper_levels, d->levels, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    FALCON_CUDA(cudaStreamSynchronize(s));
    ix->upper_stride = stride;
    ix->upper_max_level = d->max_level;
    ix->upper_max_degree = d->max_degree;
    ix->upper_entry = d->entry_point;
done:
    if (rc != FALCON_OK) free_upper(ix);
    return rc;
}

int falcon_descend(falcon_index *ix, const float *queries, int64_t nq, int64_t query_stride,
                   int32_t *out_entry_points, int32_t *out_upper_hops, int32_t memory, void *stream_v)
{
    if (!ix || !out_entry_points || (nq > 0 && !queries)) return set_error(FALCON_ERR_ARG, "null argument");
    if (query_stride < ix->dim) return set_error(FALCON_ERR_ARG, "query_stride %lld < dim %d", (long long)query_stride, ix->dim);
    if (memory != FALCON_MEM_HOST && memory != FALCON_MEM_DEVICE) return set_error(FALCON_ERR_ARG, "bad memory flag");
    if (ix->upper_max_level < 1) return set_error(FALCON_ERR_ARG, "the index has no upper layers");
    if (!ix->d_f32) return set_error(FALCON_ERR_UNSUPPORTED, "the descent needs FP32 storage");
    if (nq < 0) return set_error(FALCON_ERR_ARG, "nq < 0");
    if (nq == 0) return FALCON_OK;
    DeviceGuard guard(ix->device);
    if (!guard.ok) return set_error(FALCON_ERR_CUDA, "cannot select device %d", ix->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream_v);
    const bool host = memory == FALCON_MEM_HOST;
    int rc = FALCON_OK;
    float *d_q = nullptr;
    int32_t *d_e = nullptr, *d_h = nullptr;
    DescendLaunch a = descend_launch(ix);
    if (host) {
        FALCON_CUDA(cudaMallocAsync((void **)&d_q, (size_t)nq * query_stride * sizeof(float), s));
        FALCON_CUDA(cudaMemcpyAsync(d_q, queries, (size_t)nq * query_stride * sizeof(float), cudaMemcpyHostToDevice, s));
        FALCON_CUDA(cudaMallocAsync((void **)&d_e, (size_t)nq * sizeof(int32_t), s));
        if (out_upper_hops) FALCON_CUDA(cudaMallocAsync((void **)&d_h, (size_t)nq * sizeof(int32_t), s));
    }
    a.queries = host ? d_q : queries;
    a.qstride = query_stride;
    a.nq = nq;
    a.out_entry = host ? d_e : out_entry_points;
    a.out_hops = host ? d_h : out_upper_hops;
    FALCON_CUDA(launch_descend(a, ix->num_sms, s));
    if (host) {
        FALCON_CUDA(cudaMemcpyAsync(out_entry_points, d_e, (size_t)nq * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        if (out_upper_hops)
            FALCON_CUDA(cudaMemcpyAsync(out_upper_hops, d_h, (size_t)nq * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    }
done:
    for (void *p : {(void *)d_q, (void *)d_e, (void *)d_h})
        if (p) cudaFreeAsync(p, s);
    if (rc == FALCON_OK && host) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return set_error(FALCON_ERR_CUDA, "descend: %s", cudaGetErrorString(e));
    }
    return rc;
}

// Trace outputs of falcon_search_trace (caller memory, host or device).
struct TraceOut {
    float *cand_d;
    int32_t *cand_n;
    int32_t cand_cap;
    float *d;
    int32_t *ids;
    int32_t cap;
    int32_t *counts;
};

static int search_impl(falcon_index *ix, const float *queries, int64_t nq, int64_t query_stride,
                       const int32_t *entry_points, const falcon_search_params *params, int32_t per_query_params,
                       int32_t *out_ids, float *out_dists, int32_t out_stride, int32_t *out_hops,
                       int32_t *out_visited, int32_t memory, void *stream_v, const TraceOut *tro);

int falcon_search(falcon_index *ix, const float *queries, int64_t nq, int64_t query_stride,
                  const int32_t *entry_points, const falcon_search_params *params, int32_t per_query_params,
                  int32_t *out_ids, float *out_dists, int32_t out_stride, int32_t *out_hops, int32_t *out_visited,
                  int32_t memory, void *stream_v)
{
    return search_impl(ix, queries, nq, query_stride, entry_points, params, per_query_params, out_ids, out_dists,
                       out_stride, out_hops, out_visited, memory, stream_v, nullptr);
}

int falcon_search_trace(falcon_index *ix, const float *queries, int64_t nq, int64_t query_stride,
                        const int32_t *entry_points, const falcon_search_params *params, int32_t *out_ids,
                        float *out_dists, int32_t out_stride, int32_t *out_hops, int32_t *out_visited,
                        float *trace_cand_dists, int32_t *trace_cand_counts, int32_t cand_capacity,
                        float *trace_dists, int32_t *trace_ids, int32_t capacity, int32_t *trace_counts,
                        int32_t memory, void *stream)
{
    if (!params || !trace_counts || cand_capacity < 0 || capacity < 0 ||
        (cand_capacity > 0 && (!trace_cand_dists || !trace_cand_counts)) || (capacity > 0 && (!trace_dists || !trace_ids)))
        return set_error(FALCON_ERR_ARG, "falcon_search_trace: bad trace buffers");
    if (params->mode != FALCON_MODE_INTER || params->precision != FALCON_PREC_F32 || params->rerank)
        return set_error(FALCON_ERR_UNSUPPORTED, "falcon_search_trace: FP32 inter-query searches only");
    TraceOut t = {trace_cand_dists, trace_cand_counts, cand_capacity, trace_dists, trace_ids, capacity, trace_counts};
    return search_impl(ix, queries, nq, query_stride, entry_points, params, 0, out_ids, out_dists, out_stride,
                       out_hops, out_visited, memory, stream, &t);
}

static int search_impl(falcon_index *ix, const float *queries, int64_t nq, int64_t query_stride,
                       const int32_t *entry_points, const falcon_search_params *params, int32_t per_query_params,
                       int32_t *out_ids, float *out_dists, int32_t out_stride, int32_t *out_hops,
                       int32_t *out_visited, int32_t memory, void *stream_v, const TraceOut *tro)
{
    if (!ix || !params || !out_ids || !out_dists) return set_error(FALCON_ERR_ARG, "null argument");
    if (nq < 0 || (nq > 0 && !queries) || query_stride < ix->dim)
        return set_error(FALCON_ERR_ARG, "bad queries (nq=%lld, stride=%lld, dim=%d)", (long long)nq,
                         (long long)query_stride, ix->dim);
    if (memory != FALCON_MEM_HOST && memory != FALCON_MEM_DEVICE) return set_error(FALCON_ERR_ARG, "bad memory flag");
    if (nq == 0) return FALCON_OK;
    const int64_t np = per_query_params ? nq : 1;
    int ef_max = 0, k_max = 0, mc_max = 1, mg_max = 1, bits_max = kMinBloomBits, prec = -1, mode = -1, ch_max = 1;
    int cq_max = 1;
    bool any_rerank = false;
    std::vector<QParams> qp((size_t)np);
    for (int64_t i = 0; i < np; i++) {
        int rc = check_params(params[i], ix, i);
        if (rc != FALCON_OK) return rc;
        qp[i] = to_qparams(params[i]);
        if (prec >= 0 && prec != params[i].precision)
            return set_error(FALCON_ERR_UNSUPPORTED, "one call must use one precision");
        if (mode >= 0 && mode != params[i].mode) return set_error(FALCON_ERR_UNSUPPORTED, "one call must use one mode");
        prec = params[i].precision;
        mode = params[i].mode;
        ef_max = qp[i].ef > ef_max ? qp[i].ef : ef_max;
        k_max = qp[i].k > k_max ? qp[i].k : k_max;
        mc_max = qp[i].mc > mc_max ? qp[i].mc : mc_max;
        mg_max = qp[i].mg > mg_max ? qp[i].mg : mg_max;
        bits_max = qp[i].bloom_bits > bits_max ? qp[i].bloom_bits : bits_max;
        cq_max = qp[i].cq > cq_max ? qp[i].cq : cq_max;
        if (qp[i].mode == FALCON_MODE_INTRA && qp[i].channels > ch_max) ch_max = qp[i].channels;
        any_rerank |= (qp[i].rerank != 0 && qp[i].precision != FALCON_PREC_F32);
    }
    if (out_stride < k_max) return set_error(FALCON_ERR_ARG, "out_stride %d < k %d", out_stride, k_max);
    if (mode == FALCON_MODE_INTRA)
        for (int64_t i = 0; i < np; i++)
            if (qp[i].channels != qp[0].channels)
                return set_error(FALCON_ERR_UNSUPPORTED, "intra-query mode: one channel count per call");
    if (any_rerank)
        for (int64_t i = 0; i < np; i++)
            if (!(qp[i].rerank != 0 && qp[i].precision != FALCON_PREC_F32))
                return set_error(FALCON_ERR_UNSUPPORTED, "rerank must be set for all queries of a call or none");
    if (entry_points && memory == FALCON_MEM_HOST) {
        for (int64_t i = 0; i < nq; i++)
            if (entry_points[i] < 0 || entry_points[i] >= ix->n)
                return set_error(FALCON_ERR_ARG, "entry point of query %lld out of range", (long long)i);
    }

    DeviceGuard guard(ix->device);
    if (!guard.ok) return set_error(FALCON_ERR_CUDA, "cannot select device %d", ix->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream_v);
    int rc = FALCON_OK;
    const bool host = memory == FALCON_MEM_HOST;
    float *d_q = nullptr;
    int32_t *d_entries = nullptr, *d_ids = nullptr, *d_hops = nullptr, *d_vis = nullptr, *d_cand = nullptr;
    float *d_d = nullptr, *d_cand_d = nullptr;
    QParams *d_params = nullptr;
    int32_t *d_scratch = nullptr;   // [0..1] work counter (u64), [2] status
    uint32_t *d_bloom = nullptr;    // global Bloom filters when bloom_bits > kMaxSmemBloomBits
    float *d_tcd = nullptr, *d_td = nullptr;      // trace buffers (host-memory calls)
    int32_t *d_tcn = nullptr, *d_tid = nullptr, *d_tcnt = nullptr;
    int32_t status_h = 0;
    SearchLaunch a;
    memset(&a, 0, sizeof(a));
    {
        const size_t qbytes = (size_t)nq * query_stride * sizeof(float);
        if (host) {
            FALCON_CUDA(cudaMallocAsync((void **)&d_q, qbytes, s));
            FALCON_CUDA(cudaMemcpyAsync(d_q, queries, qbytes, cudaMemcpyHostToDevice, s));
            if (entry_points) {
                FALCON_CUDA(cudaMallocAsync((void **)&d_entries, nq * sizeof(int32_t), s));
                FALCON_CUDA(cudaMemcpyAsync(d_entries, entry_points, nq * sizeof(int32_t), cudaMemcpyHostToDevice, s));
            }
            FALCON_CUDA(cudaMallocAsync((void **)&d_ids, (size_t)nq * out_stride * sizeof(int32_t), s));
            FALCON_CUDA(cudaMallocAsync((void **)&d_d, (size_t)nq * out_stride * sizeof(float), s));
            if (out_hops) FALCON_CUDA(cudaMallocAsync((void **)&d_hops, nq * sizeof(int32_t), s));
            if (out_visited) FALCON_CUDA(cudaMallocAsync((void **)&d_vis, nq * sizeof(int32_t), s));
        }
        FALCON_CUDA(cudaMallocAsync((void **)&d_params, np * sizeof(QParams), s));
        FALCON_CUDA(cudaMemcpyAsync(d_params, qp.data(), np * sizeof(QParams), cudaMemcpyHostToDevice, s));
        FALCON_CUDA(cudaMallocAsync((void **)&d_scratch, 4 * sizeof(int32_t), s));
        FALCON_CUDA(cudaMemsetAsync(d_scratch, 0, 4 * sizeof(int32_t), s));

        a.g.vecs = reinterpret_cast<const unsigned char *>(ix->d_f32);
        a.g.vstride_bytes = (int64_t)ix->dpad * 4;
        if (prec == FALCON_PREC_BF16) {
            a.g.vecs = reinterpret_cast<const unsigned char *>(ix->d_bf16);
            a.g.vstride_bytes = (int64_t)ix->dpad * 2;
        } else if (prec == FALCON_PREC_FP8) {
            a.g.vecs = ix->d_fp8;
            a.g.vstride_bytes = ix->dpad;
        }
        a.g.scales = ix->d_scales;
        a.g.vecs32 = reinterpret_cast<const unsigned char *>(ix->d_f32);
        a.g.vstride32_bytes = (int64_t)ix->dpad * 4;
        a.g.links = ix->d_links;
        a.g.lstride = ix->link_stride;
        a.g.ids_off = ix->ids_offset;
        a.g.max_degree = ix->max_degree;
        a.g.dim = ix->dim;
        a.g.dpad = ix->dpad;
        a.g.n = ix->n;
        a.g.labels = ix->d_labels;
        a.queries = host ? d_q : queries;
        a.qstride = query_stride;
        a.entries = host ? d_entries : entry_points;
        a.default_entry = ix->entry;
        a.nq = nq;
        a.params = d_params;
        a.per_query = per_query_params ? 1 : 0;
        a.out_ids = host ? d_ids : out_ids;
        a.out_d = host ? d_d : out_dists;
        a.out_stride = out_stride;
        a.write_all_ef = 0;
        a.out_hops = host ? d_hops : out_hops;
        a.out_visited = host ? d_vis : out_visited;
        a.work_counter = d_scratch;
        a.status = d_scratch + 2;
        a.bloom_bits_max = bits_max;
        a.ef_max = ef_max;
        a.mc_max = mc_max;
        a.mg_max = mg_max;
        a.channels = (mode == FALCON_MODE_INTRA) ? qp[0].channels : 0;
        a.cq_max = cq_max;
        if (tro) {
            const size_t ncd = (size_t)nq * tro->cand_cap, nd = (size_t)nq * tro->cap;
            if (host) {
                if (ncd) FALCON_CUDA(cudaMallocAsync((void **)&d_tcd, ncd * sizeof(float), s));
                if (ncd) FALCON_CUDA(cudaMallocAsync((void **)&d_tcn, ncd * sizeof(int32_t), s));
                if (nd) FALCON_CUDA(cudaMallocAsync((void **)&d_td, nd * sizeof(float), s));
                if (nd) FALCON_CUDA(cudaMallocAsync((void **)&d_tid, nd * sizeof(int32_t), s));
                FALCON_CUDA(cudaMallocAsync((void **)&d_tcnt, (size_t)nq * 3 * sizeof(int32_t), s));
            }
            a.trace_cand_d = host ? d_tcd : tro->cand_d;
            a.trace_cand_n = host ? d_tcn : tro->cand_n;
            a.trace_cand_cap = tro->cand_cap;
            a.trace_d = host ? d_td : tro->d;
            a.trace_id = host ? d_tid : tro->ids;
            a.trace_cap = tro->cap;
            a.trace_counts = host ? d_tcnt : tro->counts;
        }
        int32_t *final_ids = a.out_ids;
        float *final_d = a.out_d;
        if (any_rerank) {
            FALCON_CUDA(cudaMallocAsync((void **)&d_cand, (size_t)nq * ef_max * sizeof(int32_t), s));
            FALCON_CUDA(cudaMallocAsync((void **)&d_cand_d, (size_t)nq * ef_max * sizeof(float), s));
            a.out_ids = d_cand;
            a.out_d = d_cand_d;
            a.out_stride = ef_max;
            a.write_all_ef = 1;
        }
        const int elem = prec == FALCON_PREC_BF16 ? kBF16 : (prec == FALCON_PREC_FP8 ? kFP8 : kF32);
        if (bits_max > kMaxSmemBloomBits) {
            int64_t slots = 0;
            FALCON_CUDA(search_bloom_slots(a, elem, ix->num_sms, &slots));
            FALCON_CUDA(cudaMallocAsync((void **)&d_bloom, (size_t)slots << (bits_max - 3), s));
            a.bloom_global = d_bloom;
        }
        if (!entry_points && ix->upper_max_level > 0) {   // entries from the upper-layer descent
            if (!ix->d_f32) { rc = set_error(FALCON_ERR_UNSUPPORTED, "the upper-layer descent needs FP32 storage"); goto done; }
            FALCON_CUDA(cudaMallocAsync((void **)&d_entries, nq * sizeof(int32_t), s));
            DescendLaunch dl = descend_launch(ix);
            dl.queries = a.queries;
            dl.qstride = query_stride;
            dl.nq = nq;
            dl.out_entry = d_entries;
            FALCON_CUDA(launch_descend(dl, ix->num_sms, s));
            a.entries = d_entries;
        }
        FALCON_CUDA(launch_search(a, elem, ix->num_sms, s));
        if (any_rerank) {
            RerankLaunch r;
            memset(&r, 0, sizeof(r));
            r.g = a.g;
            r.queries = a.queries;
            r.qstride = a.qstride;
            r.nq = nq;
            r.params = d_params;
            r.per_query = a.per_query;
            r.cand_ids = d_cand;
            r.cand_stride = ef_max;
            r.out_ids = final_ids;
            r.out_d = final_d;
            r.out_stride = out_stride;
            FALCON_CUDA(launch_rerank(r, ef_max, ix->num_sms, s));
        }
        if (host) {
            FALCON_CUDA(cudaMemcpyAsync(out_ids, d_ids, (size_t)nq * out_stride * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            FALCON_CUDA(cudaMemcpyAsync(out_dists, d_d, (size_t)nq * out_stride * sizeof(float), cudaMemcpyDeviceToHost, s));
            if (out_hops) FALCON_CUDA(cudaMemcpyAsync(out_hops, d_hops, nq * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            if (out_visited) FALCON_CUDA(cudaMemcpyAsync(out_visited, d_vis, nq * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            FALCON_CUDA(cudaMemcpyAsync(&status_h, d_scratch + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            if (tro) {
                const size_t ncd = (size_t)nq * tro->cand_cap, nd = (size_t)nq * tro->cap;
                if (ncd) {
                    FALCON_CUDA(cudaMemcpyAsync(tro->cand_d, d_tcd, ncd * sizeof(float), cudaMemcpyDeviceToHost, s));
                    FALCON_CUDA(cudaMemcpyAsync(tro->cand_n, d_tcn, ncd * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
                }
                if (nd) {
                    FALCON_CUDA(cudaMemcpyAsync(tro->d, d_td, nd * sizeof(float), cudaMemcpyDeviceToHost, s));
                    FALCON_CUDA(cudaMemcpyAsync(tro->ids, d_tid, nd * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
                }
                FALCON_CUDA(cudaMemcpyAsync(tro->counts, d_tcnt, (size_t)nq * 3 * sizeof(int32_t),
                                            cudaMemcpyDeviceToHost, s));
            }
        }
    }
done:
    for (void *p : {(void *)d_q, (void *)d_entries, (void *)d_ids, (void *)d_d, (void *)d_hops, (void *)d_vis,
                    (void *)d_params, (void *)d_scratch, (void *)d_cand, (void *)d_cand_d, (void *)d_bloom,
                    (void *)d_tcd, (void *)d_tcn, (void *)d_td, (void *)d_tid, (void *)d_tcnt})
        if (p) cudaFreeAsync(p, s);
    if (rc == FALCON_OK && host) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return set_error(FALCON_ERR_CUDA, "search: %s", cudaGetErrorString(e));
        if (status_h & 1) return FALCON_WARN_TRUNCATED;
    }
    return rc;
}

int falcon_vadd(int32_t query_num, int32_t query_batch_size, int32_t ef, int32_t candidate_queue_runtime_size,
                int32_t max_cand_batch_size, int32_t max_async_stage_num, int32_t runtime_n_bucket_addr_bits,
                uint32_t hash_seed, int32_t max_bloom_out_burst_size, int32_t max_link_num_base, int32_t dim,
                int64_t num_db_vec, const int32_t *entry_point_ids, const float *query_vectors,
                const void *db_vectors, const void *links_base, int32_t *out_id, float *out_dist,
                int32_t *mem_debug, int32_t device)
{
    if (query_num < 0 || query_batch_size < 1 || max_bloom_out_burst_size < 1 || !entry_point_ids || !query_vectors ||
        !db_vectors || !links_base || !out_id || !out_dist || !mem_debug)
        return set_error(FALCON_ERR_ARG, "falcon_vadd: invalid argument");
    falcon_index_desc d;
    memset(&d, 0, sizeof(d));
    d.num_vectors = num_db_vec;
    d.dim = dim;
    d.max_degree = max_link_num_base;
    d.vectors = reinterpret_cast<const float *>(db_vectors);
    d.vector_stride = pad16(dim) + 16;
    d.links = reinterpret_cast<const int32_t *>(links_base);
    d.link_stride = 16LL * (1 + (max_link_num_base + 15) / 16);
    d.ids_offset = 16;
    d.entry_point = query_num > 0 ? entry_point_ids[0] : 0;
    d.device = device;
    falcon_index *ix = nullptr;
    int rc = falcon_index_create(&d, &ix);
    if (rc != FALCON_OK) return rc;
    falcon_search_params p;
    falcon_default_params(&p);
    p.k = ef;
    p.ef = ef;
    p.mc = max_cand_batch_size;
    p.mg = max_async_stage_num;
    p.cand_queue_size = candidate_queue_runtime_size;
    p.bloom_bits = runtime_n_bucket_addr_bits;
    p.hash_seed = hash_seed;
    std::vector<int32_t> hops((size_t)query_num), vis((size_t)query_num);
    rc = falcon_search(ix, query_vectors, query_num, pad16(dim), entry_point_ids, &p, 0, out_id, out_dist, ef,
                       hops.data(), vis.data(), FALCON_MEM_HOST, nullptr);
    if (rc >= 0) {
        for (int32_t i = 0; i < query_num; i++) {
            mem_debug[2 * i] = hops[i];
            mem_debug[2 * i + 1] = vis[i];
        }
    }
    falcon_index_free(ix);
    return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Helpers for falcon_search_noalloc (falcon_noalloc.cu): the same validation
// and launch sequence as falcon_search, with every device buffer supplied by
// the caller.
// ---------------------------------------------------------------------------
namespace falcon {

int set_error_code(int code, const char *msg) { return set_error(code, "%s", msg); }

int check_search_params(const falcon_search_params &p, const falcon_index *ix, int64_t qi)
{
    return check_params(p, ix, qi);
}

// Device view of an index for one traversal precision (the serving kernel's
// per-request graph).  Fails if the index does not hold that storage.
int index_graph_view(const falcon_index *ix, int precision, GraphView *v, int *dim, int *entry)
{
    memset(v, 0, sizeof(*v));
    if (precision == FALCON_PREC_F32) {
        v->vecs = reinterpret_cast<const unsigned char *>(ix->d_f32);
        v->vstride_bytes = (int64_t)ix->dpad * 4;
    } else if (precision == FALCON_PREC_BF16 && ix->d_bf16) {
        v->vecs = reinterpret_cast<const unsigned char *>(ix->d_bf16);
        v->vstride_bytes = (int64_t)ix->dpad * 2;
    } else if (precision == FALCON_PREC_FP8 && ix->d_fp8) {
        v->vecs = ix->d_fp8;
        v->vstride_bytes = ix->dpad;
    } else {
        return set_error(FALCON_ERR_ARG, "index holds no storage for precision %d", precision);
    }
    v->scales = ix->d_scales;
    v->vecs32 = reinterpret_cast<const unsigned char *>(ix->d_f32);
    v->vstride32_bytes = (int64_t)ix->dpad * 4;
    v->links = ix->d_links;
    v->lstride = ix->link_stride;
    v->ids_off = ix->ids_offset;
    v->max_degree = ix->max_degree;
    v->dim = ix->dim;
    v->dpad = ix->dpad;
    v->n = ix->n;
    v->labels = ix->d_labels;
    *dim = ix->dim;
    *entry = ix->entry;
    return FALCON_OK;
}

int index_device(const falcon_index *ix) { return ix->device; }
bool index_has_upper(const falcon_index *ix) { return ix->upper_max_level > 0; }

// A server registers (+1) and releases (-1) the indexes whose device
// pointers it holds; freeing the index or replacing its upper layers is
// refused meanwhile.
void index_server_ref(falcon_index *ix, int delta) { ix->server_refs += delta; }

// The descent launch of an index (upper layers and FP32 vectors; queries and
// outputs left for the caller): false when the index has no upper layers.
// *has_f32 tells whether the FP32 vectors the descent reads are resident.
bool index_descend_launch(const falcon_index *ix, DescendLaunch *a, bool *has_f32)
{
    *has_f32 = ix->d_f32 != nullptr;
    if (ix->upper_max_level < 1) return false;
    *a = descend_launch(ix);
    return true;
}

// Validates a no-allocation request; needs ef >= k in every struct so the
// caller's structs can be copied to the device unchanged (the kernels'
// QParams has the same layout, checked below).
int prepare_search(const falcon_index *ix, int64_t nq, int64_t query_stride, const falcon_search_params *params,
                   int32_t per_query_params, int32_t out_stride, SearchPlan *plan)
{
    static_assert(sizeof(QParams) == sizeof(falcon_search_params), "QParams layout");
    static_assert(offsetof(QParams, k) == offsetof(falcon_search_params, k) &&
                      offsetof(QParams, ef) == offsetof(falcon_search_params, ef) &&
                      offsetof(QParams, mc) == offsetof(falcon_search_params, mc) &&
                      offsetof(QParams, mg) == offsetof(falcon_search_params, mg) &&
                      offsetof(QParams, cq) == offsetof(falcon_search_params, cand_queue_size) &&
                      offsetof(QParams, bloom_bits) == offsetof(falcon_search_params, bloom_bits) &&
                      offsetof(QParams, seed) == offsetof(falcon_search_params, hash_seed) &&
                      offsetof(QParams, mode) == offsetof(falcon_search_params, mode) &&
                      offsetof(QParams, channels) == offsetof(falcon_search_params, channels) &&
                      offsetof(QParams, precision) == offsetof(falcon_search_params, precision) &&
                      offsetof(QParams, rerank) == offsetof(falcon_search_params, rerank) &&
                      offsetof(QParams, max_hops) == offsetof(falcon_search_params, max_hops),
                  "QParams layout");
    // every argument check comes before the caller queues any device work
    if (nq < 0) return set_error(FALCON_ERR_ARG, "nq %lld < 0", (long long)nq);
    if (query_stride < ix->dim)
        return set_error(FALCON_ERR_ARG, "query_stride %lld < dim %d", (long long)query_stride, ix->dim);
    plan->per_query = per_query_params != 0;
    plan->np = plan->per_query ? nq : 1;
    int prec = -1, mode = -1, channels = -1;
    for (int64_t i = 0; i < plan->np; i++) {
        const falcon_search_params &p = params[i];
        const int rc = check_params(p, ix, i);
        if (rc != FALCON_OK) return rc;
        if (p.ef < p.k)
            return set_error(FALCON_ERR_ARG, "falcon_search_noalloc: query %lld has ef %d < k %d (needs ef >= k)",
                             (long long)i, p.ef, p.k);
        if (prec >= 0 && prec != p.precision) return set_error(FALCON_ERR_UNSUPPORTED, "one call must use one precision");
        if (mode >= 0 && mode != p.mode) return set_error(FALCON_ERR_UNSUPPORTED, "one call must use one mode");
        if (p.mode == FALCON_MODE_INTRA && channels >= 0 && p.channels != channels)
            return set_error(FALCON_ERR_UNSUPPORTED, "intra-query mode: one channel count per call");
        prec = p.precision;
        mode = p.mode;
        if (p.mode == FALCON_MODE_INTRA) channels = p.channels;
        plan->ef_max = p.ef > plan->ef_max ? p.ef : plan->ef_max;
        plan->k_max = p.k > plan->k_max ? p.k : plan->k_max;
        plan->mc_max = p.mc > plan->mc_max ? p.mc : plan->mc_max;
        plan->mg_max = p.mg > plan->mg_max ? p.mg : plan->mg_max;
        plan->bits_max = p.bloom_bits > plan->bits_max ? p.bloom_bits : plan->bits_max;
        plan->cq_max = p.cand_queue_size > plan->cq_max ? p.cand_queue_size : plan->cq_max;
        const bool rr = p.rerank != 0 && p.precision != FALCON_PREC_F32;
        if (i > 0 && rr != plan->any_rerank)
            return set_error(FALCON_ERR_UNSUPPORTED, "rerank must be set for all queries of a call or none");
        plan->any_rerank = rr;
    }
    plan->prec = prec;
    plan->mode = mode;
    plan->channels = (mode == FALCON_MODE_INTRA) ? channels : 0;
    if (plan->bits_max > kMaxSmemBloomBits)
        return set_error(FALCON_ERR_ARG, "falcon_search_noalloc: bloom_bits above %d need per-warp filters in "
                         "global memory, which do not fit the static scratch; use falcon_search", kMaxSmemBloomBits);
    if (out_stride < plan->k_max) return set_error(FALCON_ERR_ARG, "out_stride %d < k %d", out_stride, plan->k_max);
    return FALCON_OK;
}

int run_search_plan(const falcon_index *ix, const SearchPlan &plan, int64_t nq, const float *queries,
                    int64_t query_stride, const int32_t *entry_points, QParams *d_params, int32_t *d_scratch,
                    int32_t *d_cand_ids, float *d_cand_d, int32_t *out_ids, float *out_dists, int32_t out_stride,
                    int32_t *out_hops, int32_t *out_visited, int32_t *d_entry_scratch, cudaStream_t s)
{
    if (query_stride < ix->dim)
        return set_error(FALCON_ERR_ARG, "query_stride %lld < dim %d", (long long)query_stride, ix->dim);
    SearchLaunch a;
    memset(&a, 0, sizeof(a));
    a.g.vecs = reinterpret_cast<const unsigned char *>(ix->d_f32);
    a.g.vstride_bytes = (int64_t)ix->dpad * 4;
    if (plan.prec == FALCON_PREC_BF16) {
        a.g.vecs = reinterpret_cast<const unsigned char *>(ix->d_bf16);
        a.g.vstride_bytes = (int64_t)ix->dpad * 2;
    } else if (plan.prec == FALCON_PREC_FP8) {
        a.g.vecs = ix->d_fp8;
        a.g.vstride_bytes = ix->dpad;
    }
    a.g.scales = ix->d_scales;
    a.g.vecs32 = reinterpret_cast<const unsigned char *>(ix->d_f32);
    a.g.vstride32_bytes = (int64_t)ix->dpad * 4;
    a.g.links = ix->d_links;
    a.g.lstride = ix->link_stride;
    a.g.ids_off = ix->ids_offset;
    a.g.max_degree = ix->max_degree;
    a.g.dim = ix->dim;
    a.g.dpad = ix->dpad;
    a.g.n = ix->n;
    a.g.labels = ix->d_labels;
    a.queries = queries;
    a.qstride = query_stride;
    a.entries = entry_points;
    a.default_entry = ix->entry;
    a.nq = nq;
    a.params = d_params;
    a.per_query = plan.per_query ? 1 : 0;
    a.out_ids = plan.any_rerank ? d_cand_ids : out_ids;
    a.out_d = plan.any_rerank ? d_cand_d : out_dists;
    a.out_stride = plan.any_rerank ? plan.ef_max : out_stride;
    a.write_all_ef = plan.any_rerank ? 1 : 0;
    a.out_hops = out_hops;
    a.out_visited = out_visited;
    a.work_counter = d_scratch;
    a.status = d_scratch + 2;
    a.bloom_bits_max = plan.bits_max;
    a.ef_max = plan.ef_max;
    a.mc_max = plan.mc_max;
    a.mg_max = plan.mg_max;
    a.channels = plan.channels;
    a.cq_max = plan.cq_max;
    const int elem = plan.prec == FALCON_PREC_BF16 ? kBF16 : (plan.prec == FALCON_PREC_FP8 ? kFP8 : kF32);
    cudaError_t e;
    if (!entry_points && ix->upper_max_level > 0) {   // entries from the upper-layer descent
        if (!ix->d_f32 || !d_entry_scratch)
            return set_error(FALCON_ERR_UNSUPPORTED, "the upper-layer descent needs FP32 storage and entry scratch");
        DescendLaunch dl = descend_launch(ix);
        dl.queries = queries;
        dl.qstride = query_stride;
        dl.nq = nq;
        dl.out_entry = d_entry_scratch;
        e = launch_descend(dl, ix->num_sms, s);
        if (e != cudaSuccess) return set_error(FALCON_ERR_CUDA, "descend launch: %s", cudaGetErrorString(e));
        a.entries = d_entry_scratch;
    }
    e = launch_search(a, elem, ix->num_sms, s);
    if (e != cudaSuccess) return set_error(FALCON_ERR_CUDA, "search launch: %s", cudaGetErrorString(e));
    if (plan.any_rerank) {
        RerankLaunch r;
        memset(&r, 0, sizeof(r));
        r.g = a.g;
        r.queries = queries;
        r.qstride = query_stride;
        r.nq = nq;
        r.params = d_params;
        r.per_query = a.per_query;
        r.cand_ids = d_cand_ids;
        r.cand_stride = plan.ef_max;
        r.out_ids = out_ids;
        r.out_d = out_dists;
        r.out_stride = out_stride;
        e = launch_rerank(r, plan.ef_max, ix->num_sms, s);
        if (e != cudaSuccess) return set_error(FALCON_ERR_CUDA, "rerank launch: %s", cudaGetErrorString(e));
    }
    return FALCON_OK;
}

}  // namespace falcon
