// Serving: continuous batching of single-query requests against several
// device-resident indexes.
//
// The host appends requests to a device ring (descriptor + query vector,
// copied on a copy stream) and each ring entry to the claim queue of its
// class (traversal precision x register rows, falcon_internal.h), then
// publishes the queues' tail counters.  A persistent serve_kernel
// (falcon_kernels.cu) specialised for one class pulls that class's requests
// one at a time, so a request admitted while others are on the GPU starts as
// soon as a warp frees up and its work overlaps theirs.  Each request carries
// its own index, precision, k, ef, mc, mg (mixed freely).
//
// The kernels of all classes with work run at the same time, each on its own
// stream: with P classes wanting the GPU, each launch gets 1/P of the blocks
// and its own range of per-warp scratch slots (Bloom filters, rerank
// candidates).  Each (class, P, range) launch is captured in a CUDA graph when
// an index of the class is registered (or on first use) and replayed; a launch
// waits for the tails of the submit that caused it.  When another class gets
// work, a running launch whose share is now too large is asked to yield (its
// warps leave between requests) and is relaunched with the smaller share; a
// launch with a smaller share than the current one keeps running until its
// class idles out, so a load that comes and goes does not relaunch kernels.
// A class kernel leaves after `idle_exit_us` without a claim or completion of
// its class (its own start counts as one) and is relaunched by the next submit
// or poll, so an idle server holds no SMs.
//
// Requests to an index with HNSW upper layers get their entry from the
// descent kernel, launched at submit on the copy stream over the new queries
// and writing into the ring descriptors before the tails are published; the
// class kernels leave block slots free for it.  Results go to host-mapped
// memory and complete with a per-entry done word, so the host collects them
// without any CUDA call.
//
// Admission by memory: the ring is sized from the free device memory at
// creation, and each submit admits requests only while the requests in
// flight stay within memory_fraction of the device memory that is free plus
// what the server already holds; a request is refused (not queued) while its
// ring entry is still in use.  The free memory is read by a monitor thread
// every kMemPollMs, never on the submit path: cudaMemGetInfo has been
// measured at up to tens of milliseconds while the class kernels run, so the
// monitor reads the device's memory through NVML (loaded at run time from
// the driver's libnvidia-ml) and falls back to cudaMemGetInfo without it.
#include <cuda_runtime.h>

#include <dlfcn.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/falcon.h"
#include "falcon_internal.h"

using namespace falcon;

namespace falcon {
int set_error_code(int code, const char *msg);
int index_device(const falcon_index *ix);
int index_graph_view(const falcon_index *ix, int precision, GraphView *v, int *dim, int *entry);
bool index_descend_launch(const falcon_index *ix, DescendLaunch *a, bool *has_f32);
void index_server_ref(falcon_index *ix, int delta);
int check_search_params(const falcon_search_params &p, const falcon_index *ix, int64_t qi);
}  // namespace falcon

struct falcon_server {
    falcon_server_config cfg;
    int device = 0, num_sms = 0, epl = 8, vmax = 1, max_grid = 0;
    int grid[kServeClasses] = {};
    size_t smem[kServeClasses] = {};
    bool class_ok[kServeClasses] = {};   // compiled for this server's dim_max
    int cap = 0;                          // ring entries
    int qstride = 0;                      // floats per query slot
    std::mutex mu;
    cudaStream_t cstream = nullptr;
    cudaStream_t ystream = nullptr;       // yield requests: never queued behind a submit's descent
    cudaStream_t kstream[kServeClasses] = {};
    cudaEvent_t kernel_done[kServeClasses] = {};
    cudaEvent_t published = nullptr;      // the last submit's tail copy (copy stream)
    bool published_rec = false;
    // graph[c][P-1][r]: class c's launch over 1/P of the blocks, scratch range r
    cudaGraphExec_t graph[kServeClasses][4][4] = {};
    bool launched[kServeClasses] = {};
    int run_parts[kServeClasses] = {};    // share of the running launch (1/P)
    int run_range[kServeClasses] = {};    // its scratch range (0 .. P-1)
    uint32_t epoch[kServeClasses] = {};   // launches of the class so far; the running launch's epoch
    bool yield_sent[kServeClasses] = {};
    int64_t launches = 0;
    int64_t concurrent_max = 0;           // most class kernels running at once
    std::atomic<int64_t> mem_cap{0};      // requests in flight admitted by memory (monitor thread)
    std::thread mem_monitor;
    std::mutex mem_mu;
    std::condition_variable mem_cv;
    bool mem_stop = false;
    // device
    GraphView *d_views = nullptr;
    ServeDesc *d_ring = nullptr;
    int32_t *d_class_slots = nullptr;     // kServeClasses x cap
    float *d_qpool = nullptr;
    ServeCtl *d_ctl = nullptr;
    int32_t *d_status = nullptr;
    uint32_t *d_bloom = nullptr;
    int32_t *d_cand_ids = nullptr;
    float *d_cand_d = nullptr;
    // host pinned (staging) and host-mapped (results)
    ServeDesc *h_desc = nullptr;
    float *h_qstage = nullptr;
    int32_t *h_class_slots = nullptr;
    int32_t *h_desc_rows = nullptr;             // pinned staging of the ring entries a descent covers
    int32_t *d_desc_rows = nullptr;
    int64_t desc_rows_used = 0;
    unsigned long long *h_tail = nullptr;       // kServeClasses pinned values per ring entry (async copy source)
    uint32_t *h_run_epoch = nullptr;            // host-mapped, per class: read by each launch at start
    uint32_t *h_yield = nullptr;                // pinned sources of yield copies: per class, one per launch mod 16
    int32_t *h_out_ids = nullptr;
    float *h_out_d = nullptr;
    int32_t *h_hops = nullptr, *h_vis = nullptr;
    unsigned long long *h_done = nullptr;
    // bookkeeping
    std::vector<const falcon_index *> indexes;
    std::vector<int> index_dim, index_entry;
    std::vector<int> index_vrows;               // per index and precision
    std::vector<char> index_upper;              // requests start from the upper-layer descent
    std::vector<DescendLaunch> index_dl;
    bool any_upper = false;                     // some index descends: submits launch a descent
    unsigned long long ctail[kServeClasses] = {};   // published per class queue
    int64_t unfinished[kServeClasses] = {};     // submitted, not collected
    std::vector<int> entry_cls;
    std::vector<unsigned long long> entry_seq;  // seq occupying each entry, or ~0 when free
    std::vector<int> entry_k;
    unsigned long long next_seq = 0;
    int64_t in_flight = 0;
    int64_t device_bytes = 0;
    ServeLaunch launch;
};

namespace {

int cuda_fail(cudaError_t e, const char *what)
{
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    return set_error_code(e == cudaErrorMemoryAllocation ? FALCON_ERR_OOM : FALCON_ERR_CUDA, buf);
}

void free_server(falcon_server *sv)
{
    if (sv->mem_monitor.joinable()) {
        {
            std::lock_guard<std::mutex> l(sv->mem_mu);
            sv->mem_stop = true;
        }
        sv->mem_cv.notify_all();
        sv->mem_monitor.join();
    }
    for (int c = 0; c < kServeClasses; c++) {
        for (int p = 0; p < 4; p++)
            for (int r = 0; r < 4; r++)
                if (sv->graph[c][p][r]) cudaGraphExecDestroy(sv->graph[c][p][r]);
        if (sv->kernel_done[c]) cudaEventDestroy(sv->kernel_done[c]);
        if (sv->kstream[c]) cudaStreamDestroy(sv->kstream[c]);
    }
    if (sv->published) cudaEventDestroy(sv->published);
    if (sv->cstream) cudaStreamDestroy(sv->cstream);
    if (sv->ystream) cudaStreamDestroy(sv->ystream);
    cudaFree(sv->d_views);
    cudaFree(sv->d_ring);
    cudaFree(sv->d_class_slots);
    cudaFree(sv->d_qpool);
    cudaFree(sv->d_ctl);
    cudaFree(sv->d_status);
    cudaFree(sv->d_bloom);
    cudaFree(sv->d_cand_ids);
    cudaFree(sv->d_cand_d);
    cudaFreeHost(sv->h_desc);
    cudaFreeHost(sv->h_qstage);
    cudaFreeHost(sv->h_tail);
    cudaFreeHost(sv->h_class_slots);
    cudaFreeHost(sv->h_desc_rows);
    cudaFree(sv->d_desc_rows);
    cudaFreeHost(sv->h_run_epoch);
    cudaFreeHost(sv->h_yield);
    cudaFreeHost(sv->h_out_ids);
    cudaFreeHost(sv->h_out_d);
    cudaFreeHost(sv->h_hops);
    cudaFreeHost(sv->h_vis);
    cudaFreeHost(sv->h_done);
    delete sv;
}

// Block slots the serve kernels leave free for the submit-time descent.
constexpr int kDescendSlots = 8;
// Most classes sharing the SMs at once (more wait for a share to free up).
constexpr int kMaxParts = 4;
// Period of the free-memory monitor.
constexpr int kMemPollMs = 5;

// Whether class c has a request that is neither collected nor done: with no
// kernel running, exactly the requests still to be claimed.  Walks the
// class queue back from its tail until all of the class's uncollected
// entries have been seen (the newest are the likeliest to be pending).
bool class_pending(const falcon_server *sv, int c)
{
    int64_t seen = 0;
    const unsigned long long t = sv->ctail[c];
    for (unsigned long long k = 0; k < t && k < (unsigned long long)sv->cap && seen < sv->unfinished[c]; k++) {
        const int e = sv->h_class_slots[(size_t)c * sv->cap + (t - 1 - k) % (unsigned long long)sv->cap];
        const unsigned long long seq = sv->entry_seq[e];
        if (seq == ~0ull || sv->entry_cls[e] != c) continue;
        seen++;
        if (*reinterpret_cast<volatile unsigned long long *>(sv->h_done + e) != seq + 1) return true;
    }
    return false;
}

// Per-warp scratch slots [lo, hi) of a launch over 1/parts of the blocks in range r.
void scratch_range(const falcon_server *sv, int parts, int r, int *lo, int *hi)
{
    const int w = sv->max_grid * 4 / parts;
    *lo = r * w;
    *hi = *lo + w;
}

// The graph of class c's launch over 1/parts of its blocks in scratch range
// r, captured on first use.  Caller holds mu.
cudaError_t class_graph(falcon_server *sv, int c, int parts, int r, cudaGraphExec_t *out)
{
    cudaGraphExec_t &ge = sv->graph[c][parts - 1][r];
    if (!ge) {
        ServeLaunch L = sv->launch;
        int lo, hi;
        scratch_range(sv, parts, r, &lo, &hi);
        L.warp_base = lo;
        int grid = sv->grid[c] / parts;
        if (grid < 1) grid = 1;
        if (grid * 4 > hi - lo) grid = (hi - lo) / 4;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(sv->kstream[c], cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        e = launch_serve(L, sv->epl, c, grid, sv->smem[c], sv->kstream[c]);
        const cudaError_t e2 = cudaStreamEndCapture(sv->kstream[c], &g);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&ge, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            ge = nullptr;
            return e;
        }
    }
    *out = ge;
    return cudaSuccess;
}

// Keep a kernel running for every class with requests to claim, the classes
// sharing the SMs (see the file comment).  Caller holds mu.
int ensure_running(falcon_server *sv)
{
    bool want[kServeClasses];
    int nwant = 0;
    for (int c = 0; c < kServeClasses; c++) {
        if (sv->launched[c]) {
            const cudaError_t q = cudaEventQuery(sv->kernel_done[c]);
            if (q == cudaSuccess) sv->launched[c] = false;
            else if (q != cudaErrorNotReady) return cuda_fail(q, "serve kernel");
        }
        want[c] = sv->launched[c] || (sv->unfinished[c] > 0 && class_pending(sv, c));
        nwant += want[c] ? 1 : 0;
    }
    if (nwant == 0) return FALCON_OK;
    const int parts = nwant < kMaxParts ? nwant : kMaxParts;
    // a running launch with a larger share than `parts` makes room
    for (int c = 0; c < kServeClasses; c++) {
        if (!sv->launched[c] || sv->yield_sent[c] || sv->run_parts[c] >= parts) continue;
        uint32_t *src = sv->h_yield + c * 16 + (sv->epoch[c] % 16);
        *src = sv->epoch[c];
        const cudaError_t e = cudaMemcpyAsync(&sv->d_ctl->yield_epoch[c], src, sizeof(uint32_t),
                                              cudaMemcpyHostToDevice, sv->ystream);
        if (e != cudaSuccess) return cuda_fail(e, "serve yield");
        sv->yield_sent[c] = true;
    }
    // launch the classes that want the GPU into a free scratch range
    for (int c = 0; c < kServeClasses; c++) {
        if (!want[c] || sv->launched[c]) continue;
        int range = -1;
        for (int r = 0; r < parts && range < 0; r++) {
            int lo, hi;
            scratch_range(sv, parts, r, &lo, &hi);
            bool free_r = true;
            for (int o = 0; o < kServeClasses && free_r; o++) {
                if (!sv->launched[o]) continue;
                int olo, ohi;
                scratch_range(sv, sv->run_parts[o], sv->run_range[o], &olo, &ohi);
                free_r = ohi <= lo || hi <= olo;
            }
            if (free_r) range = r;
        }
        if (range < 0) continue;   // a yielding launch still holds the range: next pass
        cudaGraphExec_t ge;
        cudaError_t e = class_graph(sv, c, parts, range, &ge);
        if (e != cudaSuccess) return cuda_fail(e, "serve graph");
        sv->h_run_epoch[c] = ++sv->epoch[c];
        // the launch starts after the tails it is launched for have landed
        if (sv->published_rec) e = cudaStreamWaitEvent(sv->kstream[c], sv->published, 0);
        if (e == cudaSuccess) e = cudaGraphLaunch(ge, sv->kstream[c]);
        if (e == cudaSuccess) e = cudaEventRecord(sv->kernel_done[c], sv->kstream[c]);
        if (e != cudaSuccess) return cuda_fail(e, "serve kernel launch");
        sv->launched[c] = true;
        sv->run_parts[c] = parts;
        sv->run_range[c] = range;
        sv->yield_sent[c] = false;
        sv->launches++;
    }
    int64_t running = 0;
    for (int c = 0; c < kServeClasses; c++) running += sv->launched[c] ? 1 : 0;
    if (running > sv->concurrent_max) sv->concurrent_max = running;
    return FALCON_OK;
}

// NVML's memory query, resolved from the driver's library at run time.
struct NvmlMemory {
    unsigned long long total, free, used;
};
struct NvmlMem {
    void *lib = nullptr;
    void *dev = nullptr;
    int (*shutdown)() = nullptr;
    int (*mem)(void *, NvmlMemory *) = nullptr;

    bool open(int device)
    {
        char bus[32];
        if (cudaDeviceGetPCIBusId(bus, (int)sizeof(bus), device) != cudaSuccess) return false;
        lib = dlopen("libnvidia-ml.so.1", RTLD_NOW | RTLD_LOCAL);
        if (!lib) return false;
        auto init = reinterpret_cast<int (*)()>(dlsym(lib, "nvmlInit_v2"));
        auto by_bus = reinterpret_cast<int (*)(const char *, void **)>(dlsym(lib, "nvmlDeviceGetHandleByPciBusId_v2"));
        shutdown = reinterpret_cast<int (*)()>(dlsym(lib, "nvmlShutdown"));
        mem = reinterpret_cast<int (*)(void *, NvmlMemory *)>(dlsym(lib, "nvmlDeviceGetMemoryInfo"));
        if (!init || !by_bus || !shutdown || !mem || init() != 0) {
            dlclose(lib);
            lib = nullptr;
            return false;
        }
        if (by_bus(bus, &dev) != 0) {
            close();
            return false;
        }
        return true;
    }
    bool free_bytes(size_t *out)
    {
        NvmlMemory m;
        if (!lib || mem(dev, &m) != 0) return false;
        *out = (size_t)m.free;
        return true;
    }
    void close()
    {
        if (lib) {
            shutdown();
            dlclose(lib);
            lib = nullptr;
        }
    }
};

// Requests in flight that free_bytes of free device memory allows:
// memory_fraction of (free memory + the server's own), at most the ring.
int64_t memory_cap_for(const falcon_server *sv, size_t free_b)
{
    const double per = (double)(sizeof(float) * sv->qstride + sizeof(ServeDesc));
    const double budget = sv->cfg.memory_fraction * ((double)free_b + (double)sv->device_bytes);
    const int64_t cap = (int64_t)(budget / per);
    return cap < sv->cap ? (cap < 1 ? 1 : cap) : sv->cap;
}

// The monitor thread: publishes the admission cap every kMemPollMs.
void memory_monitor(falcon_server *sv)
{
    NvmlMem nv;
    const bool have_nvml = nv.open(sv->device);
    if (!have_nvml) cudaSetDevice(sv->device);
    std::unique_lock<std::mutex> l(sv->mem_mu);
    while (!sv->mem_stop) {
        l.unlock();
        size_t free_b = 0, total_b = 0;
        bool ok = have_nvml ? nv.free_bytes(&free_b) : (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess);
        if (ok) sv->mem_cap.store(memory_cap_for(sv, free_b), std::memory_order_relaxed);
        l.lock();
        sv->mem_cv.wait_for(l, std::chrono::milliseconds(kMemPollMs), [sv] { return sv->mem_stop; });
    }
    l.unlock();
    nv.close();
}

int64_t memory_admission_cap(const falcon_server *sv)
{
    return sv->mem_cap.load(std::memory_order_relaxed);
}

}  // namespace

extern "C" {

void falcon_server_default_config(falcon_server_config *c)
{
    if (!c) return;
    memset(c, 0, sizeof(*c));
    c->device = 0;
    c->ring_capacity = 16384;
    c->max_k = 100;
    c->ef_max = 256;
    c->cand_queue_max = 64;
    c->bloom_bits_max = 16;
    c->mc_max = 4;
    c->mg_max = 8;
    c->dim_max = 512;
    c->idle_exit_us = 2000;
    c->memory_fraction = 0.25;
}

int falcon_server_create(const falcon_server_config *c, falcon_server **out)
{
    if (!c || !out) return set_error_code(FALCON_ERR_ARG, "falcon_server_create: null argument");
    *out = nullptr;
    if (c->ring_capacity < 1 || c->max_k < 1 || c->ef_max < 1 || c->ef_max > kMaxEf || c->max_k > c->ef_max ||
        c->cand_queue_max < 1 || c->cand_queue_max > kMaxCandQueue || c->bloom_bits_max < kMinBloomBits ||
        c->bloom_bits_max > kMaxBloomBits || c->mc_max < 1 || c->mc_max > kMaxMc || c->mg_max < 1 ||
        c->mg_max > kMaxMg || c->dim_max < 1 || c->dim_max > kMaxDimPadded || c->idle_exit_us < 1 ||
        !(c->memory_fraction > 0.0 && c->memory_fraction <= 1.0))
        return set_error_code(FALCON_ERR_ARG, "falcon_server_create: invalid configuration");
    if (cudaSetDevice(c->device) != cudaSuccess)
        return set_error_code(FALCON_ERR_CUDA, "falcon_server_create: cannot select device");
    falcon_server *sv = new falcon_server;
    sv->cfg = *c;
    sv->device = c->device;
    sv->epl = (c->ef_max <= 256 && c->cand_queue_max <= 64) ? 8 : 32;
    sv->qstride = (c->dim_max + 15) / 16 * 16;
    sv->vmax = (sv->qstride + 127) / 128;   // FP32 16-byte rows per lane for the largest dimension
    cudaError_t e;
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, c->device)) != cudaSuccess) { free_server(sv); return cuda_fail(e, "properties"); }
    sv->num_sms = prop.multiProcessorCount;
    // admission by free device memory: per-entry device state is the query
    // slot and the descriptor
    size_t free_b = 0, total_b = 0;
    if ((e = cudaMemGetInfo(&free_b, &total_b)) != cudaSuccess) { free_server(sv); return cuda_fail(e, "mem info"); }
    const size_t per_entry = sizeof(float) * sv->qstride + sizeof(ServeDesc);
    const size_t budget = (size_t)(c->memory_fraction * (double)free_b);
    int64_t cap = c->ring_capacity;
    if ((int64_t)(budget / per_entry) < cap) cap = (int64_t)(budget / per_entry);
    if (cap < 1) { free_server(sv); return set_error_code(FALCON_ERR_OOM, "falcon_server_create: no device memory for requests"); }
    sv->cap = (int)cap;
    // kernel configuration (needs the launch struct's sizes)
    ServeLaunch &L = sv->launch;
    memset(&L, 0, sizeof(L));
    L.ring_cap = sv->cap;
    L.qstride = sv->qstride;
    L.out_stride = c->max_k;
    L.bloom_bits_max = c->bloom_bits_max;
    L.mc_max = c->mc_max;
    L.mg_max = c->mg_max;
    L.ef_max = c->ef_max;
    L.cq_max = c->cand_queue_max;
    L.idle_ns = (long long)c->idle_exit_us * 1000;
    // the classes a registered index can need: FP32 rows up to vmax, BF16 up
    // to ceil(vmax / 2), FP8 one row (dimensions <= 512)
    for (int r = 1; r <= 4; r++) sv->class_ok[serve_class(kF32, r)] = r <= sv->vmax;
    for (int r = 1; r <= 2; r++) sv->class_ok[serve_class(kBF16, r)] = r <= (sv->vmax + 1) / 2;
    sv->class_ok[serve_class(kFP8, 1)] = true;
    for (int c = 0; c < kServeClasses; c++) {
        if (!sv->class_ok[c]) continue;
        if ((e = serve_config(L, sv->epl, c, sv->num_sms, &sv->grid[c], &sv->smem[c])) != cudaSuccess) {
            free_server(sv);
            return cuda_fail(e, "serve kernel configuration");
        }
        // leave kDescendSlots block slots free, so that the descent of newly
        // submitted requests (an ordinary kernel on the copy stream) finds room
        // while a persistent class kernel holds the GPU
        if (sv->grid[c] > kDescendSlots) sv->grid[c] -= kDescendSlots;
        if (sv->grid[c] > sv->max_grid) sv->max_grid = sv->grid[c];
    }
    const size_t warps = (size_t)sv->max_grid * 4;
#define SV_ALLOC(call, what)                      \
    if ((e = (call)) != cudaSuccess) {            \
        free_server(sv);                          \
        return cuda_fail(e, what);                \
    }
    for (int c = 0; c < kServeClasses; c++) {
        SV_ALLOC(cudaStreamCreateWithFlags(&sv->kstream[c], cudaStreamNonBlocking), "stream");
        SV_ALLOC(cudaEventCreateWithFlags(&sv->kernel_done[c], cudaEventDisableTiming), "event");
    }
    SV_ALLOC(cudaStreamCreateWithFlags(&sv->cstream, cudaStreamNonBlocking), "stream");
    SV_ALLOC(cudaStreamCreateWithFlags(&sv->ystream, cudaStreamNonBlocking), "stream");
    SV_ALLOC(cudaEventCreateWithFlags(&sv->published, cudaEventDisableTiming), "event");
    SV_ALLOC(cudaMalloc(&sv->d_views, sizeof(GraphView) * 48), "views");
    SV_ALLOC(cudaMalloc(&sv->d_ring, sizeof(ServeDesc) * sv->cap), "ring");
    SV_ALLOC(cudaMalloc(&sv->d_class_slots, sizeof(int32_t) * kServeClasses * (size_t)sv->cap), "class queues");
    SV_ALLOC(cudaMalloc(&sv->d_qpool, sizeof(float) * (size_t)sv->qstride * sv->cap), "query pool");
    SV_ALLOC(cudaMalloc(&sv->d_ctl, sizeof(ServeCtl)), "control");
    SV_ALLOC(cudaMemset(sv->d_ctl, 0, sizeof(ServeCtl)), "control");
    SV_ALLOC(cudaMalloc(&sv->d_status, sizeof(int32_t)), "status");
    SV_ALLOC(cudaMemset(sv->d_status, 0, sizeof(int32_t)), "status");
    SV_ALLOC(cudaMalloc(&sv->d_cand_ids, sizeof(int32_t) * warps * c->ef_max), "rerank scratch");
    SV_ALLOC(cudaMalloc(&sv->d_cand_d, sizeof(float) * warps * c->ef_max), "rerank scratch");
    if (c->bloom_bits_max > kMaxSmemBloomBits)
        SV_ALLOC(cudaMalloc(&sv->d_bloom, warps << (c->bloom_bits_max - 3)), "Bloom filters");
    SV_ALLOC(cudaHostAlloc(&sv->h_desc, sizeof(ServeDesc) * sv->cap, cudaHostAllocDefault), "pinned");
    SV_ALLOC(cudaHostAlloc(&sv->h_qstage, sizeof(float) * (size_t)sv->qstride * sv->cap, cudaHostAllocDefault), "pinned");
    SV_ALLOC(cudaHostAlloc(&sv->h_tail, sizeof(unsigned long long) * kServeClasses * sv->cap, cudaHostAllocDefault),
             "pinned");
    SV_ALLOC(cudaHostAlloc(&sv->h_class_slots, sizeof(int32_t) * kServeClasses * (size_t)sv->cap, cudaHostAllocDefault),
             "pinned");
    // descent row lists: twice the ring, so a list copied on the copy stream is
    // not overwritten before that stream has read it (a submit admits at most
    // the ring's free entries)
    SV_ALLOC(cudaHostAlloc(&sv->h_desc_rows, sizeof(int32_t) * 2 * (size_t)sv->cap, cudaHostAllocDefault), "pinned");
    SV_ALLOC(cudaMalloc(&sv->d_desc_rows, sizeof(int32_t) * 2 * (size_t)sv->cap), "descent rows");
    SV_ALLOC(cudaHostAlloc(&sv->h_run_epoch, sizeof(uint32_t) * kServeClasses, cudaHostAllocMapped), "mapped");
    SV_ALLOC(cudaHostAlloc(&sv->h_yield, sizeof(uint32_t) * 16 * kServeClasses, cudaHostAllocDefault), "pinned");
    memset(sv->h_run_epoch, 0, sizeof(uint32_t) * kServeClasses);
    SV_ALLOC(cudaHostAlloc(&sv->h_out_ids, sizeof(int32_t) * (size_t)c->max_k * sv->cap, cudaHostAllocMapped), "mapped");
    SV_ALLOC(cudaHostAlloc(&sv->h_out_d, sizeof(float) * (size_t)c->max_k * sv->cap, cudaHostAllocMapped), "mapped");
    SV_ALLOC(cudaHostAlloc(&sv->h_hops, sizeof(int32_t) * sv->cap, cudaHostAllocMapped), "mapped");
    SV_ALLOC(cudaHostAlloc(&sv->h_vis, sizeof(int32_t) * sv->cap, cudaHostAllocMapped), "mapped");
    SV_ALLOC(cudaHostAlloc(&sv->h_done, sizeof(unsigned long long) * sv->cap, cudaHostAllocMapped), "mapped");
    memset(sv->h_done, 0, sizeof(unsigned long long) * sv->cap);
    memset(sv->h_qstage, 0, sizeof(float) * (size_t)sv->qstride * sv->cap);
    sv->device_bytes = (int64_t)(sizeof(ServeDesc) + sizeof(float) * sv->qstride + 4 * kServeClasses) * sv->cap +
                       (int64_t)warps * c->ef_max * 8 +
                       (c->bloom_bits_max > kMaxSmemBloomBits ? (int64_t)(warps << (c->bloom_bits_max - 3)) : 0);
    void *dp;
    L.views = sv->d_views;
    L.ring = sv->d_ring;
    L.class_slots = sv->d_class_slots;
    SV_ALLOC(cudaHostGetDevicePointer(&dp, sv->h_run_epoch, 0), "mapped pointer");
    L.run_epoch = (const uint32_t *)dp;
    L.qpool = sv->d_qpool;
    SV_ALLOC(cudaHostGetDevicePointer(&dp, sv->h_out_ids, 0), "mapped pointer");
    L.out_ids = (int32_t *)dp;
    SV_ALLOC(cudaHostGetDevicePointer(&dp, sv->h_out_d, 0), "mapped pointer");
    L.out_d = (float *)dp;
    SV_ALLOC(cudaHostGetDevicePointer(&dp, sv->h_hops, 0), "mapped pointer");
    L.out_hops = (int32_t *)dp;
    SV_ALLOC(cudaHostGetDevicePointer(&dp, sv->h_vis, 0), "mapped pointer");
    L.out_visited = (int32_t *)dp;
    SV_ALLOC(cudaHostGetDevicePointer(&dp, sv->h_done, 0), "mapped pointer");
    L.done = (unsigned long long *)dp;
    L.ctl = sv->d_ctl;
    L.status = sv->d_status;
    L.bloom_global = sv->d_bloom;
    L.cand_ids = sv->d_cand_ids;
    L.cand_d = sv->d_cand_d;
    L.warp_base = 0;
    // each (class, share, scratch range) launch is captured on first use (class_graph)
#undef SV_ALLOC
    sv->entry_seq.assign(sv->cap, ~0ull);
    sv->entry_k.assign(sv->cap, 0);
    sv->entry_cls.assign(sv->cap, 0);
    // the first admission cap from the reading above, then the monitor's
    sv->mem_cap.store(memory_cap_for(sv, free_b), std::memory_order_relaxed);
    try {
        sv->mem_monitor = std::thread(memory_monitor, sv);
    } catch (...) {
        free_server(sv);
        return set_error_code(FALCON_ERR_OOM, "falcon_server_create: cannot start the memory monitor");
    }
    *out = sv;
    return FALCON_OK;
}

int falcon_server_add_index(falcon_server *sv, falcon_index *ix, int32_t *index_id)
{
    if (!sv || !ix || !index_id) return set_error_code(FALCON_ERR_ARG, "falcon_server_add_index: null argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    if (index_device(ix) != sv->device) return set_error_code(FALCON_ERR_ARG, "index lives on another device");
    if (sv->indexes.size() >= 16) return set_error_code(FALCON_ERR_ARG, "at most 16 indexes per server");
    GraphView v;
    int dim = 0, entry = 0;
    int rc = index_graph_view(ix, FALCON_PREC_F32, &v, &dim, &entry);
    if (rc != FALCON_OK) return rc;
    if (dim > sv->cfg.dim_max) return set_error_code(FALCON_ERR_ARG, "index dimension above the server's dim_max");
    DescendLaunch dl;
    bool has_f32 = false;
    const bool upper = index_descend_launch(ix, &dl, &has_f32);
    if (upper && !has_f32) return set_error_code(FALCON_ERR_UNSUPPORTED, "the upper-layer descent needs FP32 storage");
    const int id = (int)sv->indexes.size();
    // one device view per precision the index holds: slot id*3 + precision
    GraphView views[3];
    for (int pr = 0; pr < 3; pr++) {
        int d2 = 0, e2 = 0;
        if (index_graph_view(ix, pr, &views[pr], &d2, &e2) != FALCON_OK) views[pr] = v;
    }
    cudaError_t e = cudaMemcpy(sv->d_views + 3 * id, views, sizeof(views), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "register index");
    // nothing below can fail: the index is registered in one step
    sv->indexes.push_back(ix);
    index_server_ref(ix, +1);
    sv->index_dim.push_back(dim);
    sv->index_entry.push_back(upper ? -1 : entry);
    sv->index_upper.push_back(upper ? 1 : 0);
    sv->index_dl.push_back(dl);
    if (upper) sv->any_upper = true;
    for (int pr = 0; pr < 3; pr++) sv->index_vrows.push_back(serve_vrows(views[pr].dpad, pr));
    *index_id = id;
    // capture the launches of the index's classes now, so that the first
    // requests of a share do not wait for a graph instantiation (a failure
    // here only leaves the capture to first use)
    for (int pr = 0; pr < 3; pr++) {
        int d2 = 0, e2 = 0;
        GraphView pv;
        if (index_graph_view(ix, pr, &pv, &d2, &e2) != FALCON_OK) continue;
        const int cls = serve_class(pr, serve_vrows(pv.dpad, pr));
        if (cls < 0 || cls >= kServeClasses || !sv->class_ok[cls] || sv->launched[cls]) continue;
        for (int parts = 1; parts <= kMaxParts; parts++)
            for (int r = 0; r < parts; r++) {
                cudaGraphExec_t ge;
                if (class_graph(sv, cls, parts, r, &ge) != cudaSuccess) cudaGetLastError();
            }
    }
    return FALCON_OK;
}

int falcon_server_submit(falcon_server *sv, int32_t n, const int32_t *index_ids, const float *queries,
                         int64_t query_stride, const falcon_search_params *params, int32_t per_request_params,
                         int64_t *request_ids)
{
    if (!sv || n < 0 || (n > 0 && (!index_ids || !queries || !params || !request_ids)))
        return set_error_code(FALCON_ERR_ARG, "falcon_server_submit: null argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    if (cudaSetDevice(sv->device) != cudaSuccess) return set_error_code(FALCON_ERR_CUDA, "select device");
    // validate every request first, so a refused call stages nothing
    for (int i = 0; i < n; i++) {
        const int idx = index_ids[i];
        if (idx < 0 || idx >= (int)sv->indexes.size()) return set_error_code(FALCON_ERR_ARG, "unknown index id");
        const falcon_search_params &p = params[per_request_params ? i : 0];
        int rc = check_search_params(p, sv->indexes[idx], i);
        if (rc != FALCON_OK) return rc;
        const int ef = p.ef < p.k ? p.k : p.ef;
        if (p.k > sv->cfg.max_k || ef > sv->cfg.ef_max || p.cand_queue_size > sv->cfg.cand_queue_max ||
            p.bloom_bits > sv->cfg.bloom_bits_max || p.mc > sv->cfg.mc_max || p.mg > sv->cfg.mg_max ||
            p.mode != FALCON_MODE_INTER)
            return set_error_code(FALCON_ERR_ARG, "request parameters exceed the server's configuration");
        if (query_stride < sv->index_dim[idx]) return set_error_code(FALCON_ERR_ARG, "query_stride < dim");
        const int cls = serve_class(p.precision, sv->index_vrows[3 * idx + p.precision]);
        if (cls < 0 || cls >= kServeClasses || !sv->class_ok[cls])
            return set_error_code(FALCON_ERR_ARG, "request class not built for this server's dim_max");
    }
    // then admit in order while ring entries are free and the free device
    // memory allows more requests in flight
    int admitted = 0;
    const unsigned long long first = sv->next_seq;
    unsigned long long ctail0[kServeClasses];
    int64_t unfinished0[kServeClasses];
    memcpy(ctail0, sv->ctail, sizeof(ctail0));
    memcpy(unfinished0, sv->unfinished, sizeof(unfinished0));
    const int64_t room = memory_admission_cap(sv) - sv->in_flight;
    for (int i = 0; i < n && i < room; i++) {
        const int idx = index_ids[i];
        const falcon_search_params &p = params[per_request_params ? i : 0];
        const int ef = p.ef < p.k ? p.k : p.ef;
        const int cls = serve_class(p.precision, sv->index_vrows[3 * idx + p.precision]);
        const unsigned long long seq = first + (unsigned long long)i;
        const int e = (int)(seq % (unsigned long long)sv->cap);
        if (sv->entry_seq[e] != ~0ull) break;   // entry still in use: stop admitting
        ServeDesc &d = sv->h_desc[e];
        d.index = 3 * idx + p.precision;
        d.precision = p.precision;
        d.entry = sv->index_entry[idx];
        d.pad = 0;
        d.seq = seq;
        d.p.k = p.k;
        d.p.ef = ef;
        d.p.mc = p.mc;
        d.p.mg = p.mg;
        d.p.cq = p.cand_queue_size;
        d.p.bloom_bits = p.bloom_bits;
        d.p.seed = p.hash_seed;
        d.p.mode = 0;
        d.p.channels = 0;
        d.p.precision = p.precision;
        d.p.rerank = p.rerank;
        d.p.max_hops = p.max_hops;
        float *qs = sv->h_qstage + (size_t)e * sv->qstride;
        memcpy(qs, queries + (size_t)i * query_stride, sizeof(float) * sv->index_dim[idx]);
        for (int j = sv->index_dim[idx]; j < sv->qstride; j++) qs[j] = 0.0f;
        sv->entry_seq[e] = seq;
        sv->entry_k[e] = p.k;
        sv->entry_cls[e] = cls;
        sv->h_class_slots[(size_t)cls * sv->cap + sv->ctail[cls] % (unsigned long long)sv->cap] = e;
        sv->ctail[cls]++;
        sv->unfinished[cls]++;
        request_ids[i] = (int64_t)seq;
        admitted++;
    }
    if (admitted == 0) return 0;
    // copy descriptors and queries (at most two contiguous ranges), then publish the tail
    const int e0 = (int)(first % (unsigned long long)sv->cap);
    const int run1 = admitted < sv->cap - e0 ? admitted : sv->cap - e0;
    cudaError_t err = cudaSuccess;
    for (int part = 0; part < 2 && err == cudaSuccess; part++) {
        const int s0 = part == 0 ? e0 : 0;
        const int cnt = part == 0 ? run1 : admitted - run1;
        if (cnt <= 0) continue;
        err = cudaMemcpyAsync(sv->d_qpool + (size_t)s0 * sv->qstride, sv->h_qstage + (size_t)s0 * sv->qstride,
                              sizeof(float) * (size_t)sv->qstride * cnt, cudaMemcpyHostToDevice, sv->cstream);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(sv->d_ring + s0, sv->h_desc + s0, sizeof(ServeDesc) * cnt, cudaMemcpyHostToDevice,
                                  sv->cstream);
    }
    // entries of requests to indexes with upper layers: the greedy descent of
    // their queries, written into the ring descriptors before the tails are
    // published (same stream); one launch per such index over the list of its
    // new ring entries, wherever they lie in the ring
    for (int idx = 0; idx < (int)sv->indexes.size() && err == cudaSuccess; idx++) {
        if (!sv->index_upper[idx]) continue;
        int cnt = 0;
        int32_t *lst = sv->h_desc_rows + (size_t)sv->desc_rows_used;
        for (int i = 0; i < admitted; i++)
            if (index_ids[i] == idx) lst[cnt++] = (int32_t)((first + (unsigned long long)i) % (unsigned long long)sv->cap);
        if (cnt == 0) continue;
        int32_t *dlst = sv->d_desc_rows + (size_t)sv->desc_rows_used;
        sv->desc_rows_used = (sv->desc_rows_used + cnt) % sv->cap;   // the staging area is reused round robin
        err = cudaMemcpyAsync(dlst, lst, sizeof(int32_t) * cnt, cudaMemcpyHostToDevice, sv->cstream);
        if (err != cudaSuccess) break;
        DescendLaunch dl = sv->index_dl[idx];
        dl.queries = sv->d_qpool;
        dl.qstride = sv->qstride;
        dl.nq = cnt;
        dl.rows = dlst;
        dl.out_entry = &sv->d_ring[0].entry;
        dl.out_entry_stride = (int64_t)(sizeof(ServeDesc) / sizeof(int32_t));
        dl.out_hops = nullptr;
        err = launch_descend(dl, sv->num_sms, sv->cstream);
    }
    // each class queue's new slots (at most two contiguous ranges), then all tails in one copy
    for (int c = 0; c < kServeClasses && err == cudaSuccess; c++) {
        const unsigned long long n_new = sv->ctail[c] - ctail0[c];
        if (n_new == 0) continue;
        const int q0 = (int)(ctail0[c] % (unsigned long long)sv->cap);
        const int r1 = (int)(n_new < (unsigned long long)(sv->cap - q0) ? n_new : (unsigned long long)(sv->cap - q0));
        int32_t *dq = sv->d_class_slots + (size_t)c * sv->cap;
        const int32_t *hq = sv->h_class_slots + (size_t)c * sv->cap;
        err = cudaMemcpyAsync(dq + q0, hq + q0, sizeof(int32_t) * r1, cudaMemcpyHostToDevice, sv->cstream);
        if (err == cudaSuccess && (int)n_new > r1)
            err = cudaMemcpyAsync(dq, hq, sizeof(int32_t) * ((int)n_new - r1), cudaMemcpyHostToDevice, sv->cstream);
    }
    const unsigned long long tail = first + admitted;
    const int te = (int)((tail - 1) % (unsigned long long)sv->cap);
    unsigned long long *tails = sv->h_tail + (size_t)te * kServeClasses;
    memcpy(tails, sv->ctail, sizeof(unsigned long long) * kServeClasses);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(sv->d_ctl->tail, tails, sizeof(unsigned long long) * kServeClasses,
                              cudaMemcpyHostToDevice, sv->cstream);
    if (err != cudaSuccess) {
        // nothing was published (the tails go last): take the admissions back,
        // so the next submit reuses the same entries and sequence numbers
        for (int i = 0; i < admitted; i++) sv->entry_seq[(first + (unsigned long long)i) % (unsigned long long)sv->cap] = ~0ull;
        memcpy(sv->ctail, ctail0, sizeof(ctail0));
        memcpy(sv->unfinished, unfinished0, sizeof(unfinished0));
        return cuda_fail(err, "publish requests");
    }
    sv->next_seq = tail;
    sv->in_flight += admitted;
    // class kernels launched from now on wait for these tails (without the
    // event a launch could start first; it then idles until they land)
    if (cudaEventRecord(sv->published, sv->cstream) == cudaSuccess) sv->published_rec = true;
    const int rc = ensure_running(sv);
    return rc != FALCON_OK ? rc : admitted;
}

}  // extern "C"

namespace {
// Collect one request if its done word is set (the lock is held): 1 done,
// 0 pending, < 0 error.  No CUDA call.
int collect_locked(falcon_server *sv, unsigned long long seq, int32_t *out_ids, float *out_dists, int32_t *hops,
                   int32_t *visited)
{
    const int e = (int)(seq % (unsigned long long)sv->cap);
    if (sv->entry_seq[e] != seq) return set_error_code(FALCON_ERR_ARG, "unknown or already collected request");
    const unsigned long long d = *reinterpret_cast<volatile unsigned long long *>(sv->h_done + e);
    if (d != seq + 1) return 0;
    std::atomic_thread_fence(std::memory_order_acquire);
    const int k = sv->entry_k[e];
    if (out_ids) memcpy(out_ids, sv->h_out_ids + (size_t)e * sv->cfg.max_k, sizeof(int32_t) * k);
    if (out_dists) memcpy(out_dists, sv->h_out_d + (size_t)e * sv->cfg.max_k, sizeof(float) * k);
    if (hops) *hops = sv->h_hops[e];
    if (visited) *visited = sv->h_vis[e];
    sv->entry_seq[e] = ~0ull;
    sv->in_flight--;
    sv->unfinished[sv->entry_cls[e]]--;
    return 1;
}
}  // namespace

extern "C" {

int falcon_server_poll(falcon_server *sv, int64_t request_id, int32_t *out_ids, float *out_dists, int32_t *hops,
                       int32_t *visited)
{
    if (!sv || request_id < 0) return set_error_code(FALCON_ERR_ARG, "falcon_server_poll: bad argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    const int rc = collect_locked(sv, (unsigned long long)request_id, out_ids, out_dists, hops, visited);
    if (rc == 0) {
        // the kernel may have left on idleness just before this request was published
        cudaSetDevice(sv->device);
        const int lr = ensure_running(sv);
        return lr != FALCON_OK ? lr : 0;
    }
    return rc;
}

int falcon_server_wait(falcon_server *sv, int64_t request_id, int64_t timeout_us, int32_t *out_ids,
                       float *out_dists, int32_t *hops, int32_t *visited)
{
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const int rc = falcon_server_poll(sv, request_id, out_ids, out_dists, hops, visited);
        if (rc != 0) return rc == 1 ? FALCON_OK : rc;
        const auto us = std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count();
        if (us > timeout_us) return set_error_code(FALCON_ERR_CUDA, "falcon_server_wait: timed out");
        std::this_thread::yield();
    }
}

int falcon_server_replay(falcon_server *sv, int32_t n, const int32_t *index_ids, const float *queries,
                         int64_t query_stride, const falcon_search_params *params, int32_t per_request_params,
                         const double *arrival_us, double *latency_us, int32_t *out_ids, int32_t out_stride,
                         float *out_dists, int32_t *hops, int32_t *visited, double *elapsed_us)
{
    if (!sv || n < 0 || !arrival_us || !latency_us || (n > 0 && (!index_ids || !queries || !params)))
        return set_error_code(FALCON_ERR_ARG, "falcon_server_replay: null argument");
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    auto now_us = [&]() { return std::chrono::duration<double, std::micro>(clk::now() - t0).count(); };
    std::vector<int64_t> rid((size_t)n, -1);
    std::vector<int> pending;            // submitted, not collected
    pending.reserve(n > 0 ? (size_t)n : 1);
    int next = 0, done = 0;
    std::vector<int32_t> tmp_ids(sv->cfg.max_k);
    std::vector<float> tmp_d(sv->cfg.max_k);
    const int kBatch = 512;
    // Every submit to an index with upper layers launches one descent, a chain
    // of dependent row reads of about 50 us that holds the copy stream; a
    // submit per few arrivals would queue them faster than the stream drains.
    // With such an index, arrivals are gathered into micro-batches instead.
    bool any_upper;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        any_upper = sv->any_upper;
    }
    const double kSubmitWindowUs = 200.0;
    double last_submit = -1e30;
    while (done < n) {
        const double t = now_us();
        // submit everything that has arrived (in order), as ring entries allow
        int end = next;
        while (end < n && arrival_us[end] <= t && end - next < kBatch) end++;
        const bool wait_window = any_upper && end - next < kBatch && t - last_submit < kSubmitWindowUs;
        if (end > next && !wait_window) {
            last_submit = t;
            const int cnt = end - next;
            const int rc = falcon_server_submit(sv, cnt, index_ids + next, queries + (size_t)next * query_stride,
                                                query_stride, params + (per_request_params ? next : 0),
                                                per_request_params, rid.data() + next);
            if (rc < 0) return rc;
            for (int i = 0; i < rc; i++) pending.push_back(next + i);
            next += rc;
        }
        // collect completions: one lock and no CUDA call per pass; the kernel is
        // relaunched (if it left on idleness) at most once per pass
        {
            std::lock_guard<std::mutex> lock(sv->mu);
            for (size_t j = 0; j < pending.size();) {
                const int i = pending[j];
                int32_t h = 0, v = 0;
                const int rc = collect_locked(sv, (unsigned long long)rid[i],
                                              out_ids ? out_ids + (size_t)i * out_stride : tmp_ids.data(),
                                              out_dists ? out_dists + (size_t)i * out_stride : tmp_d.data(), &h, &v);
                if (rc < 0) return rc;
                if (rc == 1) {
                    latency_us[i] = now_us() - arrival_us[i];
                    if (hops) hops[i] = h;
                    if (visited) visited[i] = v;
                    pending[j] = pending.back();
                    pending.pop_back();
                    done++;
                } else {
                    j++;
                }
            }
            if (!pending.empty()) {
                cudaSetDevice(sv->device);
                const int lr = ensure_running(sv);
                if (lr != FALCON_OK) return lr;
            }
        }
        if (pending.empty() && next < n) {   // idle until the next arrival
            while (now_us() < arrival_us[next]) std::this_thread::yield();
        }
    }
    if (elapsed_us) *elapsed_us = now_us();
    return FALCON_OK;
}

int falcon_server_info_get(falcon_server *sv, falcon_server_info *info)
{
    if (!sv || !info) return set_error_code(FALCON_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    info->ring_entries = sv->cap;
    info->in_flight = sv->in_flight;
    info->submitted = (int64_t)sv->next_seq;
    info->kernel_launches = sv->launches;
    info->warps = sv->max_grid * 4;
    info->device_bytes = sv->device_bytes;
    info->concurrent_classes_max = sv->concurrent_max;
    return FALCON_OK;
}

int falcon_server_free(falcon_server *sv)
{
    if (!sv) return FALCON_OK;
    cudaSetDevice(sv->device);
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        const int32_t stop = 1;
        cudaMemcpy(&sv->d_ctl->stop, &stop, sizeof(stop), cudaMemcpyHostToDevice);
    }
    cudaStreamSynchronize(sv->cstream);
    cudaStreamSynchronize(sv->ystream);
    for (int c = 0; c < kServeClasses; c++) cudaStreamSynchronize(sv->kstream[c]);
    for (const falcon_index *ix : sv->indexes) index_server_ref(const_cast<falcon_index *>(ix), -1);
    free_server(sv);
    return FALCON_OK;
}

}  // extern "C"
