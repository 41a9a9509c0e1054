/*
 * hnswlib_ref.cpp -- TEST / BASELINE INFRASTRUCTURE ONLY.
 *
 * A C-ABI wrapper around the reference's vendored header-only hnswlib
 * (networked_FPGA/CPU_programs_oldest/hnswlib/*.h), compiled from those
 * headers where they lie.  Used for three things, never by the product:
 *   - building the seeded HNSW graphs the reference's own index scripts would
 *     build (HierarchicalNSW(M, ef_construction, random_seed), points added in
 *     id order on one thread so the graph is deterministic;
 *     hnswalg.h:27-75, 988-1111);
 *   - exporting the base layer (hnswalg.h:371-376) so the same graph can be
 *     loaded into the GPU index and the oracle;
 *   - the reference CPU search baseline: searchKnn with setEf(ef) over
 *     std::threads (hnswalg.h:1115-1160, 241-325), on any graph loaded through
 *     hnsw_from_graph (base layer, given entry point) and, for HNSW graphs,
 *     hnsw_set_upper (the upper layers searchKnn descends first);
 *   - checking the hnswlib file reader (saveIndex, hnswalg.h:588-616, and the
 *     upper layers read through get_linklist) and the upper-layer descent
 *     (searchKnn's greedy part, hnswalg.h:514-541, with hnswlib's distance).
 */
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "hnswlib.h"
#include "hnswalg.h"
#include "space_l2.h"

struct hnsw_handle {
    hnswlib::L2Space *space;
    hnswlib::HierarchicalNSW<float> *index;
};

extern "C" void *hnsw_build(int64_t n, int dim, int M, int ef_construction, int seed, const float *vectors)
{
    hnsw_handle *h = new hnsw_handle;
    h->space = new hnswlib::L2Space(dim);
    h->index = new hnswlib::HierarchicalNSW<float>(h->space, (size_t)n, (size_t)M, (size_t)ef_construction,
                                                   (size_t)seed);
    for (int64_t i = 0; i < n; i++) h->index->addPoint((const void *)(vectors + i * dim), (size_t)i);
    return h;
}

/* Single-layer index over an existing graph: level-0 rows `links`
   (n x max_degree, the first counts[i] entries valid), entry point `entry`. */
extern "C" void *hnsw_from_graph(int64_t n, int dim, int max_degree, const float *vectors,
                                 const int32_t *links, const int32_t *counts, int entry)
{
    hnsw_handle *h = new hnsw_handle;
    h->space = new hnswlib::L2Space(dim);
    auto *ix = new hnswlib::HierarchicalNSW<float>(h->space, (size_t)n, (size_t)(max_degree / 2), 100, 0);
    h->index = ix;
    for (int64_t i = 0; i < n; i++) {
        char *base = ix->data_level0_memory_ + i * ix->size_data_per_element_;
        std::memcpy(base + ix->offsetData_, vectors + i * dim, sizeof(float) * dim);
        size_t label = (size_t)i;
        std::memcpy(base + ix->label_offset_, &label, sizeof(size_t));
        hnswlib::linklistsizeint *ll = ix->get_linklist0((hnswlib::tableint)i);
        int c = counts[i];
        ix->setListCount(ll, (unsigned short)c);
        hnswlib::tableint *dst = (hnswlib::tableint *)(ll + 1);
        for (int j = 0; j < c; j++) dst[j] = (hnswlib::tableint)links[i * max_degree + j];
        ix->element_levels_[i] = 0;
        ix->label_lookup_[label] = (hnswlib::tableint)i;
    }
    ix->cur_element_count = (size_t)n;
    ix->enterpoint_node_ = (hnswlib::tableint)entry;
    ix->maxlevel_ = 0;
    return h;
}

/* Upper layers for an index made by hnsw_from_graph, in hnswlib's own
   arrangement (linkLists_ holds element_levels_[v] rows of maxM_ ids per
   node, hnswalg.h:371-384): node v's level-l list (1 <= l <= levels[v]) is
   rows[(row_start[v] + l - 1) * row_stride ..], the count at [0] and the ids
   from [ids_offset].  maxlevel_ and enterpoint_node_ are set as given, so
   searchKnn descends them as it does an index it built itself.  Returns -1
   when a list is longer than maxM_. */
extern "C" int hnsw_set_upper(void *hp, const int32_t *levels, const int64_t *row_start, const int32_t *rows,
                              int64_t row_stride, int ids_offset, int max_level, int entry)
{
    hnsw_handle *h = (hnsw_handle *)hp;
    auto *ix = h->index;
    for (size_t i = 0; i < ix->cur_element_count; i++) {
        const int lv = levels[i];
        ix->element_levels_[i] = lv;
        if (lv <= 0) continue;
        ix->linkLists_[i] = (char *)calloc((size_t)lv, ix->size_links_per_element_);
        if (!ix->linkLists_[i]) return -1;
        for (int l = 1; l <= lv; l++) {
            const int32_t *row = rows + (row_start[i] + l - 1) * row_stride;
            const int c = row[0];
            if (c < 0 || (size_t)c > ix->maxM_) return -1;
            hnswlib::linklistsizeint *ll = ix->get_linklist((hnswlib::tableint)i, l);
            ix->setListCount(ll, (unsigned short)c);
            hnswlib::tableint *dst = (hnswlib::tableint *)(ll + 1);
            for (int j = 0; j < c; j++) dst[j] = (hnswlib::tableint)row[ids_offset + j];
        }
    }
    ix->maxlevel_ = max_level;
    ix->enterpoint_node_ = (hnswlib::tableint)entry;
    return 0;
}

extern "C" int hnsw_info(void *hp, int64_t *n, int *max_degree, int *entry, int *max_level)
{
    hnsw_handle *h = (hnsw_handle *)hp;
    *n = (int64_t)h->index->cur_element_count;
    *max_degree = (int)h->index->maxM0_;
    *entry = (int)h->index->enterpoint_node_;
    *max_level = h->index->maxlevel_;
    return 0;
}

/* Base layer export: links n x maxM0 (-1 padded), counts n, labels n. */
extern "C" int hnsw_export_level0(void *hp, int32_t *links, int32_t *counts, int32_t *labels)
{
    hnsw_handle *h = (hnsw_handle *)hp;
    auto *ix = h->index;
    const int md = (int)ix->maxM0_;
    for (size_t i = 0; i < ix->cur_element_count; i++) {
        hnswlib::linklistsizeint *ll = ix->get_linklist0((hnswlib::tableint)i);
        int c = ix->getListCount(ll);
        const hnswlib::tableint *src = (const hnswlib::tableint *)(ll + 1);
        counts[i] = c;
        for (int j = 0; j < md; j++) links[i * md + j] = (j < c) ? (int32_t)src[j] : -1;
        labels[i] = (int32_t)ix->getExternalLabel((hnswlib::tableint)i);
    }
    return 0;
}

/* Batch searchKnn over `threads` std::threads; results best-first. */
extern "C" int hnsw_search(void *hp, const float *queries, int64_t nq, int dim, int k, int ef, int threads,
                           int64_t *out_labels, float *out_dists)
{
    hnsw_handle *h = (hnsw_handle *)hp;
    h->index->setEf((size_t)ef);
    std::atomic<int64_t> next(0);
    if (threads < 1) threads = 1;
    auto work = [&]() {
        for (;;) {
            int64_t q = next.fetch_add(1);
            if (q >= nq) break;
            auto res = h->index->searchKnn((const void *)(queries + q * dim), (size_t)k);
            int64_t m = (int64_t)res.size();
            for (int64_t i = k - 1; i >= 0; i--) {
                if (i < m) {
                    out_labels[q * k + i] = (int64_t)res.top().second;
                    out_dists[q * k + i] = res.top().first;
                    res.pop();
                } else {
                    out_labels[q * k + i] = -1;
                    out_dists[q * k + i] = 1e20f;
                }
            }
        }
    };
    std::vector<std::thread> th;
    for (int t = 0; t < threads; t++) th.emplace_back(work);
    for (auto &t : th) t.join();
    return 0;
}

/* hnswlib's own saveIndex (hnswalg.h:588-616). */
extern "C" int hnsw_save(void *hp, const char *path)
{
    hnsw_handle *h = (hnsw_handle *)hp;
    h->index->saveIndex(std::string(path));
    return 0;
}

/* Upper layers: number of level rows (sum of element levels) and maxM. */
extern "C" int64_t hnsw_upper_rows(void *hp, int *max_m)
{
    hnsw_handle *h = (hnsw_handle *)hp;
    auto *ix = h->index;
    int64_t rows = 0;
    for (size_t i = 0; i < ix->cur_element_count; i++) rows += ix->element_levels_[i];
    *max_m = (int)ix->maxM_;
    return rows;
}

/* Export levels [n], row_start [n] and rows [num_rows x (1 + maxM)] (count,
   ids) read through hnswlib's own accessors (get_linklist, getListCount). */
extern "C" int hnsw_export_upper(void *hp, int32_t *levels, int64_t *row_start, int32_t *rows)
{
    hnsw_handle *h = (hnsw_handle *)hp;
    auto *ix = h->index;
    const int m = (int)ix->maxM_;
    int64_t r = 0;
    for (size_t i = 0; i < ix->cur_element_count; i++) {
        const int lv = ix->element_levels_[i];
        levels[i] = lv;
        row_start[i] = r;
        for (int l = 1; l <= lv; l++, r++) {
            hnswlib::linklistsizeint *ll = ix->get_linklist((hnswlib::tableint)i, l);
            const int c = ix->getListCount(ll);
            const hnswlib::tableint *src = (const hnswlib::tableint *)(ll + 1);
            rows[r * (1 + m)] = c;
            for (int j = 0; j < m; j++) rows[r * (1 + m) + 1 + j] = (j < c) ? (int32_t)src[j] : 0;
        }
    }
    return 0;
}

/* The upper-layer part of searchKnn (hnswalg.h:514-541) with hnswlib's own
   distance function: the base-layer entry point of each query. */
extern "C" int hnsw_descend(void *hp, const float *queries, int64_t nq, int dim, int32_t *out_entry)
{
    hnsw_handle *h = (hnsw_handle *)hp;
    auto *ix = h->index;
    for (int64_t q = 0; q < nq; q++) {
        const void *qd = (const void *)(queries + q * dim);
        hnswlib::tableint cur = ix->enterpoint_node_;
        float curdist = ix->fstdistfunc_(qd, ix->getDataByInternalId(cur), ix->dist_func_param_);
        for (int level = ix->maxlevel_; level > 0; level--) {
            bool changed = true;
            while (changed) {
                changed = false;
                hnswlib::linklistsizeint *ll = ix->get_linklist(cur, level);
                const int size = ix->getListCount(ll);
                const hnswlib::tableint *datal = (const hnswlib::tableint *)(ll + 1);
                for (int i = 0; i < size; i++) {
                    const float d = ix->fstdistfunc_(qd, ix->getDataByInternalId(datal[i]), ix->dist_func_param_);
                    if (d < curdist) {
                        curdist = d;
                        cur = datal[i];
                        changed = true;
                    }
                }
            }
        }
        out_entry[q] = (int32_t)cur;
    }
    return 0;
}

extern "C" void hnsw_free(void *hp)
{
    hnsw_handle *h = (hnsw_handle *)hp;
    delete h->index;
    delete h->space;
    delete h;
}
