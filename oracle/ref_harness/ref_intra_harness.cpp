/*
 * ref_intra_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's own intra-query v1.5 HLS kernel code
 * (FPGA_multi_DDR/FPGA_intra_query_v1.5_support_batching_longer_FIFO/src/*.hpp)
 * as plain C++ on the host, to pin the oracle's intra-query restatement in
 * falcon_oracle.c.
 *
 * The kernel's top level (vadd.cpp:167-1020) is a `#pragma HLS dataflow`
 * region: every process runs concurrently.  This harness wires the leaf
 * processes the way vadd.cpp and the wrappers it calls connect them
 * (bloom_fetch_compute.hpp:9-133 per channel, run_bloom_filter in
 * bloom_filter.hpp:207-317, compute_distances in compute.hpp:285-376), each on
 * its own std::thread, and feeds/collects the streams read_queries and
 * write_results would (DRAM_utils.hpp:7-125).  N_CHANNEL channels: node i
 * lives in row i >> CHANNEL_ADDR_BITS of channel i & (N_CHANNEL - 1), the
 * layout the reference's index writers produce (hnsw.py:324-335); the harness
 * splits the caller's node-ordered arrays that way.
 *
 * gather_distances_from_channels (utils.hpp:497-569) forwards channels in the
 * order their results become ready, which depends on thread timing here as
 * it does on the FPGA.  Within a group, the merge order matters only for
 * equal distances (insertion age breaks ties), so on data without repeated
 * distances the results are schedule independent.
 *
 * The reference headers are compiled from a build-time copy with the edits
 * oracle/build_oracle.py lists (constructor-local arrays to heap arrays,
 * `#define D` and `#define N_CHANNEL` set for the variant, the result-queue
 * hardware size raised from 64 to 256).
 */
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "constants.hpp"
#include "types.hpp"
#include "utils.hpp"
#include "priority_queue.hpp"
#include "bloom_filter.hpp"
#include "compute.hpp"
#include "DRAM_utils.hpp"
#include "scheduler.hpp"

extern "C" int ref_intra_dim(void) { return D; }
extern "C" int ref_intra_channels(void) { return N_CHANNEL; }
extern "C" int ref_intra_max_bloom_bits(void) { return bloom_num_bucket_addr_bits; }

namespace {

typedef BloomFilter<bloom_num_hash_funs, bloom_num_bucket_addr_bits> bloom_t;

// The streams of one channel's bloom_fetch_compute (bloom_fetch_compute.hpp).
struct Channel {
    // bloom_fetch_compute
    hls::stream<int> bfc_qbs[4];
    hls::stream<int> s_num_valid_candidates_burst;
    hls::stream<cand_t> s_valid_candidates;
    hls::stream<int> s_finish_bloom;
    hls::stream<int> s_nvcb_rep[2];
    hls::stream<cand_t> s_valid_candidates_rep[2];
    hls::stream<int> s_finish_query_replicate_candidates;
    hls::stream<ap_uint<512>> s_fetched_vectors;
    hls::stream<int> s_finish_query_fetch_vectors;
    // run_bloom_filter
    hls::stream<int> rb_qbs[4 + bloom_num_hash_funs];
    hls::stream<int> s_num_candidates_replicated[bloom_num_hash_funs + 1];
    hls::stream<cand_t> s_all_candidates_replicated[bloom_num_hash_funs + 1];
    hls::stream<int> s_finish_replicate_candidates;
    hls::stream<int> s_finish_rep_rep[bloom_num_hash_funs];
    hls::stream<ap_uint<32>> s_hash_values_per_pe[bloom_num_hash_funs];
    hls::stream<int> s_finish_hash_per_pe[bloom_num_hash_funs];
    hls::stream<int> s_finish_hash;
    // compute_distances
    hls::stream<int> cd_qbs[4];
    hls::stream<int> s_fbs_rep[3];
    hls::stream<int> s_finish_replicate_s_fetch_batch_size;
    hls::stream<float> s_partial_distances;
    hls::stream<int> s_finish_query_fetch_sub_PE_A;
    hls::stream<float_pack_t> s_partial_distances_packed;
    hls::stream<int> s_finish_pack;
    // filter_computed_distances
    hls::stream<int> s_num_filtered;
    hls::stream<result_t> s_distances_filtered;
    std::unique_ptr<bloom_t> bloom;
    std::vector<ap_uint<512>> db;      // this channel's vector rows
    std::vector<ap_uint<512>> links;   // this channel's link rows
};

}  // namespace

/*
 * queries:    nq rows of vec_AXI_num*16 floats (zero padded past D)
 * db_vectors: node-ordered reference vector rows (vec lines + 1 pad line)
 * links:      node-ordered reference link rows (1 header line + ceil(MD/16) lines)
 * out_id/out_dist: nq x ef; mem_debug: nq x debug_size (the base-layer hops)
 */
extern "C" int ref_intra_search(int nq, int ef, int cand_queue_size, int mc, int mg, int bloom_bits,
                                unsigned hash_seed, int max_bloom_out_burst_size, int max_link_num_base, int64_t n,
                                const int *entry_ids, const float *queries, const void *db_vectors,
                                const void *links, int *out_id, float *out_dist, int *mem_debug)
{
    if (ef > hardware_result_queue_size || cand_queue_size > hardware_candidate_queue_size ||
        bloom_bits > bloom_num_bucket_addr_bits || bloom_bits < 10)
        return -1;
    const int vec_AXI_num = D % FLOAT_PER_AXI == 0 ? D / FLOAT_PER_AXI : D / FLOAT_PER_AXI + 1;
    const int vec_rows = vec_AXI_num + 1;
    const int link_rows = max_link_num_base % INT_PER_AXI == 0 ? 1 + max_link_num_base / INT_PER_AXI
                                                                : 2 + max_link_num_base / INT_PER_AXI;
    const ap_uint<512> *db_all = (const ap_uint<512> *)db_vectors;
    const ap_uint<512> *lk_all = (const ap_uint<512> *)links;
    const ap_uint<32> seed = hash_seed;
    constexpr int N = N_CHANNEL;
    constexpr int nh = bloom_num_hash_funs;

    Channel ch[N];
    for (int c = 0; c < N; c++) {
        const int64_t rows = (n - c + N - 1) / N;
        ch[c].db.resize((size_t)(rows > 0 ? rows : 1) * vec_rows);
        ch[c].links.resize((size_t)(rows > 0 ? rows : 1) * link_rows);
        for (int64_t r = 0; r < rows; r++) {
            const int64_t node = r * N + c;
            for (int j = 0; j < vec_rows; j++) ch[c].db[r * vec_rows + j] = db_all[node * vec_rows + j];
            for (int j = 0; j < link_rows; j++) ch[c].links[r * link_rows + j] = lk_all[node * link_rows + j];
        }
        ch[c].bloom.reset(new bloom_t(bloom_bits));
    }

    /* top-level streams (vadd.cpp) */
    hls::stream<int> s_query_batch_size;
    hls::stream<ap_uint<512>> s_query_vectors_in;
    hls::stream<int> s_entry_point_ids;
    hls::stream<int> s_finish_query_task_scheduler;
    hls::stream<int> s_finish_query_results_collection;
    hls::stream<ap_uint<512>> s_query_vectors_replicated[N];
    hls::stream<int> s_cand_batch_size;
    hls::stream<cand_t> s_top_candidates;
    hls::stream<int> s_num_inserted_candidates;
    hls::stream<result_t> s_inserted_candidates;
    hls::stream<int> s_num_valid_candidates_base_level_total;
    hls::stream<result_t> s_distances_base_level;
    hls::stream<float> s_largest_result_queue_elements;
    hls::stream<int> s_debug_signals;
    hls::stream<float> s_largest_rep[1 + N];
    hls::stream<int> s_finish_query_replicate_s_largest_result_queue_elements;
    constexpr int kQbs = 2 * N + 9;
    hls::stream<int> s_qbs[kQbs];
    hls::stream<ap_uint<512>> s_neighbor_ids_raw;
    hls::stream<int> s_finish_query_fetch_neighbor_ids;
    hls::stream<int> s_num_neighbors_per_channel[N];
    hls::stream<cand_t> s_fetched_neighbor_ids_per_channel[N];
    hls::stream<int> s_finish_query_split_tasks_to_channels;
    hls::stream<int> s_finish_split_rep[N];
    hls::stream<int> s_num_valid_total_per_channel[N];
    hls::stream<result_t> s_distances_per_channel[N];
    hls::stream<int> s_finish_bfc_per_channel[N];
    hls::stream<int> s_num_filtered[N];
    hls::stream<result_t> s_distances_filtered[N];
    hls::stream<int> s_finish_filter_per_channel[N];
    hls::stream<int> s_finish_query_filter_computed_distances;
    hls::stream<int> s_finish_gather_distances_from_channels;
    hls::stream<int> s_out_ids;
    hls::stream<float> s_out_dists;

    std::vector<std::thread> th;
    th.emplace_back([&] { replicate_s_query_batch_size<kQbs>(s_query_batch_size, s_qbs); });
    th.emplace_back([&] {
        task_scheduler(cand_queue_size, mc, mg, s_qbs[0], s_query_vectors_in, s_entry_point_ids,
                       s_num_inserted_candidates, s_inserted_candidates, s_largest_rep[0],
                       s_finish_query_replicate_s_largest_result_queue_elements, s_query_vectors_replicated,
                       s_cand_batch_size, s_top_candidates, s_debug_signals, s_finish_query_task_scheduler);
    });
    th.emplace_back([&] {
        fetch_neighbor_ids(max_link_num_base, ch[0].links.data(),
#if N_CHANNEL >= 2
                           ch[1].links.data(),
#endif
#if N_CHANNEL >= 4
                           ch[2].links.data(), ch[3].links.data(),
#endif
#if N_CHANNEL >= 8
                           ch[4].links.data(), ch[5].links.data(), ch[6].links.data(), ch[7].links.data(),
#endif
                           s_qbs[1], s_top_candidates, s_finish_query_task_scheduler, s_neighbor_ids_raw,
                           s_finish_query_fetch_neighbor_ids);
    });
    th.emplace_back([&] {
        split_tasks_to_channels(max_link_num_base, s_qbs[2], s_cand_batch_size, s_neighbor_ids_raw,
                                s_finish_query_fetch_neighbor_ids, s_num_neighbors_per_channel,
                                s_fetched_neighbor_ids_per_channel, s_finish_query_split_tasks_to_channels);
    });
    th.emplace_back([&] { replicate_s_finish<N>(s_qbs[3], s_finish_query_split_tasks_to_channels, s_finish_split_rep); });
    for (int c = 0; c < N; c++) {
        /* bloom_fetch_compute (bloom_fetch_compute.hpp:9-133) */
        th.emplace_back([&, c] {
            Channel &C = ch[c]; replicate_s_query_batch_size<4>(s_qbs[4 + c], C.bfc_qbs); });
        /* run_bloom_filter (bloom_filter.hpp:207-317) */
        th.emplace_back([&, c] {
            Channel &C = ch[c]; replicate_s_query_batch_size<4 + nh>(C.bfc_qbs[0], C.rb_qbs); });
        th.emplace_back([&, c] {
            Channel &C = ch[c];
            replicate_s_read_iter_and_s_data<nh + 1, cand_t>(
                C.rb_qbs[0], s_num_neighbors_per_channel[c], s_fetched_neighbor_ids_per_channel[c],
                s_finish_split_rep[c], C.s_num_candidates_replicated, C.s_all_candidates_replicated,
                C.s_finish_replicate_candidates);
        });
        th.emplace_back([&, c] {
            Channel &C = ch[c]; replicate_s_finish<nh>(C.rb_qbs[1], C.s_finish_replicate_candidates, C.s_finish_rep_rep); });
        for (int pe = 0; pe < nh; pe++) {
            th.emplace_back([&, c, pe] {
                Channel &C = ch[c];
                C.bloom->stream_hash(seed + pe, C.rb_qbs[2 + pe], C.s_num_candidates_replicated[pe],
                                     C.s_all_candidates_replicated[pe], C.s_finish_rep_rep[pe],
                                     C.s_hash_values_per_pe[pe], C.s_finish_hash_per_pe[pe]);
            });
        }
        th.emplace_back([&, c] {
            Channel &C = ch[c]; gather_s_finish<nh>(C.rb_qbs[2 + nh], C.s_finish_hash_per_pe, C.s_finish_hash); });
        th.emplace_back([&, c] {
            Channel &C = ch[c];
            C.bloom->check_update(max_bloom_out_burst_size, C.rb_qbs[3 + nh], C.s_num_candidates_replicated[nh],
                                  C.s_all_candidates_replicated[nh], C.s_hash_values_per_pe, C.s_finish_hash,
                                  C.s_num_valid_candidates_burst, s_num_valid_total_per_channel[c],
                                  C.s_valid_candidates, C.s_finish_bloom);
        });
        th.emplace_back([&, c] {
            Channel &C = ch[c];
            replicate_s_read_iter_and_s_data<2, cand_t>(C.bfc_qbs[1], C.s_num_valid_candidates_burst,
                                                         C.s_valid_candidates, C.s_finish_bloom, C.s_nvcb_rep,
                                                         C.s_valid_candidates_rep,
                                                         C.s_finish_query_replicate_candidates);
        });
        th.emplace_back([&, c] {
            Channel &C = ch[c];
            fetch_vectors(C.db.data(), C.bfc_qbs[2], C.s_nvcb_rep[0], C.s_valid_candidates_rep[0],
                          C.s_finish_query_replicate_candidates, C.s_fetched_vectors, C.s_finish_query_fetch_vectors);
        });
        /* compute_distances (compute.hpp:285-376) */
        th.emplace_back([&, c] {
            Channel &C = ch[c]; replicate_s_query_batch_size<4>(C.bfc_qbs[3], C.cd_qbs); });
        th.emplace_back([&, c] {
            Channel &C = ch[c];
            replicate_s_control<3, int>(C.cd_qbs[0], C.s_nvcb_rep[1], C.s_finish_query_fetch_vectors, C.s_fbs_rep,
                                        C.s_finish_replicate_s_fetch_batch_size);
        });
        th.emplace_back([&, c] {
            Channel &C = ch[c];
            compute_distances_sub_PE_A(C.cd_qbs[1], s_query_vectors_replicated[c], C.s_fbs_rep[0], C.s_fetched_vectors,
                                       C.s_finish_replicate_s_fetch_batch_size, C.s_partial_distances,
                                       C.s_finish_query_fetch_sub_PE_A);
        });
        th.emplace_back([&, c] {
            Channel &C = ch[c];
            compute_distances_sub_PE_pack_partial_distances(C.cd_qbs[2], C.s_fbs_rep[1], C.s_partial_distances,
                                                            C.s_finish_query_fetch_sub_PE_A,
                                                            C.s_partial_distances_packed, C.s_finish_pack);
        });
        th.emplace_back([&, c] {
            Channel &C = ch[c];
            compute_distances_sub_PE_B(C.cd_qbs[3], C.s_fbs_rep[2], C.s_partial_distances_packed,
                                       C.s_valid_candidates_rep[1], C.s_finish_pack, s_distances_per_channel[c],
                                       s_finish_bfc_per_channel[c]);
        });
        /* filter_computed_distances (utils.hpp:277-347), vadd.cpp per channel */
        th.emplace_back([&, c] {
            Channel &C = ch[c];
            filter_computed_distances(s_qbs[N + 4 + c], s_num_valid_total_per_channel[c], s_largest_rep[1 + c],
                                      s_distances_per_channel[c], s_finish_bfc_per_channel[c], s_num_filtered[c],
                                      s_distances_filtered[c], s_finish_filter_per_channel[c]);
        });
    }
    th.emplace_back([&] {
        gather_s_finish<N>(s_qbs[2 * N + 4], s_finish_filter_per_channel, s_finish_query_filter_computed_distances);
    });
    th.emplace_back([&] {
        gather_distances_from_channels(s_qbs[2 * N + 5], s_num_filtered, s_distances_filtered,
                                       s_finish_query_filter_computed_distances,
                                       s_num_valid_candidates_base_level_total, s_distances_base_level,
                                       s_finish_gather_distances_from_channels);
    });
    th.emplace_back([&] {
        results_collection(ef, s_qbs[2 * N + 6], s_num_valid_candidates_base_level_total, s_distances_base_level,
                           s_finish_gather_distances_from_channels, s_inserted_candidates, s_num_inserted_candidates,
                           s_largest_result_queue_elements, s_finish_query_results_collection, s_out_ids,
                           s_out_dists);
    });
    th.emplace_back([&] {
        replicate_s_control<1 + N, float>(s_qbs[2 * N + 7], s_largest_result_queue_elements,
                                          s_finish_query_results_collection, s_largest_rep,
                                          s_finish_query_replicate_s_largest_result_queue_elements);
    });

    /* feed one batch of nq queries, then the stop token (read_queries) */
    s_query_batch_size.write(nq);
    for (int q = 0; q < nq; q++) {
        for (int j = 0; j < vec_AXI_num; j++) {
            ap_uint<512> line;
            std::memcpy(line.w, queries + ((size_t)q * vec_AXI_num + j) * 16, 64);
            s_query_vectors_in.write(line);
        }
        s_entry_point_ids.write(entry_ids[q]);
    }
    /* collect (write_results) */
    for (int q = 0; q < nq; q++) {
        for (int i = 0; i < ef; i++) out_id[(size_t)q * ef + i] = s_out_ids.read();
        for (int i = 0; i < ef; i++) out_dist[(size_t)q * ef + i] = s_out_dists.read();
        for (int i = 0; i < debug_size; i++) mem_debug[(size_t)q * debug_size + i] = s_debug_signals.read();
    }
    s_query_batch_size.write(-1);
    for (auto &t : th) t.join();
    return 0;
}
