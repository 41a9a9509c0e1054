/*
 * ref_inter_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's own inter-query v1.3 HLS kernel code
 * (FPGA_multi_DDR/FPGA_inter_query_v1.3_longer_FIFO_alt_PR/src/*.hpp) as plain
 * C++ on the host, to pin the oracle restatement in falcon_oracle.c.
 *
 * Under `#pragma HLS dataflow` every process of the kernel runs concurrently;
 * in plain C++ the wrapper functions would call them one after another and
 * deadlock on the first blocking read.  This harness therefore wires the leaf
 * processes of one channel itself, each on its own std::thread, exactly as
 * per_channel_processing_wrapper.hpp:37-183, bloom_fetch_compute.hpp:9-133,
 * bloom_filter.hpp:207-317 and compute.hpp:285-376 connect them, and feeds
 * the channel's input streams the way read_queries/split_queries do for one
 * channel (DRAM_utils.hpp:7-116).
 *
 * The reference headers are compiled from a build-time copy with three
 * edits made by oracle/build_oracle.py: the two constructor-local arrays
 * that the HLS code points members at (priority_queue.hpp:20-22,
 * bloom_filter.hpp:25-27; dangling pointers in plain C++) become heap
 * allocations, `#define D` takes the dimension of the build variant, and the
 * result-queue hardware size is raised from 64 to 256 so ef up to 256 can be
 * cross-checked (slots past ef are inert in the reference's network).
 */
#include <cstdint>
#include <cstring>
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

extern "C" int ref_dim(void) { return D; }
extern "C" int ref_max_ef(void) { return hardware_result_queue_size; }
extern "C" int ref_max_cand_queue(void) { return hardware_candidate_queue_size; }
extern "C" int ref_max_bloom_bits(void) { return bloom_num_bucket_addr_bits; }

/*
 * queries:   nq rows of vec_AXI_num*16 floats (zero padded past D)
 * db_vectors: reference vector layout, one row = vec lines + 1 pad line
 * links:     reference link layout, one row = 1 header line + ceil(MD/16) lines
 */
/*
 * Built twice: from the v1.3 kernel sources (ref_inter_search), and with
 * FALCON_REF_TRACE from eval_trace_FPGA_inter_query_v1.3/src, whose
 * scheduler sends the popped candidate with its distance and whose
 * results_collection also writes the traversal trace (DRAM_utils.hpp:389-474):
 * trace_cand_d/n and trace_d/ids are flat streams, -1 before and -2 after each
 * query; each must hold, per query, 2 markers + hops (cand) or + visited (dist).
 */
#ifdef FALCON_REF_TRACE
typedef result_t top_cand_t;
extern "C" int ref_inter_search_trace(int nq, int ef, int cand_queue_size, int mc, int mg,
                                      int bloom_bits, unsigned hash_seed, int max_bloom_out_burst_size,
                                      int max_link_num_base, const int *entry_ids, const float *queries,
                                      const void *db_vectors, const void *links,
                                      int *out_id, float *out_dist, int *mem_debug,
                                      float *trace_cand_d, int *trace_cand_n, float *trace_d, int *trace_ids)
#else
typedef cand_t top_cand_t;
extern "C" int ref_inter_search(int nq, int ef, int cand_queue_size, int mc, int mg,
                                int bloom_bits, unsigned hash_seed, int max_bloom_out_burst_size,
                                int max_link_num_base, const int *entry_ids, const float *queries,
                                const void *db_vectors, const void *links,
                                int *out_id, float *out_dist, int *mem_debug)
#endif
{
    if (ef > hardware_result_queue_size || cand_queue_size > hardware_candidate_queue_size ||
        bloom_bits > bloom_num_bucket_addr_bits || bloom_bits < 10)
        return -1;
    const int vec_AXI_num = D % FLOAT_PER_AXI == 0 ? D / FLOAT_PER_AXI : D / FLOAT_PER_AXI + 1;
    ap_uint<512> *db = (ap_uint<512> *)db_vectors;
    const ap_uint<512> *lk = (const ap_uint<512> *)links;
    const ap_uint<32> seed = hash_seed;

    /* channel input streams */
    hls::stream<int> s_query_batch_size;
    hls::stream<ap_uint<512>> s_query_vectors_in;
    hls::stream<int> s_entry_point_ids;
    /* channel output streams */
    hls::stream<int> s_out_ids;
    hls::stream<float> s_out_dists;
    hls::stream<int> s_debug_signals;

    /* per_channel_processing_wrapper internals */
    hls::stream<int> s_finish_query_task_scheduler, s_finish_query_results_collection;
    hls::stream<ap_uint<512>> s_query_vectors;
    hls::stream<int> s_cand_batch_size;
    hls::stream<top_cand_t> s_top_candidates;
    hls::stream<int> s_num_inserted_candidates;
    hls::stream<result_t> s_inserted_candidates;
    hls::stream<int> s_num_valid_candidates_base_level_total;
    hls::stream<result_t> s_distances_base_level;
    hls::stream<float> s_largest_result_queue_elements;
    hls::stream<int> s_debug_num_vec_base_layer;
#ifdef FALCON_REF_TRACE
    constexpr int kQbsRep = 5;   // one more for the top-candidate replication
#else
    constexpr int kQbsRep = 4;
#endif
    hls::stream<int> s_qbs_rep[kQbsRep];
#ifdef FALCON_REF_TRACE
    hls::stream<top_cand_t> s_top_candidates_rep[2];
    hls::stream<int> s_finish_replicate_s_top_candidates;
#endif
    hls::stream<int> s_num_neighbors_base_level;
    hls::stream<cand_t> s_fetched_neighbor_ids;
    hls::stream<int> s_finish_query_fetch_neighbor_ids;
    hls::stream<int> s_finish_query_bloom_fetch_compute;

    /* bloom_fetch_compute internals */
    hls::stream<int> s_num_valid_candidates_burst;
    hls::stream<cand_t> s_valid_candidates;
    hls::stream<int> s_finish_bloom;
    hls::stream<int> bfc_qbs[4];
    hls::stream<int> s_nvcb_rep[2];
    hls::stream<cand_t> s_valid_candidates_rep[2];
    hls::stream<int> s_finish_query_replicate_candidates;
    hls::stream<ap_uint<512>> s_fetched_vectors;
    hls::stream<int> s_finish_query_fetch_vectors;

    /* run_bloom_filter internals */
    const int nh = bloom_num_hash_funs;
    hls::stream<int> rb_qbs[4 + bloom_num_hash_funs];
    hls::stream<int> s_num_candidates_replicated[bloom_num_hash_funs + 1];
    hls::stream<cand_t> s_all_candidates_replicated[bloom_num_hash_funs + 1];
    hls::stream<int> s_finish_replicate_candidates;
    hls::stream<int> s_finish_rep_rep[bloom_num_hash_funs];
    hls::stream<ap_uint<32>> s_hash_values_per_pe[bloom_num_hash_funs];
    hls::stream<int> s_finish_hash_per_pe[bloom_num_hash_funs];
    hls::stream<int> s_finish_hash;

    /* compute_distances internals */
    hls::stream<int> cd_qbs[4];
    hls::stream<int> s_fbs_rep[3];
    hls::stream<int> s_finish_replicate_s_fetch_batch_size;
    hls::stream<float> s_partial_distances;
    hls::stream<int> s_finish_query_fetch_sub_PE_A;
    hls::stream<float_pack_t> s_partial_distances_packed;
    hls::stream<int> s_finish_pack;

    BloomFilter<bloom_num_hash_funs, bloom_num_bucket_addr_bits> bloom(bloom_bits);

    std::vector<std::thread> th;
    th.emplace_back([&] { replicate_s_query_batch_size<kQbsRep>(s_query_batch_size, s_qbs_rep); });
#ifdef FALCON_REF_TRACE
    th.emplace_back([&] {
        replicate_s_control<2, top_cand_t>(s_qbs_rep[4], s_top_candidates, s_finish_query_task_scheduler,
                                           s_top_candidates_rep, s_finish_replicate_s_top_candidates);
    });
#endif
    th.emplace_back([&] {
        task_scheduler(cand_queue_size, mc, mg, s_qbs_rep[0], s_query_vectors_in, s_entry_point_ids,
                       s_num_inserted_candidates, s_inserted_candidates, s_largest_result_queue_elements,
                       s_debug_num_vec_base_layer, s_finish_query_results_collection, s_query_vectors,
                       s_cand_batch_size, s_top_candidates, s_debug_signals, s_finish_query_task_scheduler);
    });
    th.emplace_back([&] {
#ifdef FALCON_REF_TRACE
        fetch_neighbor_ids(max_link_num_base, lk, s_qbs_rep[1], s_top_candidates_rep[0],
                           s_finish_replicate_s_top_candidates, s_num_neighbors_base_level, s_fetched_neighbor_ids,
                           s_finish_query_fetch_neighbor_ids);
#else
        fetch_neighbor_ids(max_link_num_base, lk, s_qbs_rep[1], s_top_candidates, s_finish_query_task_scheduler,
                           s_num_neighbors_base_level, s_fetched_neighbor_ids, s_finish_query_fetch_neighbor_ids);
#endif
    });
    /* bloom_fetch_compute */
    th.emplace_back([&] { replicate_s_query_batch_size<4>(s_qbs_rep[2], bfc_qbs); });
    /* run_bloom_filter */
    th.emplace_back([&] { replicate_s_query_batch_size<4 + bloom_num_hash_funs>(bfc_qbs[0], rb_qbs); });
    th.emplace_back([&] {
        replicate_s_read_iter_and_s_data<bloom_num_hash_funs + 1, cand_t>(
            rb_qbs[0], s_num_neighbors_base_level, s_fetched_neighbor_ids, s_finish_query_fetch_neighbor_ids,
            s_num_candidates_replicated, s_all_candidates_replicated, s_finish_replicate_candidates);
    });
    th.emplace_back([&] {
        replicate_s_finish<bloom_num_hash_funs>(rb_qbs[1], s_finish_replicate_candidates, s_finish_rep_rep);
    });
    for (int pe = 0; pe < nh; pe++) {
        th.emplace_back([&, pe] {
            bloom.stream_hash(seed + pe, rb_qbs[2 + pe], s_num_candidates_replicated[pe],
                              s_all_candidates_replicated[pe], s_finish_rep_rep[pe],
                              s_hash_values_per_pe[pe], s_finish_hash_per_pe[pe]);
        });
    }
    th.emplace_back([&] {
        gather_s_finish<bloom_num_hash_funs>(rb_qbs[2 + bloom_num_hash_funs], s_finish_hash_per_pe, s_finish_hash);
    });
    th.emplace_back([&] {
        bloom.check_update(max_bloom_out_burst_size, rb_qbs[3 + bloom_num_hash_funs],
                           s_num_candidates_replicated[bloom_num_hash_funs],
                           s_all_candidates_replicated[bloom_num_hash_funs], s_hash_values_per_pe, s_finish_hash,
                           s_num_valid_candidates_burst, s_num_valid_candidates_base_level_total,
                           s_valid_candidates, s_finish_bloom);
    });
    th.emplace_back([&] {
        replicate_s_read_iter_and_s_data<2, cand_t>(bfc_qbs[1], s_num_valid_candidates_burst, s_valid_candidates,
                                                     s_finish_bloom, s_nvcb_rep, s_valid_candidates_rep,
                                                     s_finish_query_replicate_candidates);
    });
    th.emplace_back([&] {
        fetch_vectors(db, bfc_qbs[2], s_nvcb_rep[0], s_valid_candidates_rep[0], s_finish_query_replicate_candidates,
                      s_fetched_vectors, s_finish_query_fetch_vectors);
    });
    /* compute_distances */
    th.emplace_back([&] { replicate_s_query_batch_size<4>(bfc_qbs[3], cd_qbs); });
    th.emplace_back([&] {
        replicate_s_control<3, int>(cd_qbs[0], s_nvcb_rep[1], s_finish_query_fetch_vectors, s_fbs_rep,
                                    s_finish_replicate_s_fetch_batch_size);
    });
    th.emplace_back([&] {
        compute_distances_sub_PE_A(cd_qbs[1], s_query_vectors, s_fbs_rep[0], s_fetched_vectors,
                                   s_finish_replicate_s_fetch_batch_size, s_partial_distances,
                                   s_finish_query_fetch_sub_PE_A);
    });
    th.emplace_back([&] {
        compute_distances_sub_PE_pack_partial_distances(cd_qbs[2], s_fbs_rep[1], s_partial_distances,
                                                        s_finish_query_fetch_sub_PE_A, s_partial_distances_packed,
                                                        s_finish_pack);
    });
    th.emplace_back([&] {
        compute_distances_sub_PE_B(cd_qbs[3], s_fbs_rep[2], s_partial_distances_packed, s_valid_candidates_rep[1],
                                   s_finish_pack, s_distances_base_level, s_finish_query_bloom_fetch_compute);
    });
    th.emplace_back([&] {
#ifdef FALCON_REF_TRACE
        results_collection(ef, s_qbs_rep[3], s_cand_batch_size, s_top_candidates_rep[1],
                           s_num_valid_candidates_base_level_total, s_distances_base_level,
                           s_finish_query_bloom_fetch_compute, trace_cand_d, trace_cand_n, trace_d, trace_ids,
                           s_inserted_candidates, s_num_inserted_candidates, s_largest_result_queue_elements,
                           s_debug_num_vec_base_layer, s_finish_query_results_collection, s_out_ids, s_out_dists);
#else
        results_collection(ef, s_qbs_rep[3], s_cand_batch_size, s_num_valid_candidates_base_level_total,
                           s_distances_base_level, s_finish_query_bloom_fetch_compute, s_inserted_candidates,
                           s_num_inserted_candidates, s_largest_result_queue_elements, s_debug_num_vec_base_layer,
                           s_finish_query_results_collection, s_out_ids, s_out_dists);
#endif
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
    /* collect (write_results, one channel) */
    for (int q = 0; q < nq; q++) {
        for (int i = 0; i < ef; i++) out_id[(size_t)q * ef + i] = s_out_ids.read();
        for (int i = 0; i < ef; i++) out_dist[(size_t)q * ef + i] = s_out_dists.read();
        for (int i = 0; i < debug_size; i++) mem_debug[(size_t)q * debug_size + i] = s_debug_signals.read();
    }
    s_query_batch_size.write(-1);
    for (auto &t : th) t.join();
    return 0;
}
