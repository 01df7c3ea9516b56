/* CPU oracle for the Vamana hot path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference algorithm (ParlayANN Vamana as
 * forked by distributed_diskann), used by tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg as the checker.  The product library never
 * links, loads or calls it.  Parity is pinned by tests/test_oracle_pin.py
 * against outputs of the reference's own sources (oracle/_ref/ref_harness)
 * committed as golden fixtures under tests/golden/.
 *
 * dtype: 0 = float32, 1 = int8, 2 = uint8.   metric: 0 = L2, 1 = MIPS.
 * Points are row-major with an arbitrary row stride in bytes.
 * Graphs use the reference's in-memory layout: n rows of (R+1) uint32,
 * row[0] = degree (include/utils/graph.h:126-128, 202). */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

float ddo_distance(int dtype, int metric, const void* a, const void* b, uint32_t d);

/* Batched Vamana build with the BSP schedule (src/bsp_index.hpp:141-434) or,
 * with knn_mode != 0, knn_index::build_index (include/index.h:125-137:
 * max_fraction 1.0, optional two_pass, final per-row distance sort).
 * stats_out (may be NULL): [0] rounds, [1] sum visited, [2] sum dist_cmps,
 * [3] reverse groups, [4] reverse prunes, [5] sum prune candidates. */
int ddo_build(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
              uint64_t stride, uint32_t R, uint32_t L, double alpha, double xita,
              uint64_t max_build, uint32_t start, int two_pass, int knn_mode,
              int nthreads, uint32_t* graph_out, uint64_t* stats_out);

/* One rank's steps of a round of the build spread over `world` ranks, every
 * rank holding the whole graph (src/bsp_index.hpp:247-407): new out-lists of
 * the batch slice [lo, hi) (rows_out, (hi-lo) x (R+1)); update_neighbors of
 * the batch [floor, ceiling) from batch_rows, then the reverse edges of the
 * targets t with t % world == rank, whose ids / new rows (ascending ids) go to
 * ids_out / rows_out (room for cap rows; *count = their number); and the
 * application of rows received from other ranks. */
int ddo_shard_search_prune(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
                           uint64_t stride, const uint32_t* graph, uint32_t R, uint32_t L,
                           double alpha, uint32_t start, uint64_t lo, uint64_t hi, int nthreads,
                           uint32_t* rows_out);
int ddo_shard_apply_reverse(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
                            uint64_t stride, uint32_t* graph, uint32_t R, double alpha,
                            uint64_t floor_, uint64_t ceiling, const uint32_t* batch_rows,
                            uint32_t rank, uint32_t world, int nthreads, uint32_t* ids_out,
                            uint32_t* rows_out, uint64_t cap, uint64_t* count);
int ddo_shard_set_rows(uint32_t* graph, uint64_t n, uint32_t R, const uint32_t* ids,
                       const uint32_t* rows, uint64_t count);

/* One beam_search (include/utils/beamSearch.h:51-184). graph is n x (R+1).
 * self_id is the id the search must skip (p.id() in the reference).
 * Returns 0, or -1 if an output buffer is too small. */
int ddo_beam_search(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
                    uint64_t stride, const uint32_t* graph, uint32_t R,
                    const void* query, int64_t self_id, uint32_t start, int64_t k,
                    int64_t L, double cut, int64_t limit, int64_t degree_limit,
                    uint32_t* fr_ids, float* fr_d, uint32_t* n_fr, uint32_t* vis_ids,
                    float* vis_d, uint32_t* n_vis, uint32_t vis_cap, uint64_t* dist_cmps);

/* searchAll (include/utils/beamSearch.h:314-346): query i skips base id i.
 * ids_out nq x k; visited_out, cmps_out per query (may be NULL). */
int ddo_search(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
               uint64_t stride, const uint32_t* graph, uint32_t R, const void* queries,
               uint64_t nq, uint64_t qstride, const uint32_t* L_per_query, int64_t k,
               double cut, int64_t limit, int64_t degree_limit, uint32_t start,
               int nthreads, uint32_t* ids_out, uint32_t* visited_out, uint32_t* cmps_out);

/* robustPrune (include/index.h:63-123) on an explicit candidate list. */
int ddo_robust_prune(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
                     uint64_t stride, const uint32_t* graph, uint32_t R, uint32_t p,
                     const uint32_t* cand_ids, const float* cand_d, uint32_t m,
                     double alpha, uint32_t* out, uint32_t* out_len);

/* Brute-force ground truth: FP64 distances for float data, exact integers for
 * integer data; ties ordered by id.  dists_out holds the distance as float. */
int ddo_groundtruth(int dtype, int metric, const void* points, uint64_t n, uint32_t d,
                    uint64_t stride, const void* queries, uint64_t nq, uint64_t qstride,
                    uint32_t k, int nthreads, uint32_t* ids_out, float* dists_out);

/* Round schedule (src/bsp_index.hpp:155-166, 238-246). Returns the number of
 * rounds (it may exceed cap; only cap are written). */
uint64_t ddo_schedule(uint64_t n, uint64_t max_build, double xita, int knn_mode,
                      uint64_t* floors, uint64_t* ceilings, uint64_t cap);

#ifdef __cplusplus
}
#endif
