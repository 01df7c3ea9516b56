/* C ABI of the B200-native Vamana hot path (distributed_diskann_b200).
 *
 * One opaque handle owns a device-resident index: the points, the
 * fixed-degree graph and all build/search scratch live in HBM of one GPU.
 * Every entry point takes plain pointers and sizes and returns an int status
 * (DD_OK = 0); dd_last_error() gives the message of the last failure.
 * Host buffers are ordinary (or pinned) host memory; *_device entry points
 * take device pointers.  Calls on one handle must be serialized (the handle is
 * thread-compatible, not thread-safe), like the reference's Graph objects.
 *
 * Reference interfaces replaced (paths within Mr1BW/distributed_diskann):
 *   BSP_index<Point,PointRange,indexType>::bsp_build   src/bsp_index.hpp:551-556
 *   knn_index<...>::build_index / batch_insert          include/index.h:125-137, 213-341
 *   knn_index<...>::robustPrune                         include/index.h:63-123
 *   beam_search                                         include/utils/beamSearch.h:41-184
 *   searchAll                                           include/utils/beamSearch.h:314-346
 *   Graph<indexType>(char*), Graph::save                include/utils/graph.h:130-200
 *   PointRange<T,Point>(char*)                          include/utils/point_range.h:61-97
 *   dataset_para (para.json keys R L alpha xita max start_point_index two_pass)
 *                                                       src/dataset.hpp:50-89
 */
#ifndef DD_GPU_H
#define DD_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define DD_OK 0
#define DD_ERR_ARG 1          /* invalid argument (reference: abort() with a message) */
#define DD_ERR_CUDA 2         /* CUDA runtime error */
#define DD_ERR_OOM 3          /* device allocation failed */
#define DD_ERR_DEVICE 4       /* a kernel raised its error word (bad id, capacity, degree) */
#define DD_ERR_UNSUPPORTED 5  /* parameter outside the supported range */
#define DD_ERR_IO 6           /* file could not be read or written */

/* computation forms (dd_build_params.mode, dd_set_search_mode).  Both give
 * the same graph and the same search results, bit for bit:
 *   DD_MODE_FAST  : tensor-core distance tiles where they apply (INT8 Gram
 *                   tiles of robustPrune for integer data), optionally for
 *                   float data (DD_SCREEN=1 in the environment) a BF16 screen
 *                   of search candidates with an exact FP32 re-rank of the
 *                   ones it cannot rule out (a BF16 copy of the points, n x
 *                   round_up(2d, 16) bytes, is then kept on the device; off
 *                   by default: slower than exact distances on B200; so is
 *                   DD_FGROUP, exact float distances by lane groups),
 *                   persistent kernels
 *                   fed by a device work queue, each build captured as one CUDA
 *                   graph, autotuned CTA shapes, queries bucketed by beam width;
 *   DD_MODE_PLAIN : every distance on the CUDA cores, grid-stride kernels
 *                   launched round by round, one query launch sized for the
 *                   largest beam width (the exact form the fast one is checked
 *                   and timed against). */
#define DD_MODE_FAST 0
#define DD_MODE_PLAIN 1

/* element types (the reference's dtype dispatch, src/diskann.cpp:118-120) */
#define DD_DTYPE_F32 0
#define DD_DTYPE_I8 1
#define DD_DTYPE_U8 2
/* metrics: Euclidian_Point (include/utils/euclidian_point.h) and
 * Mips_Point (include/utils/mips_point.h) */
#define DD_METRIC_L2 0
#define DD_METRIC_MIPS 1

typedef struct dd_index dd_index;

/* Build parameters: the para.json surface of the reference (src/dataset.hpp:64-89)
 * plus the BuildParams fields it feeds (include/utils/types.h:103-142). */
typedef struct dd_build_params {
  uint32_t L;            /* beam width of the insert searches ("L") */
  double alpha;          /* robustPrune alpha ("alpha") */
  double max_fraction;   /* max batch = max_fraction * m, capped at 1e6 ("xita") */
  uint64_t max_build;    /* insert only the first max_build points, 0 = all ("max") */
  uint32_t start_point;  /* search entry point ("start_point_index") */
  int32_t two_pass;      /* first pass with alpha = 1 ("two_pass"; knn_index semantics) */
  int32_t knn_mode;      /* 1: knn_index::build_index (max_fraction 1, sorted rows) */
  int32_t collect_stats; /* 1: fill visited / distance-count statistics */
  uint32_t vcap;         /* starting visited-list capacity per search (0 = 4 * L); it is
                            doubled and the build rerun while a search overflows it */
  int32_t mode;          /* DD_MODE_FAST (0) or DD_MODE_PLAIN */
} dd_build_params;

typedef struct dd_stats {
  uint64_t rounds;         /* batches inserted (all passes) */
  uint64_t visited;        /* sum of visited-list sizes (reference BuildStats visited) */
  uint64_t dist_cmps;      /* sum of beam-search distance computations */
  uint64_t groups;         /* reverse-edge targets (group_by_key groups) */
  uint64_t reverse_prunes; /* targets whose row overflowed and was pruned */
  uint64_t prune_cands;    /* candidates of those prunes */
  uint64_t big_groups;     /* targets handled by the global-memory path */
  double build_ms;         /* device time of the whole build */
  double search_prune_ms;  /* device time of the insert search + prune kernels */
  double reverse_ms;       /* device time of the reverse-edge kernels */
  double search_ms;        /* device time of the insert beam searches alone (part of
                              search_prune_ms) */
  uint32_t search_warps_per_cta; /* CTA shape of the insert searches (autotuned: fast form) */
  uint32_t prune_warps_per_cta;  /* CTA shape of the insert prunes */
  int32_t search_queue;    /* 1: persistent searches fed by a device work queue */
  int32_t prune_queue;     /* 1: persistent prunes fed by a device work queue */
  int32_t graph_replay;    /* 1: the build ran as one replayed CUDA graph */
  uint32_t vcap;           /* visited-list capacity the build ran with */
} dd_stats;

/* ------------------------------------------------------------------ handle */
/* Creates an empty index for n points of dimension d and maximum degree R on
 * CUDA device `device`.  R <= 128. */
int dd_create(int dtype, int metric, uint64_t n, uint32_t d, uint32_t R, int device,
              dd_index** out);
int dd_destroy(dd_index* h);
const char* dd_last_error(const dd_index* h);
/* all work of the handle is issued on this CUDA stream (cudaStream_t); 0 = default */
int dd_set_stream(dd_index* h, void* stream);
/* form of dd_search / dd_search_device (DD_MODE_FAST by default) */
int dd_set_search_mode(dd_index* h, int mode);
/* waits for the handle's stream and reports the device error word that the
 * asynchronous entry points (dd_search_device) leave: DD_ERR_DEVICE with the
 * message when a kernel raised it since the last check, else DD_OK */
int dd_check_errors(dd_index* h);

/* ------------------------------------------------------------------ data */
/* PointRange: copies n rows of d elements; row_stride_bytes between rows */
int dd_upload_points(dd_index* h, const void* rows, uint64_t row_stride_bytes);
int dd_upload_points_device(dd_index* h, const void* rows, uint64_t row_stride_bytes);
/* the same copy ordered on the handle's stream without waiting for it: rows
 * should be pinned host memory (cudaMallocHost) for the copy to overlap other
 * work, and must stay valid until the stream reaches the copy (any
 * synchronizing call of the handle, or dd_check_errors) */
int dd_upload_points_async(dd_index* h, const void* rows, uint64_t row_stride_bytes);
/* reads a reference .bin file ([u32 n][u32 d][n*d elements]) into the index,
 * through two pinned staging buffers: disk reads overlap the uploads
 * (PointRange(char*), include/utils/point_range.h:61-97) */
int dd_load_points_file(dd_index* h, const char* path);
/* Graph rows in the reference layout: n rows of (R+1) uint32, row[0] = degree */
int dd_upload_graph(dd_index* h, const uint32_t* rows);
int dd_download_graph(dd_index* h, uint32_t* rows);
/* Graph(char*) / Graph::save file format ([u32 n][u32 R][degrees][edges]) */
int dd_load_graph_file(dd_index* h, const char* path);
int dd_save_graph_file(dd_index* h, const char* path);

/* ------------------------------------------------------------------ build */
/* bsp_build / knn_index::build_index: batched prefix-doubling insertion of the
 * points into an empty graph.  stats may be NULL. */
int dd_build(dd_index* h, const dd_build_params* params, dd_stats* stats);

/* The round schedule (src/bsp_index.hpp:155-166, 238-246): writes up to cap
 * [floor, ceiling) pairs and the number of rounds. */
int dd_schedule(uint64_t n, uint64_t max_build, double max_fraction, int knn_mode,
                uint64_t* floors, uint64_t* ceilings, uint64_t cap, uint64_t* nrounds);

/* ------------------------------------------------------------------ sharded build
 * One rank's steps of the build spread over P ranks, one GPU each, every rank
 * holding the whole points and graph: BSP_index's superstep pair
 * (src/bsp_index.hpp:238-407) with the MPI broadcasts of
 * include/bsp/broadcast_bsp_framework.cpp:166-218 left to the caller (NCCL
 * all-gathers of device buffers).  Per round [floor, ceiling) of dd_schedule:
 *   1. dd_shard_search_prune on the rank's slice [lo, hi) of the batch
 *      (slice r of P: floor + r*(B/P) + min(r, B%P), B/P + (r < B%P) points,
 *      src/bsp_index.hpp:247-252): hi-lo new out-lists of dd_device_row_len
 *      ids (padding 0xFFFFFFFF) into `rows` (device);
 *   2. all-gather the slices into the batch's B rows, in batch order;
 *   3. dd_shard_apply_reverse: update_neighbors of the batch, then the reverse
 *      edges of the targets this rank owns (t % P == rank, :362-373), append
 *      or robustPrune; the changed targets' ids and rows go to ids_out /
 *      rows_out (device, room for cap), their number to *count;
 *   4. all-gather those and apply the other ranks' with dd_shard_set_rows.
 * The result equals dd_build's graph.  Single-pass builds only (no two_pass,
 * no knn_mode); vcap 0 means 8 * L here, and an overflow is an error. */
int dd_shard_begin(dd_index* h, const dd_build_params* params, uint64_t max_batch);
int dd_shard_search_prune(dd_index* h, uint64_t lo, uint64_t hi, uint32_t* rows);
int dd_shard_apply_reverse(dd_index* h, uint64_t floor, uint64_t ceiling, const uint32_t* batch_rows,
                           int rank, int world, uint32_t* ids_out, uint32_t* rows_out,
                           uint64_t cap, uint64_t* count);
int dd_shard_set_rows(dd_index* h, const uint32_t* ids, const uint32_t* rows, uint64_t count);

/* ------------------------------------------------------------------ search */
/* searchAll: nq queries (rows of d elements, qstride bytes apart) searched
 * from `start` with QueryParams(k, L_per_query[i], cut, limit, degree_limit);
 * limit 0 = n, degree_limit 0 = R.  skip_self != 0 reproduces the reference's
 * p.id() skip (query i never expands base id i).  Outputs nq x k ids/dists
 * (0xFFFFFFFF / +inf where the final frontier is shorter than k); visited and
 * cmps (per query, may be NULL) are the reference's QueryStats counters. */
int dd_search(dd_index* h, const void* queries, uint64_t nq, uint64_t qstride,
              const uint32_t* L_per_query, uint32_t k, double cut, uint64_t limit,
              uint32_t degree_limit, uint32_t start, int skip_self, uint32_t* ids,
              float* dists, uint32_t* visited, uint32_t* cmps);
/* same with device pointers; queries must be rows zero padded to a multiple of
 * 16 bytes with qstride a multiple of 16 */
int dd_search_device(dd_index* h, const void* queries, uint64_t nq, uint64_t qstride,
                     const uint32_t* L_per_query, uint32_t Lmax, uint32_t k, double cut,
                     uint64_t limit, uint32_t degree_limit, uint32_t start, int skip_self,
                     uint32_t* ids, float* dists, uint32_t* visited, uint32_t* cmps);

/* beam_search per query with the full final frontier (nq x L) and the sorted
 * visited list (nq x vcap); self_ids[i] is the id p.id() skips (-1: none). */
int dd_beam_search(dd_index* h, const void* queries, uint64_t nq, uint64_t qstride,
                   const int64_t* self_ids, uint32_t L, uint32_t k, double cut, uint64_t limit,
                   uint32_t degree_limit, uint32_t start, uint32_t vcap, uint32_t* fr_ids,
                   float* fr_dists, uint32_t* fr_sizes, uint32_t* vis_ids, float* vis_dists,
                   uint32_t* vis_sizes, uint32_t* cmps);

/* robustPrune(p, cand, G, Points, alpha) for ntasks explicit candidate lists
 * against the current graph; candidates of task t are
 * cand_ids/cand_dists[offsets[t], offsets[t+1]).  out is ntasks x R. */
int dd_robust_prune(dd_index* h, uint32_t ntasks, const uint32_t* p, const uint64_t* offsets,
                    const uint32_t* cand_ids, const float* cand_dists, double alpha,
                    uint32_t* out, uint32_t* out_len);

/* dd_robust_prune without any device allocation (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc at this point: a
 * serving process that reserved its whole device-memory budget at start-up
 * and forbids later allocation (cudaMalloc may also synchronize the device),
 * or a host whose device memory belongs to another allocator that must not be
 * bypassed.  All
 * arguments are DEVICE pointers: p (ntasks), offsets (ntasks + 1, with
 * offsets[ntasks] == total_cands), cand_ids / cand_dists (total_cands), and out
 * (ntasks x dd_device_row_len(h) ids, each row padded with 0xFFFFFFFF).  The
 * candidate workspace is a fixed device array inside the library, held by every
 * GPU that loads it until the process exits: at most 2048 tasks and
 * total_cands + ntasks * dd_device_row_len(h) <= 65536 slots, larger calls
 * return DD_ERR_UNSUPPORTED.  The first call on a device looks up that array's
 * device address; make it before any stream capture.  All calls on a device
 * share the array: calls whose kernels overlap on the GPU race and must be
 * serialized.  The kernel runs on the handle's stream; with synchronize != 0
 * the call waits for it and reports invalid device inputs as DD_ERR_DEVICE,
 * otherwise the handle's error word reports them at its next synchronizing
 * call.  Offsets that decrease or do not end at total_cands invalidate the
 * whole call (every row is padding); an id >= n (p[t] or a candidate of task
 * t) pads only row t.  Rows of valid tasks are correct in both cases. */
int dd_robust_prune_noalloc(dd_index* h, uint32_t ntasks, const uint32_t* p,
                            const uint64_t* offsets, uint64_t total_cands,
                            const uint32_t* cand_ids, const float* cand_dists, double alpha,
                            uint32_t* out, int synchronize);

/* brute-force k nearest neighbours (k <= 32): FP64 distances for float data,
 * exact integers for integer data; ties ordered by id */
int dd_groundtruth(dd_index* h, const void* queries, uint64_t nq, uint64_t qstride, uint32_t k,
                   uint32_t* ids, float* dists);

/* ------------------------------------------------------------------ device views */
void* dd_device_points(dd_index* h);      /* n rows, dd_device_row_stride bytes apart */
uint64_t dd_device_row_stride(dd_index* h);
void* dd_device_graph(dd_index* h);       /* n rows of dd_device_row_len uint32 */
uint32_t dd_device_row_len(dd_index* h);
/* kernels launched by the last dd_build / dd_search call */
uint64_t dd_last_launch_count(dd_index* h);

#ifdef __cplusplus
}
#endif
#endif /* DD_GPU_H */
