// Host-visible launch interface of the device kernels (kernels.cu).
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

namespace ddk {

constexpr uint32_t kMaxL = 512;   // frontier capacity: 16 entries per lane
constexpr uint32_t kMaxRp = 128;  // graph row capacity: 4 candidates per lane

// Per-warp shared-memory carve-up of the search kernels (byte offsets, 16-byte
// aligned).  The lossy hash table of each search lives in global memory.
struct WarpLayout {
  uint32_t qv, fr_id, fr_d, c_id, c_d, s_id, s_d, vis_id, vis_d, ws;
  uint32_t total;
  uint32_t vcap;   // visited / evicted list capacity
  uint32_t ccap;   // prune candidate capacity (visited list + out-list)
  uint32_t hbits;  // hash bits of the largest beam width of the launch
  uint32_t h24;    // hash table of 24-bit ids (every id < 0xFFFFFF)
  uint32_t keep_vis;  // query layout holds the visited list (debug beam search)
  uint32_t fastf;     // build search with the fast form's seen filter (16-bit tags)
  uint32_t hash_global;  // query layout: the seen table lives in a global slice per warp
  uint32_t hash_words;   // its size in 32-bit words (16-byte multiple)
  uint32_t ev;           // query layout: evicted list in shared memory (keep_vis layouts)
};

// Per-warp shared-memory carve-up of k_prune (byte offsets, 16-byte aligned).
struct PruneLayout {
  uint32_t qv, cid, ckey, ws, total, ccap;
};

// CTA shape of a one-warp-per-item kernel
struct LaunchPlan {
  int warps_per_cta;
  int blocks_per_sm;
};

struct IndexView {
  int dtype, metric;
  const uint8_t* points;
  uint64_t stride;
  uint32_t* graph;
  uint32_t Rp, R;
  uint64_t n;
  uint32_t d;
  uint32_t* err;
  // fast form, float data: BF16 copies of the rows (sstride bytes apart) and
  // the squared norm of each copy, which search steps screen candidates with
  // (null: every candidate gets its exact distance)
  const uint8_t* screen = nullptr;
  uint64_t sstride = 0;
  const float* snorm = nullptr;
  // fast form, float data: log2 of the lanes that compute one candidate's
  // exact distance in a search step (0: one lane, the plain form; 4: chosen
  // per step from the candidate count)
  uint32_t fgroup_lg = 0;
};

// keep_vis: the query layout reserves the visited list (k_beam keeps it;
// k_query only needs the evicted list)
// fastf (build only): the fast form's seen filter, 16-bit tags (search_core.cuh)
// hash_global (query only): the seen table goes to a global slice per resident
// warp (QueryArgs::hash_scratch) instead of shared memory
WarpLayout make_search_layout(uint32_t d, int dtype, uint32_t L, uint32_t Rp, uint32_t vcap,
                              bool build, bool h24, bool keep_vis = true, bool fastf = false,
                              bool hash_global = false);
// tensor: the fast form's tensor-core greedy (integer data); false: the plain form
PruneLayout make_prune_layout(uint32_t d, int dtype, uint32_t Rp, uint32_t ccap, bool tensor);


struct RoundArgs {
  uint64_t floor;
  uint32_t B;            // batch points this round
  uint32_t L;
  double alpha;
  uint32_t start;
  uint32_t* new_out;     // B x Rp
  float* new_key;        // B x Rp distances of new_out's entries to their row's point, or
                         // null (the reverse step then recomputes them)
  float* row_key;        // with new_key: n x Rp, each graph entry's distance to its row's
                         // point (kept by every row write of the build), or null
  uint32_t* stat_vis;    // B visited-list lengths (k_search writes, k_prune reads)
  uint32_t* stat_cmps;   // B (may be null)
  uint32_t* vis_all;     // per batch point: vcap visited ids, then vcap distances
  int vis_sorted_tail;   // 1: each list is already in (dist, id) order at the end of its
                         // slice (the fast search's layout); 0: visit order from the start
  // device work queues (zeroed before the round): with a queue the launch is
  // persistent and each warp takes its next batch point from the counter;
  // null = static grid-stride assignment
  uint32_t* qsearch;
  uint32_t* qprune;
};

// The round's reverse edges grouped by target (see semisort.cuh): segment k
// holds pairs [heads[k], heads[k+1]) of st (targets) / sv (keys b*Rp + j).
struct ReverseScratch {
  const uint32_t* st;
  const uint32_t* sv;
  const uint32_t* heads;
  uint32_t* counters;  // [0] pairs V [1] segments T [2] pruned groups [3] prune cands
                       // [4] big segments [5] largest big candidate list
  uint32_t* big;       // segments for the CTA path
  // CTA path workspace, one slice per CTA (kBigSlots slices of gcap candidates):
  uint32_t* gcand;     // gcap ids
  float* gkey;         // gcap distances
  int* gpos;           // 2*gcap rank scratch
  uint32_t* gbits;     // gcap/32 + 2 leaf bitmap words
  int* granges;        // 3*(gcap/8 + 64) short-range records
  uint64_t gcap;
};

constexpr int kScanBlocks = 512;
// stack room of the sort emulation for any list length below 2^32
constexpr int kGlobalStackInts = 3 * (2 * 32 + 4);
constexpr uint32_t kRevCandCap = 256;   // per-warp shared-memory candidates (reverse)
constexpr uint32_t kRevWarps = 2;       // warps per CTA of the reverse kernel
constexpr uint32_t kBigThreads = 512;   // threads per CTA of the big-target path
constexpr uint32_t kBigSlots = 148;     // CTAs (and workspace slices) of the big-target path

LaunchPlan plan_search(const IndexView& ix, const WarpLayout& lay, uint32_t L);
// the CTA shapes an autotuner may time (see warp_kernel_candidates)
std::vector<LaunchPlan> search_plan_candidates(const IndexView& ix, const WarpLayout& lay,
                                               uint32_t L);
std::vector<LaunchPlan> prune_plan_candidates(const IndexView& ix, const PruneLayout& lay,
                                              bool tensor);
void launch_search(const IndexView& ix, const RoundArgs& ra, const WarpLayout& lay,
                   const LaunchPlan& plan, int grid, cudaStream_t st);
LaunchPlan plan_prune(const IndexView& ix, const PruneLayout& lay, bool tensor);
void launch_prune_round(const IndexView& ix, const RoundArgs& ra, const PruneLayout& lay,
                        uint32_t vcap, const LaunchPlan& plan, int grid, bool tensor,
                        cudaStream_t st);
void launch_apply_rows(const IndexView& ix, const RoundArgs& ra, cudaStream_t st);
// append-or-prune per target over the segments the semisort produced
void launch_reverse(const IndexView& ix, const RoundArgs& ra, const ReverseScratch& rs,
                    bool tensor, cudaStream_t st, int sm_count);

struct QueryArgs {
  const uint8_t* queries;  // device rows, stride qstride (zero padded to 16 bytes)
  uint64_t qstride;
  uint64_t nq;
  const uint32_t* Ls;      // per-query beam width
  uint32_t Lmax;
  uint32_t k;
  double cut;
  uint64_t limit;
  uint32_t degree_limit;
  uint32_t start;
  int skip_self;           // searchAll semantics: query i skips base id i
  uint32_t* ids;           // nq x k
  float* dists;            // nq x k
  uint32_t* visited;       // nq (may be null)
  uint32_t* cmps;          // nq (may be null)
  // beam-width class of the launch (fast form): the launch serves the
  // queries listed in cls_items[0, *cls_count), taken from the work queue
  // cls_queue; null = every query, grid-stride
  const uint32_t* cls_items;
  const uint32_t* cls_count;
  uint32_t* cls_queue;
  uint32_t Lvalid;         // largest valid beam width (the caller's Lmax; Lmax is the class's)
  uint32_t* hash_scratch;  // layouts with hash_global: one table per warp of the grid
  uint32_t* ev_scratch;    // evicted lists, ev_cap ids per warp of the grid
  uint32_t ev_cap;
};

// Beam-width classes of the bucketed query launch: class c serves beam widths
// in (16 << (c-1), 16 << c]; its launch is laid out for 16 << c.
constexpr int kQueryClasses = 6;
__host__ __device__ inline int query_class(uint32_t L) {
  int c = 0;
  while (c + 1 < kQueryClasses && L > (16u << c)) c++;
  return c;
}
// Lists the queries of each class: items[c * nq + i], counts[c] (zeroed before).
// A query whose beam width is invalid (0, below k or above Lvalid) goes to the
// class of Lvalid, whose launch reports it.
void launch_bin_queries(const uint32_t* Ls, uint64_t nq, uint32_t k, uint32_t Lvalid,
                        uint32_t* items, uint32_t* counts, cudaStream_t st);
LaunchPlan plan_query(const IndexView& ix, const WarpLayout& lay, uint32_t Lmax);
void launch_query(const IndexView& ix, const QueryArgs& qa, const WarpLayout& lay,
                  int warps_per_cta, int grid, cudaStream_t st);

// beam_search with full frontier + visited outputs (kernel-level parity tests)
struct BeamArgs {
  const uint8_t* queries;
  uint64_t qstride;
  uint64_t nq;
  const int64_t* self_ids;  // per query (-1: none)
  uint32_t L, k;
  double cut;
  uint64_t limit;
  uint32_t degree_limit;
  uint32_t start;
  uint32_t vcap;
  uint32_t* fr_ids; float* fr_d; uint32_t* fr_n;     // nq x L
  uint32_t* vis_ids; float* vis_d; uint32_t* vis_n;  // nq x vcap
  uint32_t* cmps;
};
void launch_beam(const IndexView& ix, const BeamArgs& ba, const WarpLayout& lay, int grid,
                 cudaStream_t st);

// robustPrune on explicit candidate lists (kernel-level parity tests)
struct PruneArgs {
  uint32_t ntasks;
  const uint32_t* p;          // ntasks
  const uint64_t* offsets;    // ntasks + 1 into cand arrays
  const uint32_t* cand_ids;
  const float* cand_d;
  double alpha;
  uint32_t* out;              // ntasks x Rp
  // workspace: gcand/gkey hold W = offsets[ntasks] + ntasks*Rp entries, gws
  // 3*W + ntasks*kGlobalStackInts ints
  uint32_t* gcand; float* gkey; int* gws;
};
void launch_prune_tasks(const IndexView& ix, const PruneArgs& pa, cudaStream_t st);

// brute-force ground truth (FP64 for float data, exact integers otherwise)
void launch_groundtruth(const IndexView& ix, const uint8_t* queries, uint64_t qstride, uint64_t nq,
                        uint32_t k, uint32_t* ids, float* dists, double* part_d,
                        uint32_t* part_i, uint32_t nchunks, cudaStream_t st);

// sharded build exchange: the rows of the targets this rank's reverse step
// changed (segments of the grouped pairs, st/heads/counters as in
// ReverseScratch), and the application of rows received from other ranks
void launch_export_rows(const IndexView& ix, const uint32_t* st, const uint32_t* heads,
                        const uint32_t* counters, uint64_t cap, uint32_t* ids_out,
                        uint32_t* rows_out, cudaStream_t stream);
void launch_set_rows(const IndexView& ix, const uint32_t* ids, const uint32_t* rows,
                     uint64_t count, cudaStream_t stream);

// graph format conversion (device rows <-> reference [deg, nbr...] rows)
void launch_to_ref_rows(const IndexView& ix, uint32_t* out, cudaStream_t st);
void launch_from_ref_rows(const IndexView& ix, const uint32_t* in, cudaStream_t st);
// knn_index::build_index final step: sort each row by distance to its owner
void launch_sort_rows(const IndexView& ix, cudaStream_t st);
// fast form, float data: BF16 copies of the rows (round to nearest, zero
// padded to sstride bytes) and their squared norms, which the search steps'
// screen reads (search_core.cuh screen_and_rerank)
void launch_screen_rows(const IndexView& ix, uint8_t* screen, uint64_t sstride, float* snorm,
                        cudaStream_t st);

}  // namespace ddk
