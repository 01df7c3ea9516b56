// Host-visible launch interface of the device kernels (kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ddk {

constexpr uint32_t kMaxL = 512;   // frontier capacity: 16 entries per lane
constexpr uint32_t kMaxRp = 128;  // graph row capacity: 4 candidates per lane

// Per-warp shared-memory carve-up of the fused search+prune kernel and of the
// query kernel (all offsets in bytes, 16-byte aligned).
struct WarpLayout {
  uint32_t qv, fr_id, fr_d, c_id, c_d, s_id, s_d, vis_id, vis_d, ws;
  uint32_t total;
  uint32_t vcap;   // visited/evicted capacity
  uint32_t ccap;   // prune candidate capacity (vis arrays hold vcap + Rp)
  uint32_t hbits;
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
};

WarpLayout make_search_layout(uint32_t d, int dtype, uint32_t L, uint32_t Rp, uint32_t vcap,
                              bool with_prune);

struct RoundArgs {
  uint64_t floor;
  uint32_t B;          // batch points this round
  uint32_t L;
  double alpha;
  uint32_t start;
  uint32_t* new_out;   // B x Rp
  uint32_t* stat_vis;  // B (may be null)
  uint32_t* stat_cmps; // B (may be null)
};

struct ReverseScratch {
  uint32_t* cnt;       // n, zero between rounds
  uint32_t* cursor;    // n
  uint32_t* touched;   // list of targets with incoming edges
  uint32_t* seg_start; // per touched entry
  uint32_t* keys;      // B*Rp segment keys (b*Rp + j)
  uint32_t* counters;  // [0] touched, [1] big entries, [2] pruned groups, [3] prune cands
  uint32_t* big;       // touched entries handled by the global-memory path
  uint32_t* block_sums;// scan partials (kScanBlocks + 1)
  uint32_t* gcand;     // global candidate workspace for the big path
  float* gkey;
  int* gleaf;          // 2x workspace for leaves + stack
  uint64_t gcap;       // candidate capacity of the big path
};

constexpr int kScanBlocks = 512;
// stack room of the sort emulation for any list length below 2^32
constexpr int kGlobalStackInts = 3 * (2 * 32 + 4);
constexpr uint32_t kRevCandCap = 512;   // shared-memory candidate capacity per target
constexpr uint32_t kRevWarps = 4;       // warps per CTA of the reverse kernel

void launch_search_prune(const IndexView& ix, const RoundArgs& ra, const WarpLayout& lay,
                         int warps_per_cta, int grid, cudaStream_t st);
void launch_apply_rows(const IndexView& ix, const RoundArgs& ra, cudaStream_t st);
void launch_reverse(const IndexView& ix, const RoundArgs& ra, const ReverseScratch& rs,
                    cudaStream_t st, int sm_count);
void launch_reverse_big(const IndexView& ix, const RoundArgs& ra, const ReverseScratch& rs,
                        uint32_t slots, cudaStream_t st);

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
};
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
void launch_beam(const IndexView& ix, const BeamArgs& ba, const WarpLayout& lay, cudaStream_t st);

// robustPrune on explicit candidate lists (kernel-level parity tests)
struct PruneArgs {
  uint32_t ntasks;
  const uint32_t* p;          // ntasks
  const uint64_t* offsets;    // ntasks + 1 into cand arrays
  const uint32_t* cand_ids;
  const float* cand_d;
  double alpha;
  uint32_t* out;              // ntasks x Rp
  // workspace: gcand/gkey hold offsets[ntasks] + ntasks*Rp entries, gleaf twice
  // that plus ntasks*kGlobalStackInts
  uint32_t* gcand; float* gkey; int* gleaf;
};
void launch_prune_tasks(const IndexView& ix, const PruneArgs& pa, cudaStream_t st);

// brute-force ground truth (FP64 for float data, exact integers otherwise)
void launch_groundtruth(const IndexView& ix, const uint8_t* queries, uint64_t qstride, uint64_t nq,
                        uint32_t k, uint32_t* ids, float* dists, double* part_d,
                        uint32_t* part_i, uint32_t nchunks, cudaStream_t st);

// graph format conversion (device rows <-> reference [deg, nbr...] rows)
void launch_to_ref_rows(const IndexView& ix, uint32_t* out, cudaStream_t st);
void launch_from_ref_rows(const IndexView& ix, const uint32_t* in, cudaStream_t st);
// knn_index::build_index final step: sort each row by distance to its owner
void launch_sort_rows(const IndexView& ix, cudaStream_t st);

}  // namespace ddk
