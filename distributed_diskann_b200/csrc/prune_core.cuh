// Warp-cooperative robustPrune (include/index.h:63-123; src/bsp_index.hpp:483-545).
//
//  1. the candidate list (ids + distances to p) is ordered exactly as the
//     reference's std::sort orders it (sort_emul.cuh: lane 0 replays the
//     partition phase, then every lane finishes whole leaves);
//  2. greedy selection: walk the sorted list, skip p and removed entries,
//     select p*, and remove every later p' with alpha * d(p*, p') <= d(p, p')
//     (alpha is a double in the reference, so the test is done in double).
//     The occlusion distances of one p* are spread over the 32 lanes.
#pragma once
#include "dd_common.cuh"
#include "sort_emul.cuh"

namespace ddk {

struct PruneSmem {
  uint32_t* cid;   // candidate ids (DD_NONE = removed)
  float* ckey;     // distance to p
  int* leaf_lo;    // leaf ranges of the sort emulation (capacity = candidates)
  int* leaf_hi;
  int* stack;      // ddsort::stack_ints(capacity) ints
  int* scalar;     // one shared int
};

// Orders cid/ckey[0, m) exactly like std::sort with the distance-only comparator.
__device__ __forceinline__ void warp_std_sort(const PruneSmem& S, uint32_t m) {
  const uint32_t lane = lane_id();
  ddsort::Arr<uint32_t> A{S.cid, S.ckey};
  if (lane == 0) S.scalar[0] = ddsort::partition_phase(A, (int)m, S.stack, S.leaf_lo, S.leaf_hi);
  __syncwarp();
  const int nl = S.scalar[0];
  for (int i = (int)lane; i < nl; i += 32) ddsort::insertion_sort_range(A, S.leaf_lo[i], S.leaf_hi[i]);
  __syncwarp();
}

// Greedy selection over the sorted candidates; writes the selected ids to
// out_row[0, nsel) and DD_NONE to out_row[nsel, Rp).  Returns nsel.
template <int DT, int MT>
__device__ uint32_t warp_greedy_select(const uint8_t* points, uint64_t stride, uint32_t d,
                                       uint32_t p, const PruneSmem& S, uint32_t m, double alpha,
                                       uint32_t R, uint32_t* out_row, uint32_t Rp) {
  const uint32_t lane = lane_id();
  uint32_t nsel = 0, idx = 0;
  while (nsel < R && idx < m) {
    const uint32_t ps = S.cid[idx];
    idx++;
    if (ps == p || ps == DD_NONE) continue;
    if (lane == 0) out_row[nsel] = ps;
    nsel++;
    const uint8_t* prow = points + (uint64_t)ps * stride;
    for (uint32_t i = idx + lane; i < m; i += 32) {
      const uint32_t c = S.cid[i];
      if (c != DD_NONE) {
        const float dsp = Dist<DT, MT>::eval(prow, points + (uint64_t)c * stride, d);
        if (__dmul_rn(alpha, (double)dsp) <= (double)S.ckey[i]) S.cid[i] = DD_NONE;
      }
    }
    __syncwarp();
  }
  for (uint32_t j = nsel + lane; j < Rp; j += 32) out_row[j] = DD_NONE;
  __syncwarp();
  return nsel;
}

// In-place ascending sort of (key, id) pairs by (key, id) on one warp:
// bitonic network with all comparators ascending (the partner of i in the
// first step of each stage is i ^ (k - 1)), so a ragged tail needs no padding.
__device__ __forceinline__ void warp_sort_pairs(uint32_t* ids, float* keys, uint32_t n) {
  const uint32_t lane = lane_id();
  uint32_t N = 1;
  while (N < n) N <<= 1;
  for (uint32_t k = 2; k <= N; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = lane; i < N; i += 32) {
        uint32_t l = (j == (k >> 1)) ? (i ^ (k - 1)) : (i ^ j);
        if (l > i && l < n) {
          float ki = keys[i], kl = keys[l];
          uint32_t ii = ids[i], il = ids[l];
          if (pair_less(kl, il, ki, ii)) {
            keys[i] = kl; keys[l] = ki;
            ids[i] = il; ids[l] = ii;
          }
        }
      }
      __syncwarp();
    }
  }
}

// same network on plain uint32 keys (reverse-edge segments)
__device__ __forceinline__ void warp_sort_u32(uint32_t* a, uint32_t n) {
  const uint32_t lane = lane_id();
  uint32_t N = 1;
  while (N < n) N <<= 1;
  for (uint32_t k = 2; k <= N; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = lane; i < N; i += 32) {
        uint32_t l = (j == (k >> 1)) ? (i ^ (k - 1)) : (i ^ j);
        if (l > i && l < n) {
          uint32_t x = a[i], y = a[l];
          if (y < x) { a[i] = y; a[l] = x; }
        }
      }
      __syncwarp();
    }
  }
}

}  // namespace ddk
