// Helpers shared by the kernel translation units: sizes, vector loads,
// dtype/metric dispatch and CTA-shape planning of one-warp-per-item kernels.
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

#include "dd_common.cuh"
#include "kernels.cuh"

namespace ddk {

static __host__ __device__ inline uint32_t r16(uint64_t x) {
  return (uint32_t)((x + 15) & ~(uint64_t)15);
}

// copy a padded vector row into shared memory (16-byte granules)
__device__ __forceinline__ void load_vec(uint8_t* dst, const uint8_t* src, uint32_t bytes16) {
  const uint4* s4 = (const uint4*)src;
  uint4* d4 = (uint4*)dst;
  for (uint32_t i = lane_id(); i < bytes16 / 16; i += 32) d4[i] = __ldg(s4 + i);
}

// number of valid neighbours (the valid entries are a prefix of the row)
__device__ __forceinline__ uint32_t row_degree(const uint32_t* row, uint32_t Rp) {
  uint32_t deg = 0;
  for (uint32_t base = 0; base < Rp; base += 32) {
    uint32_t j = base + lane_id();
    bool v = (j < Rp) && (row[j] != DD_NONE);
    deg += __popc(__ballot_sync(0xffffffffu, v));
  }
  return deg;
}

// The next work item of a warp: from the device queue `q` (one atomic by
// lane 0, broadcast) when the launch is persistent, else the static
// grid-stride sequence cur, cur + step, ...  `q` is uniform over the launch.
__device__ __forceinline__ uint64_t warp_next_item(uint32_t* q, uint64_t& cur, uint64_t step) {
  if (q) {
    uint32_t v = 0;
    if (lane_id() == 0) v = atomicAdd(q, 1u);
    return __shfl_sync(0xffffffffu, v, 0);
  }
  const uint64_t r = cur;
  cur += step;
  return r;
}

#define DD_DISPATCH_DM(dtype, metric, CALL)                                          \
  do {                                                                               \
    if ((dtype) == DD_F32 && (metric) == DD_L2) { CALL(DD_F32, DD_L2); }             \
    else if ((dtype) == DD_F32) { CALL(DD_F32, DD_MIPS); }                           \
    else if ((dtype) == DD_I8 && (metric) == DD_L2) { CALL(DD_I8, DD_L2); }          \
    else if ((dtype) == DD_I8) { CALL(DD_I8, DD_MIPS); }                             \
    else if ((metric) == DD_L2) { CALL(DD_U8, DD_L2); }                              \
    else { CALL(DD_U8, DD_MIPS); }                                                   \
  } while (0)

// frontier / row register buckets: (L <= 128 | L <= 512) x (Rp <= 64 | Rp <= 128)
#define DD_DISPATCH_FC(L, Rp, DT, MT, CALL4)                                         \
  do {                                                                               \
    if ((L) <= 128 && (Rp) <= 64) { CALL4(DT, MT, 4, 2); }                           \
    else if ((L) <= 128) { CALL4(DT, MT, 4, 4); }                                    \
    else if ((Rp) <= 64) { CALL4(DT, MT, 16, 2); }                                   \
    else { CALL4(DT, MT, 16, 4); }                                                   \
  } while (0)

template <typename K>
static void set_smem(K kernel, size_t bytes) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename K>
static int occupancy(K kernel, int threads, size_t smem) {
  set_smem(kernel, smem);
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem) != cudaSuccess) b = 1;
  return b > 0 ? b : 1;
}


// Warps per CTA of a per-warp kernel: the CTA size (up to 16 warps) that keeps
// the most warps resident per SM, the smaller CTA on ties.
template <typename K>
static LaunchPlan plan_warp_kernel(K kernel, uint32_t bytes_per_warp) {
  LaunchPlan best{1, 0};
  static const int cand[] = {1, 2, 4, 5, 7, 8, 11, 16};
  cudaFuncAttributes fa{};
  const int max_threads =
      cudaFuncGetAttributes(&fa, kernel) == cudaSuccess ? fa.maxThreadsPerBlock : 512;
  for (int wpc : cand) {
    const size_t sm = (size_t)bytes_per_warp * wpc;
    if (sm > 227 * 1024 || wpc * 32 > max_threads) break;
    const int b = occupancy(kernel, wpc * 32, sm);
    if (b * wpc > best.warps_per_cta * best.blocks_per_sm) best = LaunchPlan{wpc, b};
  }
  if (best.blocks_per_sm == 0) best.blocks_per_sm = 1;
  return best;
}

// The CTA shapes the autotuner times for a per-warp kernel: 2, 4, 7, 8, 11
// and 16 warps per CTA (within the kernel's launch bounds), each with the
// CTAs per SM the occupancy API allows.
template <typename K>
static std::vector<LaunchPlan> warp_kernel_candidates(K kernel, uint32_t bytes_per_warp) {
  std::vector<LaunchPlan> v;
  static const int cand[] = {2, 4, 7, 8, 11, 16};
  cudaFuncAttributes fa{};
  const int max_threads =
      cudaFuncGetAttributes(&fa, kernel) == cudaSuccess ? fa.maxThreadsPerBlock : 512;
  for (int wpc : cand) {
    const size_t sm = (size_t)bytes_per_warp * wpc;
    if (sm > 227 * 1024 || wpc * 32 > max_threads) break;
    const int b = occupancy(kernel, wpc * 32, sm);
    if (b >= 1) v.push_back(LaunchPlan{wpc, b});
  }
  return v;
}

}  // namespace ddk
