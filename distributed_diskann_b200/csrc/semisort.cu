// Stable radix sort of the round's (target, key) pairs and segment heads
// (see semisort.cuh).
#include "dd_common.cuh"
#include "kernels.cuh"
#include "semisort.cuh"

#include <algorithm>

namespace ddk {

uint64_t semisort_hist_words(uint64_t E) { return 256ull * ((E + kRadixTile - 1) / kRadixTile); }

// ---- generic exclusive scan of a[0, N) in place; N from *n_dev when given
__global__ void k_gscan1(const uint32_t* a, uint64_t n_host, const uint32_t* n_dev,
                         uint32_t* block_sums) {
  __shared__ uint32_t sh[32];
  const uint64_t N = n_dev ? *n_dev : n_host;
  const uint64_t chunk = (N + gridDim.x - 1) / gridDim.x;
  const uint64_t lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  uint32_t s = 0;
  for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s += a[i];
  uint32_t tot;
  cta_scan_excl(s, &tot, sh);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void k_gscan2(uint32_t* block_sums, int nb, uint32_t* total_out) {
  __shared__ uint32_t sh[32];
  uint32_t v = threadIdx.x < (uint32_t)nb ? block_sums[threadIdx.x] : 0;
  uint32_t tot;
  uint32_t ex = cta_scan_excl(v, &tot, sh);
  if (threadIdx.x < (uint32_t)nb) block_sums[threadIdx.x] = ex;
  if (threadIdx.x == 0 && total_out) *total_out = tot;
}

__global__ void k_gscan3(uint32_t* a, uint64_t n_host, const uint32_t* n_dev,
                         const uint32_t* block_sums) {
  __shared__ uint32_t sh[32];
  const uint64_t N = n_dev ? *n_dev : n_host;
  const uint64_t chunk = (N + gridDim.x - 1) / gridDim.x;
  const uint64_t lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  uint32_t run = block_sums[blockIdx.x];
  for (uint64_t base = lo; base < hi; base += blockDim.x) {
    uint64_t i = base + threadIdx.x;
    uint32_t v = i < hi ? a[i] : 0;
    uint32_t tot;
    uint32_t ex = cta_scan_excl(v, &tot, sh);
    if (i < hi) a[i] = run + ex;
    run += tot;
  }
}

static void gscan(uint32_t* a, uint64_t n_host, const uint32_t* n_dev, uint32_t* block_sums,
                  uint32_t* total_out, cudaStream_t st) {
  k_gscan1<<<kScanBlocks, 256, 0, st>>>(a, n_host, n_dev, block_sums);
  k_gscan2<<<1, kScanBlocks, 0, st>>>(block_sums, kScanBlocks, total_out);
  k_gscan3<<<kScanBlocks, 256, 0, st>>>(a, n_host, n_dev, block_sums);
}

// ---- radix passes; the first pass reads new_out directly (key = index) and
// drops empty slots
// a slot of new_out the first pass keeps: filled, and owned by this rank
__device__ __forceinline__ bool owned_pair(uint32_t t, uint32_t world, uint32_t rank) {
  return t != DD_NONE && (world == 1 || t % world == rank);
}

__global__ void __launch_bounds__(kRadixThreads) k_radix_hist(const uint32_t* t_in,
                                                              const uint32_t* counters, uint64_t E,
                                                              int first, int shift, uint32_t G,
                                                              uint32_t* hist, uint32_t world,
                                                              uint32_t rank) {
  __shared__ uint32_t h[256];
  const uint32_t tid = threadIdx.x;
  h[tid] = 0;
  __syncthreads();
  const uint64_t len = first ? E : counters[0];
  const uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
  for (uint32_t it = 0; it < kRadixItems; it++) {
    uint64_t i = base + (uint64_t)it * kRadixThreads + tid;
    if (i < len) {
      uint32_t t = t_in[i];
      if (!first || owned_pair(t, world, rank)) atomicAdd(&h[(t >> shift) & 255u], 1u);
    }
  }
  __syncthreads();
  hist[(uint64_t)tid * G + blockIdx.x] = h[tid];
}

__global__ void __launch_bounds__(kRadixThreads) k_radix_scatter(
    const uint32_t* t_in, const uint32_t* v_in, const uint32_t* counters, uint64_t E, int first,
    int shift, uint32_t G, const uint32_t* hist, uint32_t* t_out, uint32_t* v_out,
    uint32_t world, uint32_t rank) {
  __shared__ uint32_t run[256];
  __shared__ uint32_t boff[256];
  __shared__ uint32_t wcnt[kRadixThreads / 32][256];
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  run[tid] = 0;
  boff[tid] = hist[(uint64_t)tid * G + blockIdx.x];
  const uint64_t len = first ? E : counters[0];
  const uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
  uint32_t lt;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
  __syncthreads();
  for (uint32_t it = 0; it < kRadixItems; it++) {
    const uint64_t i = base + (uint64_t)it * kRadixThreads + tid;
    bool valid = i < len;
    uint32_t t = 0, v = 0;
    if (valid) {
      t = t_in[i];
      v = first ? (uint32_t)i : v_in[i];
      if (first && !owned_pair(t, world, rank)) valid = false;
    }
    const uint32_t dig = (t >> shift) & 255u;
    for (uint32_t d = lane; d < 256; d += 32) wcnt[warp][d] = 0;
    __syncwarp();
    const uint32_t m = __match_any_sync(0xffffffffu, valid ? dig : (0x100u | lane));
    const uint32_t wr = __popc(m & lt);
    if (valid && wr == 0) wcnt[warp][dig] = __popc(m);
    __syncthreads();
    if (valid) {
      uint32_t pre = 0;
      for (uint32_t w = 0; w < warp; w++) pre += wcnt[w][dig];
      const uint32_t pos = boff[dig] + run[dig] + pre + wr;
      t_out[pos] = t;
      v_out[pos] = v;
    }
    __syncthreads();
    uint32_t s = 0;
    for (uint32_t w = 0; w < kRadixThreads / 32; w++) s += wcnt[w][tid];
    run[tid] += s;
    __syncthreads();
  }
}

// ---- segment heads: flags, scan, scatter
__global__ void k_head_flags(const uint32_t* t, const uint32_t* counters, uint64_t E,
                             uint32_t* flags) {
  const uint64_t V = counters[0];
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < V;
       i += (uint64_t)gridDim.x * blockDim.x)
    flags[i] = (i == 0 || t[i] != t[i - 1]) ? 1u : 0u;
}

__global__ void k_head_scatter(const uint32_t* t, const uint32_t* counters, const uint32_t* pos,
                               uint32_t* heads) {
  const uint64_t V = counters[0];
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < V;
       i += (uint64_t)gridDim.x * blockDim.x)
    if (i == 0 || t[i] != t[i - 1]) heads[pos[i]] = (uint32_t)i;
}

int launch_semisort(const uint32_t* new_out, uint64_t E, uint64_t n, SemisortScratch& s,
                    cudaStream_t st) {
  const uint32_t G = (uint32_t)((E + kRadixTile - 1) / kRadixTile);
  int bits = 1;
  while (bits < 32 && ((uint64_t)1 << bits) < n) bits++;
  const int passes = (bits + 7) / 8;
  const uint32_t* tin = new_out;
  const uint32_t* vin = nullptr;
  int cur = 0;
  for (int p = 0; p < passes; p++) {
    const int first = p == 0;
    k_radix_hist<<<G, kRadixThreads, 0, st>>>(tin, s.counters, E, first, 8 * p, G, s.hist,
                                              s.world, s.rank);
    gscan(s.hist, 256ull * G, nullptr, s.block_sums, first ? &s.counters[0] : nullptr, st);
    k_radix_scatter<<<G, kRadixThreads, 0, st>>>(tin, vin, s.counters, E, first, 8 * p, G, s.hist,
                                                 s.t[cur], s.v[cur], s.world, s.rank);
    tin = s.t[cur];
    vin = s.v[cur];
    cur ^= 1;
  }
  const int res = cur ^ 1;
  const int g = (int)std::min<uint64_t>((E + 255) / 256, 4096);
  k_head_flags<<<g, 256, 0, st>>>(s.t[res], s.counters, E, s.flags);
  gscan(s.flags, 0, &s.counters[0], s.block_sums, &s.counters[1], st);
  k_head_scatter<<<g, 256, 0, st>>>(s.t[res], s.counters, s.flags, s.heads);
  return res;
}

}  // namespace ddk
