// Device kernels of the B200 Vamana hot path.
//
//   k_search_prune : one warp per batch point: beam_search on the round-start
//                    graph, then robustPrune of the visited list
//                    (include/index.h:274-285; src/bsp_index.hpp:259-277)
//   k_apply_rows   : update_neighbors of the batch (src/bsp_index.hpp:354-357)
//   k_emit_count / scan / k_scatter : flatten (target, source) pairs and group
//                    them by target keeping batch order inside a target
//                    (src/bsp_index.hpp:362-376, parlay group_by_key)
//   k_reverse      : one warp per target: append, or robustPrune when the row
//                    would overflow R (src/bsp_index.hpp:384-407)
//   k_query        : searchAll (include/utils/beamSearch.h:314-346), mixed L
//   k_gt_*         : brute-force ground truth (FP64 for float data)
#include <cfloat>
#include <cstdio>

#include "dd_common.cuh"
#include "kernels.cuh"
#include "prune_core.cuh"
#include "search_core.cuh"
#include "sort_emul.cuh"

namespace ddk {

static __host__ __device__ inline uint32_t r16(uint64_t x) { return (uint32_t)((x + 15) & ~(uint64_t)15); }

WarpLayout make_search_layout(uint32_t d, int dtype, uint32_t L, uint32_t Rp, uint32_t vcap,
                              bool with_prune) {
  WarpLayout w{};
  uint32_t esz = dtype == DD_F32 ? 4 : 1;
  uint32_t off = 0;
  w.qv = off; off += r16((uint64_t)d * esz);
  w.fr_id = off; off += r16(4ull * L);
  w.fr_d = off; off += r16(4ull * L);
  w.c_id = off; off += r16(4ull * Rp);
  w.c_d = off; off += r16(4ull * Rp);
  w.s_id = off; off += r16(4ull * Rp);
  w.s_d = off; off += r16(4ull * Rp);
  w.vcap = vcap;
  w.ccap = vcap + Rp;
  w.vis_id = off; off += r16(4ull * w.ccap);
  w.vis_d = off; off += r16(4ull * w.ccap);
  w.hbits = hash_bits_for(L);
  w.ws = off;
  uint32_t hash_bytes = 4u << w.hbits;
  uint32_t ev_bytes = r16(4ull * vcap);
  uint32_t search_ws = hash_bytes + ev_bytes;
  uint32_t prune_ws = 0;
  if (with_prune)
    prune_ws = r16(4ull * w.ccap) * 2 + r16(4ull * ddsort::stack_ints((int)w.ccap)) + 16;
  off += search_ws > prune_ws ? search_ws : prune_ws;
  w.total = r16(off);
  return w;
}

struct WarpPtrs {
  SearchSmem S;
  PruneSmem Pm;
};

__device__ __forceinline__ WarpPtrs carve(uint8_t* base, const WarpLayout& w) {
  WarpPtrs r;
  r.S.qv = base + w.qv;
  r.S.fr_id = (uint32_t*)(base + w.fr_id);
  r.S.fr_d = (float*)(base + w.fr_d);
  r.S.c_id = (uint32_t*)(base + w.c_id);
  r.S.c_d = (float*)(base + w.c_d);
  r.S.s_id = (uint32_t*)(base + w.s_id);
  r.S.s_d = (float*)(base + w.s_d);
  r.S.vis_id = (uint32_t*)(base + w.vis_id);
  r.S.vis_d = (float*)(base + w.vis_d);
  r.S.hash = (uint32_t*)(base + w.ws);
  r.S.ev_id = (uint32_t*)(base + w.ws + (4u << w.hbits));
  // prune workspace overlays the hash region (dead after the search)
  r.Pm.cid = r.S.vis_id;
  r.Pm.ckey = r.S.vis_d;
  uint8_t* ws = base + w.ws;
  uint32_t lb = r16(4ull * w.ccap);
  r.Pm.leaf_lo = (int*)ws;
  r.Pm.leaf_hi = (int*)(ws + lb);
  r.Pm.stack = (int*)(ws + 2 * lb);
  r.Pm.scalar = (int*)(ws + 2 * lb + r16(4ull * ddsort::stack_ints((int)w.ccap)));
  return r;
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

// ============================================================ build round
template <int DT, int MT>
__global__ void __launch_bounds__(128) k_search_prune(IndexView ix, RoundArgs ra, WarpLayout lay) {
  extern __shared__ uint4 smem_raw[];
  const uint32_t wpc = blockDim.x >> 5;
  const uint32_t wic = threadIdx.x >> 5;
  const uint32_t lane = lane_id();
  WarpPtrs W = carve((uint8_t*)smem_raw + (size_t)wic * lay.total, lay);
  SearchParams P;
  P.points = ix.points; P.stride = ix.stride; P.graph = ix.graph; P.Rp = ix.Rp; P.n = ix.n;
  P.d = ix.d; P.start = ra.start; P.L = ra.L; P.k = 0; P.cut = 0.0; P.limit = ix.n;
  P.degree_limit = ix.R; P.hbits = lay.hbits; P.vcap = lay.vcap; P.query_mode = 0;
  P.keep_visited = 1; P.err = ix.err;
  const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
  for (uint64_t b = (uint64_t)blockIdx.x * wpc + wic; b < ra.B; b += (uint64_t)gridDim.x * wpc) {
    const uint32_t p = (uint32_t)(ra.floor + b);
    load_vec(W.S.qv, ix.points + (uint64_t)p * ix.stride, qb);
    __syncwarp();
    SearchOut o = warp_beam_search<DT, MT>(P, W.S, p);
    uint32_t m = o.vis_n;
    // the reference's visited list is sorted by (dist, id)
    warp_sort_pairs(W.S.vis_id, W.S.vis_d, m);
    // robustPrune adds p's current out-list (round-start snapshot)
    const uint32_t* prow = ix.graph + (uint64_t)p * ix.Rp;
    for (uint32_t base = 0; base < ix.Rp; base += 32) {
      uint32_t j = base + lane;
      uint32_t a = (j < ix.Rp) ? prow[j] : DD_NONE;
      bool v = a != DD_NONE;
      uint32_t vb = __ballot_sync(0xffffffffu, v);
      if (v) {
        uint32_t pos = m + __popc(vb & lanemask_lt());
        W.Pm.cid[pos] = a;
        W.Pm.ckey[pos] = Dist<DT, MT>::eval(W.S.qv, ix.points + (uint64_t)a * ix.stride, ix.d);
      }
      m += __popc(vb);
    }
    __syncwarp();
    warp_std_sort(W.Pm, m);
    warp_greedy_select<DT, MT>(ix.points, ix.stride, ix.d, p, W.Pm, m, ra.alpha, ix.R,
                               ra.new_out + b * ix.Rp, ix.Rp);
    if (lane == 0) {
      if (ra.stat_vis) ra.stat_vis[b] = o.vis_n;
      if (ra.stat_cmps) ra.stat_cmps[b] = o.cmps;
    }
    __syncwarp();
  }
}

__global__ void k_apply_rows(uint32_t* graph, const uint32_t* new_out, uint64_t floor,
                             uint64_t nvec, uint32_t Rp) {
  // rows are Rp uint32 = Rp/4 uint4; batch rows are contiguous in the graph
  const uint4* src = (const uint4*)new_out;
  uint4* dst = (uint4*)(graph + floor * Rp);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvec;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

__global__ void k_emit_count(const uint32_t* new_out, uint64_t total, uint32_t* cnt,
                             uint32_t* touched, uint32_t* counters) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t t = new_out[i];
    if (t == DD_NONE) continue;
    if (atomicAdd(&cnt[t], 1u) == 0u) touched[atomicAdd(&counters[0], 1u)] = t;
  }
}

// ---- exclusive scan of cnt[touched[i]] over the touched list (length in counters[0])
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total, uint32_t* sh) {
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < nw ? sh[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= (uint32_t)o) s += y;
    }
    if (lane < nw) sh[lane] = s;
  }
  __syncthreads();
  uint32_t wbase = w ? sh[w - 1] : 0;
  *total = sh[nw - 1];
  __syncthreads();
  return wbase + x - v;
}

__global__ void k_scan1(const uint32_t* touched, const uint32_t* cnt, const uint32_t* counters,
                        uint32_t* block_sums) {
  uint32_t T = counters[0];
  uint32_t chunk = (T + gridDim.x - 1) / gridDim.x;
  uint32_t lo = blockIdx.x * chunk, hi = min(T, lo + chunk);
  uint32_t s = 0;
  for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s += cnt[touched[i]];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ uint32_t sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (uint32_t w = 0; w < (blockDim.x >> 5); w++) t += sh[w];
    block_sums[blockIdx.x] = t;
  }
}

__global__ void k_scan2(uint32_t* block_sums, int nb) {
  __shared__ uint32_t sh[32];
  uint32_t v = threadIdx.x < (uint32_t)nb ? block_sums[threadIdx.x] : 0;
  uint32_t tot;
  uint32_t ex = block_exclusive_scan(v, &tot, sh);
  if (threadIdx.x < (uint32_t)nb) block_sums[threadIdx.x] = ex;
}

__global__ void k_scan3(const uint32_t* touched, const uint32_t* cnt, const uint32_t* counters,
                        const uint32_t* block_sums, uint32_t* seg_start, uint32_t* cursor) {
  __shared__ uint32_t sh[32];
  uint32_t T = counters[0];
  uint32_t chunk = (T + gridDim.x - 1) / gridDim.x;
  uint32_t lo = blockIdx.x * chunk, hi = min(T, lo + chunk);
  uint32_t run = block_sums[blockIdx.x];
  for (uint32_t base = lo; base < hi; base += blockDim.x) {
    uint32_t i = base + threadIdx.x;
    uint32_t t = i < hi ? touched[i] : 0;
    uint32_t v = i < hi ? cnt[t] : 0;
    uint32_t tot;
    uint32_t ex = block_exclusive_scan(v, &tot, sh);
    if (i < hi) {
      seg_start[i] = run + ex;
      cursor[t] = run + ex;
    }
    run += tot;
  }
}

__global__ void k_scatter(const uint32_t* new_out, uint64_t total, uint32_t* cursor,
                          uint32_t* keys) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t t = new_out[i];
    if (t == DD_NONE) continue;
    keys[atomicAdd(&cursor[t], 1u)] = (uint32_t)i;  // i = b*Rp + j: batch order
  }
}

// per-warp shared layout of the reverse kernel
struct RevLayout {
  uint32_t tv, keys, cid, ckey, lo, hi, stack, scalar, total;
};
__host__ __device__ inline RevLayout rev_layout(uint32_t d, int dtype) {
  RevLayout r;
  uint32_t off = 0;
  uint32_t esz = dtype == DD_F32 ? 4 : 1;
  auto a16 = [](uint64_t x) { return (uint32_t)((x + 15) & ~(uint64_t)15); };
  r.tv = off; off += a16((uint64_t)d * esz);
  r.keys = off; off += a16(4ull * kRevCandCap);
  r.cid = off; off += a16(4ull * kRevCandCap);
  r.ckey = off; off += a16(4ull * kRevCandCap);
  r.lo = off; off += a16(4ull * kRevCandCap);
  r.hi = off; off += a16(4ull * kRevCandCap);
  r.stack = off; off += a16(4ull * ddsort::stack_ints((int)kRevCandCap));
  r.scalar = off; off += 16;
  r.total = off;
  return r;
}

// Append the (sorted) sources, or prune when the row would exceed R.
// `sk` holds the s segment keys sorted ascending.
template <int DT, int MT>
__device__ void reverse_one(const IndexView& ix, const RoundArgs& ra, uint32_t t, uint32_t s,
                            const uint32_t* sk, uint32_t deg, uint8_t* tv, PruneSmem Pm,
                            uint32_t* counters) {
  const uint32_t lane = lane_id();
  uint32_t* row = ix.graph + (uint64_t)t * ix.Rp;
  if (s + deg <= ix.R) {
    for (uint32_t j = lane; j < s; j += 32) row[deg + j] = (uint32_t)(ra.floor + sk[j] / ix.Rp);
    __syncwarp();
    return;
  }
  const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
  load_vec(tv, ix.points + (uint64_t)t * ix.stride, qb);
  __syncwarp();
  for (uint32_t j = lane; j < s; j += 32) {
    uint32_t c = (uint32_t)(ra.floor + sk[j] / ix.Rp);
    Pm.cid[j] = c;
    Pm.ckey[j] = Dist<DT, MT>::eval(tv, ix.points + (uint64_t)c * ix.stride, ix.d);
  }
  for (uint32_t j = lane; j < deg; j += 32) {
    uint32_t c = row[j];
    Pm.cid[s + j] = c;
    Pm.ckey[s + j] = Dist<DT, MT>::eval(tv, ix.points + (uint64_t)c * ix.stride, ix.d);
  }
  __syncwarp();
  const uint32_t m = s + deg;
  warp_std_sort(Pm, m);
  warp_greedy_select<DT, MT>(ix.points, ix.stride, ix.d, t, Pm, m, ra.alpha, ix.R, row, ix.Rp);
  if (lane == 0) {
    atomicAdd(&counters[2], 1u);
    atomicAdd(&counters[3], m);
  }
}

template <int DT, int MT>
__global__ void __launch_bounds__(kRevWarps * 32) k_reverse(IndexView ix, RoundArgs ra, ReverseScratch rs) {
  extern __shared__ uint4 smem_raw[];
  const RevLayout L = rev_layout(ix.d, DT);
  const uint32_t wic = threadIdx.x >> 5, lane = lane_id();
  uint8_t* base = (uint8_t*)smem_raw + (size_t)wic * L.total;
  uint32_t* sk = (uint32_t*)(base + L.keys);
  PruneSmem Pm{(uint32_t*)(base + L.cid), (float*)(base + L.ckey), (int*)(base + L.lo),
               (int*)(base + L.hi), (int*)(base + L.stack), (int*)(base + L.scalar)};
  const uint32_t T = rs.counters[0];
  for (uint32_t i = blockIdx.x * kRevWarps + wic; i < T; i += gridDim.x * kRevWarps) {
    const uint32_t t = rs.touched[i];
    const uint32_t s = rs.cnt[t];
    const uint32_t st0 = rs.seg_start[i];
    const uint32_t deg = row_degree(ix.graph + (uint64_t)t * ix.Rp, ix.Rp);
    if (s + deg > kRevCandCap) {
      if (lane == 0) rs.big[atomicAdd(&rs.counters[1], 1u)] = i;
      continue;  // handled by k_reverse_big (which also clears cnt[t])
    }
    for (uint32_t j = lane; j < s; j += 32) sk[j] = rs.keys[st0 + j];
    __syncwarp();
    warp_sort_u32(sk, s);
    reverse_one<DT, MT>(ix, ra, t, s, sk, deg, base + L.tv, Pm, rs.counters);
    if (lane == 0) rs.cnt[t] = 0;
    __syncwarp();
  }
}

// Large targets: same logic with the candidate workspace in global memory.
// One warp per entry; `slot` selects this warp's workspace slice.
template <int DT, int MT>
__global__ void k_reverse_big(IndexView ix, RoundArgs ra, ReverseScratch rs) {
  __shared__ __align__(16) uint8_t tvbuf[4 * 1024];
  __shared__ int scalar[4];
  const uint32_t lane = lane_id();
  const uint32_t slot = blockIdx.x;
  uint32_t* cid = rs.gcand + (uint64_t)slot * rs.gcap;
  float* ckey = rs.gkey + (uint64_t)slot * rs.gcap;
  int* lo = rs.gleaf + (uint64_t)slot * (2 * rs.gcap + ddsort::stack_ints((int)rs.gcap));
  int* hi = lo + rs.gcap;
  int* stack = hi + rs.gcap;
  PruneSmem Pm{cid, ckey, lo, hi, stack, scalar};
  const uint32_t nbig = rs.counters[1];
  for (uint32_t e = slot; e < nbig; e += gridDim.x) {
    const uint32_t i = rs.big[e];
    const uint32_t t = rs.touched[i];
    const uint32_t s = rs.cnt[t];
    const uint32_t st0 = rs.seg_start[i];
    const uint32_t deg = row_degree(ix.graph + (uint64_t)t * ix.Rp, ix.Rp);
    if ((uint64_t)s + deg > rs.gcap) {
      if (lane == 0) dd_set_error(ix.err, DD_ESEG_CAP);
      continue;
    }
    // the segment keys are sorted in place in the key buffer
    uint32_t* sk = rs.keys + st0;
    warp_sort_u32(sk, s);
    reverse_one<DT, MT>(ix, ra, t, s, sk, deg, tvbuf, Pm, rs.counters);
    if (lane == 0) rs.cnt[t] = 0;
    __syncwarp();
  }
}

// ============================================================ queries
template <int DT, int MT>
__global__ void __launch_bounds__(128) k_query(IndexView ix, QueryArgs qa, WarpLayout lay) {
  extern __shared__ uint4 smem_raw[];
  const uint32_t wpc = blockDim.x >> 5, wic = threadIdx.x >> 5, lane = lane_id();
  WarpPtrs W = carve((uint8_t*)smem_raw + (size_t)wic * lay.total, lay);
  const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
  for (uint64_t q = (uint64_t)blockIdx.x * wpc + wic; q < qa.nq; q += (uint64_t)gridDim.x * wpc) {
    SearchParams P;
    P.points = ix.points; P.stride = ix.stride; P.graph = ix.graph; P.Rp = ix.Rp; P.n = ix.n;
    uint32_t Lq = qa.Ls[q];
    if (Lq == 0 || Lq > qa.Lmax || Lq < qa.k) {
      if (lane == 0) dd_set_error(ix.err, DD_ECAND_CAP);
      Lq = qa.Lmax;
    }
    P.d = ix.d; P.start = qa.start; P.L = Lq; P.k = qa.k; P.cut = qa.cut; P.limit = qa.limit;
    P.degree_limit = qa.degree_limit; P.hbits = hash_bits_for(P.L); P.vcap = lay.vcap;
    P.query_mode = 1; P.keep_visited = 0; P.err = ix.err;
    load_vec(W.S.qv, qa.queries + q * qa.qstride, qb);
    __syncwarp();
    SearchOut o = warp_beam_search<DT, MT>(P, W.S, qa.skip_self ? q : (uint64_t)-1);
    for (uint32_t j = lane; j < qa.k; j += 32) {
      bool v = j < o.fr_n;
      qa.ids[q * qa.k + j] = v ? (W.S.fr_id[j] & ~DD_VBIT) : DD_NONE;
      qa.dists[q * qa.k + j] = v ? W.S.fr_d[j] : INFINITY;
    }
    if (lane == 0) {
      if (qa.visited) qa.visited[q] = o.vis_n;
      if (qa.cmps) qa.cmps[q] = o.cmps;
    }
    __syncwarp();
  }
}

template <int DT, int MT>
__global__ void __launch_bounds__(32) k_beam(IndexView ix, BeamArgs ba, WarpLayout lay) {
  extern __shared__ uint4 smem_raw[];
  const uint32_t lane = lane_id();
  WarpPtrs W = carve((uint8_t*)smem_raw, lay);
  const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
  for (uint64_t q = blockIdx.x; q < ba.nq; q += gridDim.x) {
    SearchParams P;
    P.points = ix.points; P.stride = ix.stride; P.graph = ix.graph; P.Rp = ix.Rp; P.n = ix.n;
    P.d = ix.d; P.start = ba.start; P.L = ba.L; P.k = ba.k; P.cut = ba.cut; P.limit = ba.limit;
    P.degree_limit = ba.degree_limit; P.hbits = lay.hbits; P.vcap = lay.vcap;
    P.query_mode = ba.k > 0; P.keep_visited = 1; P.err = ix.err;
    load_vec(W.S.qv, ba.queries + q * ba.qstride, qb);
    __syncwarp();
    SearchOut o = warp_beam_search<DT, MT>(P, W.S, (uint64_t)ba.self_ids[q]);
    warp_sort_pairs(W.S.vis_id, W.S.vis_d, o.vis_n);
    for (uint32_t j = lane; j < o.fr_n; j += 32) {
      ba.fr_ids[q * ba.L + j] = W.S.fr_id[j] & ~DD_VBIT;
      ba.fr_d[q * ba.L + j] = W.S.fr_d[j];
    }
    for (uint32_t j = lane; j < o.vis_n; j += 32) {
      ba.vis_ids[q * ba.vcap + j] = W.S.vis_id[j];
      ba.vis_d[q * ba.vcap + j] = W.S.vis_d[j];
    }
    if (lane == 0) {
      ba.fr_n[q] = o.fr_n;
      ba.vis_n[q] = o.vis_n;
      ba.cmps[q] = o.cmps;
    }
    __syncwarp();
  }
}

// robustPrune on explicit candidate lists: one warp per task, global workspace
template <int DT, int MT>
__global__ void k_prune_tasks(IndexView ix, PruneArgs pa) {
  __shared__ int scalar[4];
  const uint32_t lane = lane_id();
  for (uint32_t t = blockIdx.x; t < pa.ntasks; t += gridDim.x) {
    const uint32_t p = pa.p[t];
    const uint64_t o0 = pa.offsets[t], o1 = pa.offsets[t + 1];
    const uint64_t wbase = o0 + (uint64_t)t * ix.Rp;  // room for the out-list too
    const uint64_t cap = (o1 - o0) + ix.Rp;
    uint32_t* cid = pa.gcand + wbase;
    float* ckey = pa.gkey + wbase;
    int* lo = pa.gleaf + 2 * wbase + (uint64_t)t * kGlobalStackInts;
    int* hi = lo + cap;
    int* stack = hi + cap;
    uint32_t m = (uint32_t)(o1 - o0);
    for (uint32_t j = lane; j < m; j += 32) {
      cid[j] = pa.cand_ids[o0 + j];
      ckey[j] = pa.cand_d[o0 + j];
    }
    const uint32_t* prow = ix.graph + (uint64_t)p * ix.Rp;
    const uint8_t* pv = ix.points + (uint64_t)p * ix.stride;
    for (uint32_t base = 0; base < ix.Rp; base += 32) {
      uint32_t j = base + lane;
      uint32_t a = j < ix.Rp ? prow[j] : DD_NONE;
      bool v = a != DD_NONE;
      uint32_t vb = __ballot_sync(0xffffffffu, v);
      if (v) {
        uint32_t pos = m + __popc(vb & lanemask_lt());
        cid[pos] = a;
        ckey[pos] = Dist<DT, MT>::eval(pv, ix.points + (uint64_t)a * ix.stride, ix.d);
      }
      m += __popc(vb);
    }
    __syncwarp();
    PruneSmem Pm{cid, ckey, lo, hi, stack, scalar};
    warp_std_sort(Pm, m);
    warp_greedy_select<DT, MT>(ix.points, ix.stride, ix.d, p, Pm, m, pa.alpha, ix.R,
                               pa.out + (uint64_t)t * ix.Rp, ix.Rp);
  }
}

// knn_index final step (include/index.h:133-136): per-row std::sort of the
// neighbour ids by distance to the row's owner (ties in library order)
template <int DT, int MT>
__global__ void __launch_bounds__(32) k_sort_rows(IndexView ix) {
  __shared__ uint32_t cid[kMaxRp];
  __shared__ float ckey[kMaxRp];
  __shared__ int lo[kMaxRp], hi[kMaxRp];
  __shared__ int stack[64];
  __shared__ int scalar[4];
  const uint32_t lane = lane_id();
  for (uint64_t v = blockIdx.x; v < ix.n; v += gridDim.x) {
    uint32_t* row = ix.graph + v * ix.Rp;
    const uint8_t* pv = ix.points + v * ix.stride;
    uint32_t deg = row_degree(row, ix.Rp);
    for (uint32_t j = lane; j < deg; j += 32) {
      cid[j] = row[j];
      ckey[j] = Dist<DT, MT>::eval(pv, ix.points + (uint64_t)row[j] * ix.stride, ix.d);
    }
    __syncwarp();
    PruneSmem Pm{cid, ckey, lo, hi, stack, scalar};
    warp_std_sort(Pm, deg);
    for (uint32_t j = lane; j < deg; j += 32) row[j] = cid[j];
    __syncwarp();
  }
}

// ============================================================ ground truth
template <int DT, int MT>
__device__ __forceinline__ double exact_dist64(const uint8_t* q, const uint8_t* x, uint32_t d) {
  if (DT == DD_F32) {
    const float* a = (const float*)q;
    const float* b = (const float*)x;
    double acc = 0.0;
    for (uint32_t t = 0; t < d; t++) {
      if (MT == DD_L2) {
        double df = __dsub_rn((double)a[t], (double)__ldg(b + t));
        acc = __dadd_rn(acc, __dmul_rn(df, df));
      } else {
        acc = __dsub_rn(acc, __dmul_rn((double)a[t], (double)__ldg(b + t)));
      }
    }
    return acc;
  } else {
    return (double)DistIntRaw<DT, MT>::eval(q, x, d);  // exact int32 (d < 33025)
  }
}

// grid (query blocks of 8 warps, chunks); each warp keeps a top-k (k <= 32)
// sorted across its lanes by (distance, id)
template <int DT, int MT>
__global__ void __launch_bounds__(256) k_gt_partial(IndexView ix, const uint8_t* queries, uint64_t qstride,
                                                    uint64_t nq, uint32_t k, uint32_t nchunks,
                                                    double* part_d, uint32_t* part_i) {
  __shared__ __align__(16) uint8_t qbuf[8][1024];
  const uint32_t wic = threadIdx.x >> 5, lane = lane_id();
  const uint64_t q = (uint64_t)blockIdx.x * 8 + wic;
  if (q >= nq) return;
  const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
  load_vec(qbuf[wic], queries + q * qstride, qb);
  __syncwarp();
  const uint64_t chunk = (ix.n + nchunks - 1) / nchunks;
  const uint64_t c0 = (uint64_t)blockIdx.y * chunk;
  const uint64_t c1 = min(ix.n, c0 + chunk);
  double bd = INFINITY;
  uint32_t bi = DD_NONE;
  for (uint64_t base = c0; base < c1; base += 32) {
    uint64_t i = base + lane;
    double dv = INFINITY;
    uint32_t iv = DD_NONE;
    if (i < c1) {
      dv = exact_dist64<DT, MT>(qbuf[wic], ix.points + i * ix.stride, ix.d);
      iv = (uint32_t)i;
    }
    double td = __shfl_sync(0xffffffffu, bd, k - 1);
    uint32_t ti = __shfl_sync(0xffffffffu, bi, k - 1);
    bool cand = (dv < td) || (dv == td && iv < ti);
    uint32_t mask = __ballot_sync(0xffffffffu, cand);
    while (mask) {
      int src = __ffs(mask) - 1;
      mask &= mask - 1;
      double cd = __shfl_sync(0xffffffffu, dv, src);
      uint32_t ci = __shfl_sync(0xffffffffu, iv, src);
      double kd = __shfl_sync(0xffffffffu, bd, k - 1);
      uint32_t ki = __shfl_sync(0xffffffffu, bi, k - 1);
      if (!((cd < kd) || (cd == kd && ci < ki))) continue;
      bool before = (lane < k) && ((bd < cd) || (bd == cd && bi < ci));
      uint32_t pos = __popc(__ballot_sync(0xffffffffu, before));
      double ud = __shfl_up_sync(0xffffffffu, bd, 1);
      uint32_t ui = __shfl_up_sync(0xffffffffu, bi, 1);
      if (lane == pos) { bd = cd; bi = ci; }
      else if (lane > pos) { bd = ud; bi = ui; }
    }
  }
  if (lane < k) {
    uint64_t o = (q * nchunks + blockIdx.y) * k + lane;
    part_d[o] = bd;
    part_i[o] = bi;
  }
}

__global__ void k_gt_merge(const double* part_d, const uint32_t* part_i, uint64_t nq, uint32_t k,
                           uint32_t nchunks, uint32_t* ids, float* dists) {
  const uint32_t lane = lane_id();
  const uint64_t q = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= nq) return;
  double bd = INFINITY;
  uint32_t bi = DD_NONE;
  const uint64_t tot = (uint64_t)nchunks * k;
  for (uint64_t base = 0; base < tot; base += 32) {
    uint64_t e = base + lane;
    double dv = e < tot ? part_d[q * tot + e] : INFINITY;
    uint32_t iv = e < tot ? part_i[q * tot + e] : DD_NONE;
    double td = __shfl_sync(0xffffffffu, bd, k - 1);
    uint32_t ti = __shfl_sync(0xffffffffu, bi, k - 1);
    bool cand = (dv < td) || (dv == td && iv < ti);
    uint32_t mask = __ballot_sync(0xffffffffu, cand);
    while (mask) {
      int src = __ffs(mask) - 1;
      mask &= mask - 1;
      double cd = __shfl_sync(0xffffffffu, dv, src);
      uint32_t ci = __shfl_sync(0xffffffffu, iv, src);
      double kd = __shfl_sync(0xffffffffu, bd, k - 1);
      uint32_t ki = __shfl_sync(0xffffffffu, bi, k - 1);
      if (!((cd < kd) || (cd == kd && ci < ki))) continue;
      bool before = (lane < k) && ((bd < cd) || (bd == cd && bi < ci));
      uint32_t pos = __popc(__ballot_sync(0xffffffffu, before));
      double ud = __shfl_up_sync(0xffffffffu, bd, 1);
      uint32_t ui = __shfl_up_sync(0xffffffffu, bi, 1);
      if (lane == pos) { bd = cd; bi = ci; }
      else if (lane > pos) { bd = ud; bi = ui; }
    }
  }
  if (lane < k) {
    ids[q * k + lane] = bi;
    dists[q * k + lane] = (float)bd;
  }
}

// ============================================================ graph formats
__global__ void k_to_ref_rows(const uint32_t* graph, uint64_t n, uint32_t R, uint32_t Rp,
                              uint32_t* out) {
  const uint32_t lane = lane_id();
  for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n;
       v += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
    const uint32_t* row = graph + v * Rp;
    uint32_t* o = out + v * (uint64_t)(R + 1);
    uint32_t deg = 0;
    for (uint32_t base = 0; base < R; base += 32) {
      uint32_t j = base + lane;
      uint32_t a = j < R ? row[j] : DD_NONE;
      deg += __popc(__ballot_sync(0xffffffffu, a != DD_NONE));
      if (j < R) o[1 + j] = a == DD_NONE ? 0u : a;
    }
    if (lane == 0) o[0] = deg;
  }
}

__global__ void k_from_ref_rows(uint32_t* graph, uint64_t n, uint32_t R, uint32_t Rp,
                                const uint32_t* in, uint32_t* err) {
  const uint32_t lane = lane_id();
  for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n;
       v += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
    const uint32_t* r = in + v * (uint64_t)(R + 1);
    uint32_t deg = r[0];
    if (deg > R) {
      if (lane == 0) dd_set_error(err, DD_EDEGREE);
      deg = R;
    }
    for (uint32_t j = lane; j < Rp; j += 32) {
      uint32_t a = j < deg ? r[1 + j] : DD_NONE;
      if (a != DD_NONE && a >= n) {
        dd_set_error(err, DD_EBAD_ID);
        a = DD_NONE;
      }
      graph[v * Rp + j] = a;
    }
  }
}

// ============================================================ launchers
#define DD_DISPATCH(dtype, metric, KERNEL_CALL)                      \
  do {                                                               \
    if ((dtype) == DD_F32 && (metric) == DD_L2) { KERNEL_CALL(DD_F32, DD_L2); }        \
    else if ((dtype) == DD_F32) { KERNEL_CALL(DD_F32, DD_MIPS); }                      \
    else if ((dtype) == DD_I8 && (metric) == DD_L2) { KERNEL_CALL(DD_I8, DD_L2); }     \
    else if ((dtype) == DD_I8) { KERNEL_CALL(DD_I8, DD_MIPS); }                        \
    else if ((metric) == DD_L2) { KERNEL_CALL(DD_U8, DD_L2); }                         \
    else { KERNEL_CALL(DD_U8, DD_MIPS); }                                              \
  } while (0)

template <typename K>
static void set_smem(K kernel, size_t bytes) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

void launch_search_prune(const IndexView& ix, const RoundArgs& ra, const WarpLayout& lay,
                         int wpc, int grid, cudaStream_t st) {
  size_t sm = (size_t)lay.total * wpc;
#define CALL(DT, MT)                                                   \
  set_smem(k_search_prune<DT, MT>, sm);                                \
  k_search_prune<DT, MT><<<grid, wpc * 32, sm, st>>>(ix, ra, lay);
  DD_DISPATCH(ix.dtype, ix.metric, CALL);
#undef CALL
}

void launch_apply_rows(const IndexView& ix, const RoundArgs& ra, cudaStream_t st) {
  uint64_t nvec = (uint64_t)ra.B * ix.Rp / 4;
  if (!nvec) return;
  int grid = (int)std::min<uint64_t>((nvec + 255) / 256, 4096);
  k_apply_rows<<<grid, 256, 0, st>>>(ix.graph, ra.new_out, ra.floor, nvec, ix.Rp);
}

void launch_reverse(const IndexView& ix, const RoundArgs& ra, const ReverseScratch& rs,
                    cudaStream_t st, int sm_count) {
  uint64_t total = (uint64_t)ra.B * ix.Rp;
  if (!total) return;
  int g = (int)std::min<uint64_t>((total + 255) / 256, (uint64_t)sm_count * 16);
  k_emit_count<<<g, 256, 0, st>>>(ra.new_out, total, rs.cnt, rs.touched, rs.counters);
  k_scan1<<<kScanBlocks, 256, 0, st>>>(rs.touched, rs.cnt, rs.counters, rs.block_sums);
  k_scan2<<<1, kScanBlocks, 0, st>>>(rs.block_sums, kScanBlocks);
  k_scan3<<<kScanBlocks, 256, 0, st>>>(rs.touched, rs.cnt, rs.counters, rs.block_sums,
                                       rs.seg_start, rs.cursor);
  k_scatter<<<g, 256, 0, st>>>(ra.new_out, total, rs.cursor, rs.keys);
  RevLayout L = rev_layout(ix.d, ix.dtype);
  size_t sm = (size_t)L.total * kRevWarps;
  int rg = sm_count * 8;
#define CALL(DT, MT)                                                    \
  set_smem(k_reverse<DT, MT>, sm);                                      \
  k_reverse<DT, MT><<<rg, kRevWarps * 32, sm, st>>>(ix, ra, rs);
  DD_DISPATCH(ix.dtype, ix.metric, CALL);
#undef CALL
}

void launch_reverse_big(const IndexView& ix, const RoundArgs& ra, const ReverseScratch& rs,
                        uint32_t slots, cudaStream_t st) {
  // the number of big entries is read on the device; `slots` workspaces exist
  int g = (int)slots;
#define CALL(DT, MT) k_reverse_big<DT, MT><<<g, 32, 0, st>>>(ix, ra, rs);
  DD_DISPATCH(ix.dtype, ix.metric, CALL);
#undef CALL
}

void launch_query(const IndexView& ix, const QueryArgs& qa, const WarpLayout& lay, int wpc,
                  int grid, cudaStream_t st) {
  size_t sm = (size_t)lay.total * wpc;
#define CALL(DT, MT)                                                   \
  set_smem(k_query<DT, MT>, sm);                                       \
  k_query<DT, MT><<<grid, wpc * 32, sm, st>>>(ix, qa, lay);
  DD_DISPATCH(ix.dtype, ix.metric, CALL);
#undef CALL
}

void launch_beam(const IndexView& ix, const BeamArgs& ba, const WarpLayout& lay, cudaStream_t st) {
  size_t sm = lay.total;
  int grid = (int)std::min<uint64_t>(ba.nq, 4096);
#define CALL(DT, MT)                                                   \
  set_smem(k_beam<DT, MT>, sm);                                        \
  k_beam<DT, MT><<<grid, 32, sm, st>>>(ix, ba, lay);
  DD_DISPATCH(ix.dtype, ix.metric, CALL);
#undef CALL
}

void launch_prune_tasks(const IndexView& ix, const PruneArgs& pa, cudaStream_t st) {
  if (!pa.ntasks) return;
  int grid = (int)std::min<uint32_t>(pa.ntasks, 4096);
#define CALL(DT, MT) k_prune_tasks<DT, MT><<<grid, 32, 0, st>>>(ix, pa);
  DD_DISPATCH(ix.dtype, ix.metric, CALL);
#undef CALL
}

void launch_sort_rows(const IndexView& ix, cudaStream_t st) {
  int grid = (int)std::min<uint64_t>(ix.n, 65536);
#define CALL(DT, MT) k_sort_rows<DT, MT><<<grid, 32, 0, st>>>(ix);
  DD_DISPATCH(ix.dtype, ix.metric, CALL);
#undef CALL
}

void launch_groundtruth(const IndexView& ix, const uint8_t* queries, uint64_t qstride, uint64_t nq,
                        uint32_t k, uint32_t* ids, float* dists, double* part_d, uint32_t* part_i,
                        uint32_t nchunks, cudaStream_t st) {
  dim3 grid((unsigned)((nq + 7) / 8), nchunks);
#define CALL(DT, MT)                                                                  \
  k_gt_partial<DT, MT><<<grid, 256, 0, st>>>(ix, queries, qstride, nq, k, nchunks, part_d, part_i);
  DD_DISPATCH(ix.dtype, ix.metric, CALL);
#undef CALL
  k_gt_merge<<<(unsigned)((nq + 7) / 8), 256, 0, st>>>(part_d, part_i, nq, k, nchunks, ids, dists);
}

void launch_to_ref_rows(const IndexView& ix, uint32_t* out, cudaStream_t st) {
  int grid = (int)std::min<uint64_t>((ix.n * 32 + 255) / 256, 65536);
  k_to_ref_rows<<<grid, 256, 0, st>>>(ix.graph, ix.n, ix.R, ix.Rp, out);
}

void launch_from_ref_rows(const IndexView& ix, const uint32_t* in, cudaStream_t st) {
  int grid = (int)std::min<uint64_t>((ix.n * 32 + 255) / 256, 65536);
  k_from_ref_rows<<<grid, 256, 0, st>>>(ix.graph, ix.n, ix.R, ix.Rp, in, ix.err);
}

}  // namespace ddk
