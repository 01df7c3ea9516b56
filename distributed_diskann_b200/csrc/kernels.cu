// Device kernels of the B200 Vamana hot path.
//
//   k_search       : one warp per batch point: beam_search on the round-start
//                    graph; the visited list goes to the point's global slice
//                    (include/index.h:274-278; src/bsp_index.hpp:259-268)
//   k_prune        : one warp per batch point: robustPrune of the visited list
//                    and the point's out-list (include/index.h:279-285;
//                    src/bsp_index.hpp:269-277)
//   k_apply_rows   : update_neighbors of the batch (src/bsp_index.hpp:354-357)
//   k_emit_count / scan / k_scatter : flatten (target, source) pairs and group
//                    them by target keeping batch order inside a target
//                    (src/bsp_index.hpp:362-376, parlay group_by_key)
//   k_reverse      : one warp per target: append, or robustPrune when the row
//                    would overflow R (src/bsp_index.hpp:384-407); targets with
//                    more candidates go to k_reverse_big (one CTA, shared
//                    memory) or, beyond that, k_reverse_huge (global memory)
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

static __host__ __device__ inline uint32_t r16(uint64_t x) {
  return (uint32_t)((x + 15) & ~(uint64_t)15);
}

// Per-warp shared memory of the search kernels:
//   build search: qv | frontier | step candidates | hash table; the visited
//     list goes to the point's slice of a global array (read by k_prune).
//   query / debug: qv | frontier | step candidates | visited | evicted | hash.
// With h24 the hash table stores 24-bit ids (3 bytes a slot instead of 4),
// which is exact whenever every id is below 0xFFFFFF.
WarpLayout make_search_layout(uint32_t d, int dtype, uint32_t L, uint32_t Rp, uint32_t vcap,
                              bool build, bool h24, bool keep_vis) {
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
  w.hbits = hash_bits_for(L);
  w.h24 = h24 ? 1u : 0u;
  const uint32_t hash_bytes = r16(hash_table_bytes(w.hbits, h24));
  if (build) {
    w.vis_id = w.vis_d = 0;  // global
    w.ws = off;
    off += hash_bytes;
  } else {
    w.keep_vis = keep_vis ? 1u : 0u;
    if (keep_vis) {
      w.vis_id = off; off += r16(4ull * vcap);
      w.vis_d = off; off += r16(4ull * vcap);
    }
    w.ws = off; off += r16(4ull * vcap);  // evicted list
    off += hash_bytes;
  }
  w.total = r16(off);
  return w;
}

// Per-warp shared memory of k_prune: p's vector | candidate ids | distances |
// sort workspace, which the fast greedy forms share after the sort.
PruneLayout make_prune_layout(uint32_t d, int dtype, uint32_t Rp, uint32_t ccap) {
  PruneLayout w{};
  uint32_t esz = dtype == DD_F32 ? 4 : 1;
  uint32_t off = 0;
  w.qv = off; off += r16((uint64_t)d * esz);
  w.cid = off; off += r16(4ull * ccap);
  w.ckey = off; off += r16(4ull * ccap);
  w.ws = off; off += prune_ws_bytes_sel(ccap, greedy_sel_bytes(d, dtype, Rp));
  w.ccap = ccap;
  w.total = r16(off);
  return w;
}

// build search: visited list in the global slice vis_g (vcap ids then vcap dists)
__device__ __forceinline__ SearchSmem carve_build(uint8_t* base, const WarpLayout& w, uint32_t* vis_g) {
  SearchSmem S;
  S.qv = base + w.qv;
  S.fr_id = (uint32_t*)(base + w.fr_id);
  S.fr_d = (float*)(base + w.fr_d);
  S.c_id = (uint32_t*)(base + w.c_id);
  S.c_d = (float*)(base + w.c_d);
  S.s_id = (uint32_t*)(base + w.s_id);
  S.s_d = (float*)(base + w.s_d);
  S.vis_id = vis_g;
  S.vis_d = (float*)(vis_g + w.vcap);
  S.ev_id = nullptr;
  S.hash = (uint32_t*)(base + w.ws);
  S.h24 = (int)w.h24;
  return S;
}

// query / debug layout: everything in shared memory
__device__ __forceinline__ SearchSmem carve_query(uint8_t* base, const WarpLayout& w) {
  SearchSmem S;
  S.qv = base + w.qv;
  S.fr_id = (uint32_t*)(base + w.fr_id);
  S.fr_d = (float*)(base + w.fr_d);
  S.c_id = (uint32_t*)(base + w.c_id);
  S.c_d = (float*)(base + w.c_d);
  S.s_id = (uint32_t*)(base + w.s_id);
  S.s_d = (float*)(base + w.s_d);
  S.vis_id = w.keep_vis ? (uint32_t*)(base + w.vis_id) : nullptr;
  S.vis_d = w.keep_vis ? (float*)(base + w.vis_d) : nullptr;
  S.ev_id = (uint32_t*)(base + w.ws);
  S.hash = (uint32_t*)(base + w.ws + r16(4ull * w.vcap));
  S.h24 = (int)w.h24;
  return S;
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
// k_search: one warp per batch point runs beam_search on the round-start graph
// and leaves its visited list in the point's global slice
// (include/index.h:274-278; src/bsp_index.hpp:259-268).
template <int DT, int MT, int FPL, int CPL>
__global__ void __launch_bounds__(512) k_search(IndexView ix, RoundArgs ra, WarpLayout lay) {
  extern __shared__ uint4 smem_raw[];
  const uint32_t wpc = blockDim.x >> 5;
  const uint32_t wic = threadIdx.x >> 5;
  const uint64_t gw = (uint64_t)blockIdx.x * wpc + wic;
  uint8_t* base = (uint8_t*)smem_raw + (size_t)wic * lay.total;
  SearchParams P;
  P.points = ix.points; P.stride = ix.stride; P.graph = ix.graph; P.Rp = ix.Rp; P.n = ix.n;
  P.d = ix.d; P.start = ra.start; P.L = ra.L; P.k = 0; P.cut = 0.0; P.limit = ix.n;
  P.degree_limit = ix.R; P.hbits = lay.hbits; P.vcap = lay.vcap; P.query_mode = 0;
  P.keep_visited = 1; P.err = ix.err;
  const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
  for (uint64_t b = gw; b < ra.B; b += (uint64_t)gridDim.x * wpc) {
    const uint32_t p = (uint32_t)(ra.floor + b);
    const SearchSmem S = carve_build(base, lay, ra.vis_all + b * 2ull * lay.vcap);
    load_vec(S.qv, ix.points + (uint64_t)p * ix.stride, qb);
    __syncwarp();
    const SearchOut o = warp_beam_search<DT, MT, FPL, CPL>(P, S, p);
    if (lane_id() == 0) {
      ra.stat_vis[b] = o.vis_n;
      if (ra.stat_cmps) ra.stat_cmps[b] = o.cmps;
    }
    __syncwarp();
  }
}

// k_prune: one warp per batch point runs robustPrune of its visited list plus
// its current out-list (include/index.h:279-285; src/bsp_index.hpp:269-277).
template <int DT, int MT>
__global__ void __launch_bounds__(512) k_prune(IndexView ix, RoundArgs ra, PruneLayout lay,
                                               uint32_t vcap) {
  extern __shared__ uint4 smem_raw[];
  const uint32_t wpc = blockDim.x >> 5;
  const uint32_t wic = threadIdx.x >> 5;
  const uint32_t lane = lane_id();
  const uint64_t gw = (uint64_t)blockIdx.x * wpc + wic;
  uint8_t* base = (uint8_t*)smem_raw + (size_t)wic * lay.total;
  uint8_t* qv = base + lay.qv;
  PruneSmem Pm = prune_ws((uint32_t*)(base + lay.cid), (float*)(base + lay.ckey), base + lay.ws,
                          lay.ccap);
  Pm.sel = (uint4*)(base + lay.ws + prune_sel_offset(lay.ccap));
  const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
  for (uint64_t b = gw; b < ra.B; b += (uint64_t)gridDim.x * wpc) {
    const uint32_t p = (uint32_t)(ra.floor + b);
    load_vec(qv, ix.points + (uint64_t)p * ix.stride, qb);
    // the visited list, sorted by (dist, id) like the reference's
    const uint32_t* vis = ra.vis_all + b * 2ull * vcap;
    uint32_t m = min(ra.stat_vis[b], vcap);
    for (uint32_t j = lane; j < m; j += 32) {
      Pm.cid[j] = vis[j];
      Pm.ckey[j] = __uint_as_float(vis[vcap + j]);
    }
    __syncwarp();
    warp_sort_pairs(Pm.cid, Pm.ckey, m);
    // robustPrune adds p's current out-list (round-start snapshot)
    const uint32_t* prow = ix.graph + (uint64_t)p * ix.Rp;
    for (uint32_t b0 = 0; b0 < ix.Rp; b0 += 32) {
      const uint32_t j = b0 + lane;
      const uint32_t a = (j < ix.Rp) ? prow[j] : DD_NONE;
      const bool v = a != DD_NONE;
      const uint32_t vb = __ballot_sync(0xffffffffu, v);
      if (v) {
        const uint32_t pos = m + __popc(vb & lanemask_lt());
        Pm.cid[pos] = a;
        Pm.ckey[pos] = Dist<DT, MT>::eval(qv, ix.points + (uint64_t)a * ix.stride, ix.d);
      }
      m += __popc(vb);
    }
    __syncwarp();
    warp_std_sort(Pm, m);
    warp_greedy_select_fast<DT, MT>(ix.points, ix.stride, ix.d, p, Pm, m, ra.alpha, ix.R,
                                    ra.new_out + b * ix.Rp, ix.Rp, Pm.sel);
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

// per-warp shared layout of the reverse kernel
struct RevLayout {
  uint32_t tv, cid, ckey, ws, total;
};
__host__ __device__ inline RevLayout rev_layout(uint32_t d, int dtype, uint32_t Rp) {
  RevLayout r;
  uint32_t off = 0;
  uint32_t esz = dtype == DD_F32 ? 4 : 1;
  const uint32_t sel_bytes = greedy_sel_bytes(d, dtype, Rp);
  r.tv = off; off += r16((uint64_t)d * esz);
  r.cid = off; off += r16(4ull * kRevCandCap);
  r.ckey = off; off += r16(4ull * kRevCandCap);
  r.ws = off; off += prune_ws_bytes_sel(kRevCandCap, sel_bytes);
  r.total = off;
  return r;
}

// The segment of sorted pairs for one target: [start, end) of rs.st / rs.sv.
__device__ __forceinline__ void segment_of(const ReverseScratch& rs, uint32_t k, uint32_t& start,
                                           uint32_t& end) {
  start = rs.heads[k];
  end = (k + 1 < rs.counters[1]) ? rs.heads[k + 1] : rs.counters[0];
}

// Append the sources of segment [start, end) (already in batch order), or
// prune when the row would exceed R (one warp; s + deg <= kRevCandCap).
template <int DT, int MT>
__device__ void reverse_one(const IndexView& ix, const RoundArgs& ra, const ReverseScratch& rs,
                            uint32_t t, uint32_t start, uint32_t s, uint32_t deg, uint8_t* tv,
                            PruneSmem Pm) {
  const uint32_t lane = lane_id();
  uint32_t* row = ix.graph + (uint64_t)t * ix.Rp;
  const uint32_t* sk = rs.sv + start;
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
  // the candidate rows were just read for their distances to t: no prefetch
  warp_greedy_select_fast<DT, MT, false>(ix.points, ix.stride, ix.d, t, Pm, m, ra.alpha, ix.R, row,
                                         ix.Rp, Pm.sel);
  if (lane == 0) {
    atomicAdd(&rs.counters[2], 1u);
    atomicAdd(&rs.counters[3], m);
  }
}

template <int DT, int MT>
__global__ void __launch_bounds__(kRevWarps * 32, 8) k_reverse(IndexView ix, RoundArgs ra, ReverseScratch rs) {
  extern __shared__ uint4 smem_raw[];
  const RevLayout L = rev_layout(ix.d, DT, ix.Rp);
  const uint32_t wic = threadIdx.x >> 5, lane = lane_id();
  uint8_t* base = (uint8_t*)smem_raw + (size_t)wic * L.total;
  PruneSmem Pm = prune_ws((uint32_t*)(base + L.cid), (float*)(base + L.ckey), base + L.ws,
                          kRevCandCap);
  Pm.sel = (uint4*)(base + L.ws + prune_sel_offset(kRevCandCap));
  const uint32_t T = rs.counters[1];
  for (uint32_t k = blockIdx.x * kRevWarps + wic; k < T; k += gridDim.x * kRevWarps) {
    uint32_t start, end;
    segment_of(rs, k, start, end);
    const uint32_t t = rs.st[start];
    const uint32_t s = end - start;
    const uint32_t deg = row_degree(ix.graph + (uint64_t)t * ix.Rp, ix.Rp);
    if (s + deg > kRevCandCap) {
      if (lane == 0) {
        atomicMax(&rs.counters[5], s + deg);  // largest candidate list of the round
        rs.big[atomicAdd(&rs.counters[4], 1u)] = k;
      }
      continue;  // handled by k_reverse_big
    }
    reverse_one<DT, MT>(ix, ra, rs, t, start, s, deg, base + L.tv, Pm);
  }
}

// Targets with more than kRevCandCap candidates: one CTA each, candidates in
// this CTA's global workspace slice.  The sort emulation splits the work:
// ranges longer than cta_range are partitioned by the whole CTA, shorter ones
// by single warps; then all threads finish the leaves.  The greedy selection
// spreads each occlusion pass over the CTA and compacts the survivors while
// the list is long.
//
// The short ranges are recorded in `ranges` (room for cap/8 + 64 records).
// Ranges longer than K at one recursion depth are disjoint and the depth is
// at most 2 log2(m), so there are at most (m / K) * 2 log2(m) + 1 records:
// K = 256 keeps that within m/8 + 1 for m <= 65536, K = 1024 for every m
// below 2^32.
__device__ __forceinline__ int big_cta_range(uint32_t m) { return m <= 65536u ? 256 : 1024; }
constexpr int kBigStackInts = 3 * 72;
// mma_sel_bytes(kMaxRp): staged rows, norms and thresholds of the warp greedy
constexpr uint32_t kBigSelBytes = (kMaxRp + kMmaChunk) * 128u + (kMaxRp + kMmaChunk) * 4u +
                                  kMmaChunk * 4u;

template <int DT, int MT>
__global__ void __launch_bounds__(kBigThreads) k_reverse_big(IndexView ix, RoundArgs ra, ReverseScratch rs) {
  __shared__ __align__(16) uint8_t tv[1024];
  __shared__ uint32_t sh[32];
  __shared__ int cstack[kBigStackInts];
  __shared__ int wstack[kBigThreads / 32][kBigStackInts];
  __shared__ uint32_t s_deg, s_nsmall, s_next, s_mm;
  // rows and norms of the tensor-core greedy (integer data, rows <= 128 bytes)
  __shared__ __align__(16) uint8_t gsel[kBigSelBytes];
  const uint32_t tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
  const uint64_t cap = rs.gcap;
  const uint64_t slot = blockIdx.x;
  uint32_t* cid = rs.gcand + slot * cap;
  float* ckey = rs.gkey + slot * cap;
  int* posL = rs.gpos + slot * 2 * cap;
  int* posR = posL + cap;
  uint32_t* bits = rs.gbits + slot * (cap / 32 + 2);
  int* ranges = rs.granges + slot * 3 * (cap / 8 + 64);
  const uint32_t nbig = rs.counters[4];
  ddsort::Arr<uint32_t> A{cid, ckey};
  for (uint32_t e = blockIdx.x; e < nbig; e += gridDim.x) {
    const uint32_t k = rs.big[e];
    uint32_t start, end;
    segment_of(rs, k, start, end);
    const uint32_t t = rs.st[start];
    const uint32_t s = end - start;
    uint32_t* row = ix.graph + (uint64_t)t * ix.Rp;
    if (wid == 0) {
      uint32_t dg = row_degree(row, ix.Rp);
      if (lane == 0) s_deg = dg;
    }
    const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
    for (uint32_t j = tid; j < qb / 16; j += blockDim.x)
      ((uint4*)tv)[j] = __ldg((const uint4*)(ix.points + (uint64_t)t * ix.stride) + j);
    __syncthreads();
    const uint32_t deg = s_deg;
    const uint32_t m = s + deg;
    if ((uint64_t)m > cap) {  // cannot happen: s <= batch size, cap = batch + Rp
      if (tid == 0) dd_set_error(ix.err, DD_ESEG_CAP);
      __syncthreads();
      continue;
    }
    for (uint32_t j = tid; j < s; j += blockDim.x) {
      uint32_t c = (uint32_t)(ra.floor + rs.sv[start + j] / ix.Rp);
      cid[j] = c;
      ckey[j] = Dist<DT, MT>::eval(tv, ix.points + (uint64_t)c * ix.stride, ix.d);
    }
    for (uint32_t j = tid; j < deg; j += blockDim.x) {
      uint32_t c = row[j];
      cid[s + j] = c;
      ckey[s + j] = Dist<DT, MT>::eval(tv, ix.points + (uint64_t)c * ix.stride, ix.d);
    }
    for (uint32_t w = tid; w < (m + 31) / 32; w += blockDim.x) bits[w] = 0;
    if (tid == 0) {
      s_nsmall = 0;
      s_next = 0;
      cstack[0] = 0;
      cstack[1] = (int)m;
      cstack[2] = 2 * ddsort::floor_log2((int)m);
    }
    __syncthreads();
    // ---- sort emulation, phase 1: long ranges, whole CTA
    const int cta_range = big_cta_range(m);
    int sp = 3;
    while (sp > 0) {
      int depth = cstack[sp - 1], last = cstack[sp - 2], first = cstack[sp - 3];
      sp -= 3;
      __syncthreads();
      while (last - first > cta_range && depth > 0) {
        --depth;
        const int mid = first + (last - first) / 2;
        if (tid == 0) ddsort::move_median_to_first(A, first, first + 1, mid, last - 1);
        __syncthreads();
        const int cut = cta_partition_rank(A, first + 1, last, first, posL, posR, sh);
        if (tid == 0) {
          cstack[sp] = cut;
          cstack[sp + 1] = last;
          cstack[sp + 2] = depth;
        }
        sp += 3;
        last = cut;
        __syncthreads();
      }
      if (tid == 0) {  // the rest of this range goes to a warp
        int r = (int)s_nsmall++;
        ranges[3 * r] = first;
        ranges[3 * r + 1] = last;
        ranges[3 * r + 2] = depth;
      }
      __syncthreads();
    }
    // ---- phase 2: short ranges, one warp each (disjoint scratch: posL + first)
    while (true) {
      uint32_t r = 0;
      if (lane == 0) r = atomicAdd(&s_next, 1u);
      r = __shfl_sync(0xffffffffu, r, 0);
      if (r >= s_nsmall) break;
      const int first = ranges[3 * r], last = ranges[3 * r + 1], depth = ranges[3 * r + 2];
      warp_partition_loop(A, first, last, depth, wstack[wid], bits, posL + first, posR + first,
                          true);
    }
    __syncthreads();
    // ---- phase 3: leaves
    for (uint32_t q = tid; q < m; q += blockDim.x)
      if (bits[q >> 5] & (1u << (q & 31)))
        ddsort::insertion_sort_range(A, (int)q, ddsort::leaf_end(bits, (int)q, (int)m));
    __syncthreads();
    // ---- greedy selection (the row of t is rewritten; its old entries are in cid)
    if (DT != DD_F32 && greedy_uses_mma(ix.d, DT)) {
      // chunked greedy on one warp: every candidate row is read once, and the
      // walk stops at the R-th selection (hub lists are far longer than that)
      if (wid == 0) {
        PruneSmem Pg{};
        Pg.cid = cid;
        Pg.ckey = ckey;
        Pg.sel = (uint4*)gsel;
        warp_greedy_select_mma<DT, MT>(ix.points, ix.stride, ix.d, t, Pg, m, ra.alpha, ix.R, row,
                                       ix.Rp, Pg.sel);
        if (lane == 0) {
          atomicAdd(&rs.counters[2], 1u);
          atomicAdd(&rs.counters[3], m);
        }
      }
      __syncthreads();
      continue;
    }
    uint32_t nsel = 0, idx = 0, mm = m;
    while (nsel < ix.R && idx < mm) {
      const uint32_t ps = cid[idx];
      idx++;
      if (ps == t || ps == DD_NONE) continue;
      if (tid == 0) row[nsel] = ps;
      nsel++;
      const uint8_t* prow = ix.points + (uint64_t)ps * ix.stride;
      for (uint32_t q = idx + tid; q < mm; q += blockDim.x) {
        const uint32_t c = cid[q];
        if (c != DD_NONE) {
          const float dsp = Dist<DT, MT>::eval(prow, ix.points + (uint64_t)c * ix.stride, ix.d);
          if (__dmul_rn(ra.alpha, (double)dsp) <= (double)ckey[q]) cid[q] = DD_NONE;
        }
      }
      __syncthreads();
      if (mm - idx > 2048) {  // compact [idx, mm): drop removed entries, keep the order
        const uint32_t n2 = mm - idx;
        const uint32_t ch = (n2 + blockDim.x - 1) / blockDim.x;
        const uint32_t lo = idx + tid * ch, hi = min(mm, lo + ch);
        uint32_t c = 0;
        for (uint32_t q = lo; q < hi; q++) c += cid[q] != DD_NONE ? 1u : 0u;
        uint32_t tot;
        uint32_t w = cta_scan_excl(c, &tot, sh);
        for (uint32_t q = lo; q < hi; q++)
          if (cid[q] != DD_NONE) {
            posL[w] = (int)cid[q];
            posR[w] = __float_as_int(ckey[q]);
            w++;
          }
        __syncthreads();
        for (uint32_t q = tid; q < tot; q += blockDim.x) {
          cid[idx + q] = (uint32_t)posL[q];
          ckey[idx + q] = __int_as_float(posR[q]);
        }
        if (tid == 0) s_mm = idx + tot;
        __syncthreads();
        mm = s_mm;
      }
    }
    for (uint32_t j = nsel + tid; j < ix.Rp; j += blockDim.x) row[j] = DD_NONE;
    if (tid == 0) {
      atomicAdd(&rs.counters[2], 1u);
      atomicAdd(&rs.counters[3], m);
    }
    __syncthreads();
  }
}

// ============================================================ queries
template <int DT, int MT, int FPL, int CPL>
__global__ void __launch_bounds__(512) k_query(IndexView ix, QueryArgs qa, WarpLayout lay) {
  extern __shared__ uint4 smem_raw[];
  const uint32_t wpc = blockDim.x >> 5, wic = threadIdx.x >> 5, lane = lane_id();
  const uint64_t gw = (uint64_t)blockIdx.x * wpc + wic;
  const SearchSmem S = carve_query((uint8_t*)smem_raw + (size_t)wic * lay.total, lay);
  const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
  for (uint64_t q = gw; q < qa.nq; q += (uint64_t)gridDim.x * wpc) {
    SearchParams P;
    uint32_t Lq = qa.Ls[q];
    if (Lq == 0 || Lq > qa.Lmax || Lq < qa.k) {
      if (lane == 0) dd_set_error(ix.err, DD_ECAND_CAP);
      Lq = qa.Lmax;
    }
    P.points = ix.points; P.stride = ix.stride; P.graph = ix.graph; P.Rp = ix.Rp; P.n = ix.n;
    P.d = ix.d; P.start = qa.start; P.L = Lq; P.k = qa.k; P.cut = qa.cut; P.limit = qa.limit;
    P.degree_limit = qa.degree_limit; P.hbits = hash_bits_for(P.L); P.vcap = lay.vcap;
    P.query_mode = 1; P.keep_visited = 0; P.err = ix.err;
    load_vec(S.qv, qa.queries + q * qa.qstride, qb);
    __syncwarp();
    SearchOut o = warp_beam_search<DT, MT, FPL, CPL>(P, S, qa.skip_self ? q : (uint64_t)-1);
    for (uint32_t j = lane; j < qa.k; j += 32) {
      bool v = j < o.fr_n;
      qa.ids[q * qa.k + j] = v ? (S.fr_id[j] & ~DD_VBIT) : DD_NONE;
      qa.dists[q * qa.k + j] = v ? S.fr_d[j] : INFINITY;
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
  const SearchSmem S = carve_query((uint8_t*)smem_raw, lay);
  const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
  for (uint64_t q = blockIdx.x; q < ba.nq; q += gridDim.x) {
    SearchParams P;
    P.points = ix.points; P.stride = ix.stride; P.graph = ix.graph; P.Rp = ix.Rp; P.n = ix.n;
    P.d = ix.d; P.start = ba.start; P.L = ba.L; P.k = ba.k; P.cut = ba.cut; P.limit = ba.limit;
    P.degree_limit = ba.degree_limit; P.hbits = lay.hbits; P.vcap = lay.vcap;
    P.query_mode = ba.k > 0; P.keep_visited = 1; P.err = ix.err;
    load_vec(S.qv, ba.queries + q * ba.qstride, qb);
    __syncwarp();
    SearchOut o = warp_beam_search<DT, MT, 16, 4>(P, S, (uint64_t)ba.self_ids[q]);
    warp_sort_pairs(S.vis_id, S.vis_d, o.vis_n);
    for (uint32_t j = lane; j < o.fr_n; j += 32) {
      ba.fr_ids[q * ba.L + j] = S.fr_id[j] & ~DD_VBIT;
      ba.fr_d[q * ba.L + j] = S.fr_d[j];
    }
    for (uint32_t j = lane; j < o.vis_n; j += 32) {
      ba.vis_ids[q * ba.vcap + j] = S.vis_id[j];
      ba.vis_d[q * ba.vcap + j] = S.vis_d[j];
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
  const uint32_t lane = lane_id();
  for (uint32_t t = blockIdx.x; t < pa.ntasks; t += gridDim.x) {
    const uint32_t p = pa.p[t];
    const uint64_t o0 = pa.offsets[t], o1 = pa.offsets[t + 1];
    const uint64_t wbase = o0 + (uint64_t)t * ix.Rp;  // room for the out-list too
    const uint64_t cap = (o1 - o0) + ix.Rp;
    uint32_t* cid = pa.gcand + wbase;
    float* ckey = pa.gkey + wbase;
    uint8_t* ws = (uint8_t*)(pa.gws + 3 * wbase + (uint64_t)t * kGlobalStackInts);
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
    PruneSmem Pm = prune_ws(cid, ckey, ws, (uint32_t)cap);
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
  __shared__ __align__(16) uint8_t ws[2048];  // >= prune_ws_bytes(kMaxRp)
  const uint32_t lane = lane_id();
  PruneSmem Pm = prune_ws(cid, ckey, ws, kMaxRp);
  for (uint64_t v = blockIdx.x; v < ix.n; v += gridDim.x) {
    uint32_t* row = ix.graph + v * ix.Rp;
    const uint8_t* pv = ix.points + v * ix.stride;
    uint32_t deg = row_degree(row, ix.Rp);
    for (uint32_t j = lane; j < deg; j += 32) {
      cid[j] = row[j];
      ckey[j] = Dist<DT, MT>::eval(pv, ix.points + (uint64_t)row[j] * ix.stride, ix.d);
    }
    __syncwarp();
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

// warp-distributed sorted top-k (k <= 32): lane i holds the i-th best (dist, id)
__device__ __forceinline__ void topk_insert(double& bd, uint32_t& bi, uint32_t k, double dv,
                                            uint32_t iv, bool cand) {
  const uint32_t lane = lane_id();
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

// grid (query blocks of 8 warps, chunks); each warp keeps a top-k of its chunk
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
    topk_insert(bd, bi, k, dv, iv, (dv < td) || (dv == td && iv < ti));
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
    topk_insert(bd, bi, k, dv, iv, (dv < td) || (dv == td && iv < ti));
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
  static const int cand[] = {1, 2, 4, 5, 8, 16};
  for (int wpc : cand) {
    const size_t sm = (size_t)bytes_per_warp * wpc;
    if (sm > 227 * 1024) break;
    const int b = occupancy(kernel, wpc * 32, sm);
    if (b * wpc > best.warps_per_cta * best.blocks_per_sm) best = LaunchPlan{wpc, b};
  }
  if (best.blocks_per_sm == 0) best.blocks_per_sm = 1;
  return best;
}

LaunchPlan plan_query(const IndexView& ix, const WarpLayout& lay, uint32_t Lmax) {
  LaunchPlan p{1, 1};
#define CALL4(DT, MT, F, C) p = plan_warp_kernel(k_query<DT, MT, F, C>, lay.total);
#define CALL(DT, MT) DD_DISPATCH_FC(Lmax, ix.Rp, DT, MT, CALL4)
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
#undef CALL4
  return p;
}

LaunchPlan plan_search(const IndexView& ix, const WarpLayout& lay, uint32_t L) {
  LaunchPlan p{1, 1};
#define CALL4(DT, MT, F, C) p = plan_warp_kernel(k_search<DT, MT, F, C>, lay.total);
#define CALL(DT, MT) DD_DISPATCH_FC(L, ix.Rp, DT, MT, CALL4)
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
#undef CALL4
  return p;
}

void launch_search(const IndexView& ix, const RoundArgs& ra, const WarpLayout& lay,
                   const LaunchPlan& plan, int grid, cudaStream_t st) {
  const size_t sm = (size_t)lay.total * plan.warps_per_cta;
#define CALL4(DT, MT, F, C)                                                          \
  set_smem(k_search<DT, MT, F, C>, sm);                                              \
  k_search<DT, MT, F, C><<<grid, plan.warps_per_cta * 32, sm, st>>>(ix, ra, lay);
#define CALL(DT, MT) DD_DISPATCH_FC(ra.L, ix.Rp, DT, MT, CALL4)
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
#undef CALL4
}

LaunchPlan plan_prune(const IndexView& ix, const PruneLayout& lay) {
  LaunchPlan p{1, 1};
#define CALL(DT, MT) p = plan_warp_kernel(k_prune<DT, MT>, lay.total);
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
  return p;
}

void launch_prune_round(const IndexView& ix, const RoundArgs& ra, const PruneLayout& lay,
                        uint32_t vcap, const LaunchPlan& plan, int grid, cudaStream_t st) {
  const size_t sm = (size_t)lay.total * plan.warps_per_cta;
#define CALL(DT, MT)                                                                 \
  set_smem(k_prune<DT, MT>, sm);                                                     \
  k_prune<DT, MT><<<grid, plan.warps_per_cta * 32, sm, st>>>(ix, ra, lay, vcap);
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
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
  if (!ra.B) return;
  RevLayout L = rev_layout(ix.d, ix.dtype, ix.Rp);
  size_t sm = (size_t)L.total * kRevWarps;
#define CALL(DT, MT)                                                                  \
  set_smem(k_reverse<DT, MT>, sm);                                                    \
  k_reverse<DT, MT><<<sm_count * occupancy(k_reverse<DT, MT>, kRevWarps * 32, sm),     \
                      kRevWarps * 32, sm, st>>>(ix, ra, rs);                          \
  k_reverse_big<DT, MT><<<kBigSlots, kBigThreads, 0, st>>>(ix, ra, rs);
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
}

void launch_query(const IndexView& ix, const QueryArgs& qa, const WarpLayout& lay, int wpc,
                  int grid, cudaStream_t st) {
  size_t sm = (size_t)lay.total * wpc;
#define CALL4(DT, MT, F, C)                                                          \
  set_smem(k_query<DT, MT, F, C>, sm);                                               \
  k_query<DT, MT, F, C><<<grid, wpc * 32, sm, st>>>(ix, qa, lay);
#define CALL(DT, MT) DD_DISPATCH_FC(qa.Lmax, ix.Rp, DT, MT, CALL4)
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
#undef CALL4
}

void launch_beam(const IndexView& ix, const BeamArgs& ba, const WarpLayout& lay, int grid,
                 cudaStream_t st) {
  size_t sm = lay.total;
#define CALL(DT, MT)                                                   \
  set_smem(k_beam<DT, MT>, sm);                                        \
  k_beam<DT, MT><<<grid, 32, sm, st>>>(ix, ba, lay);
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
}

void launch_prune_tasks(const IndexView& ix, const PruneArgs& pa, cudaStream_t st) {
  if (!pa.ntasks) return;
  int grid = (int)std::min<uint32_t>(pa.ntasks, 4096);
#define CALL(DT, MT) k_prune_tasks<DT, MT><<<grid, 32, 0, st>>>(ix, pa);
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
}

void launch_sort_rows(const IndexView& ix, cudaStream_t st) {
  int grid = (int)std::min<uint64_t>(ix.n, 65536);
#define CALL(DT, MT) k_sort_rows<DT, MT><<<grid, 32, 0, st>>>(ix);
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
}

void launch_groundtruth(const IndexView& ix, const uint8_t* queries, uint64_t qstride, uint64_t nq,
                        uint32_t k, uint32_t* ids, float* dists, double* part_d, uint32_t* part_i,
                        uint32_t nchunks, cudaStream_t st) {
  dim3 grid((unsigned)((nq + 7) / 8), nchunks);
#define CALL(DT, MT)                                                                  \
  k_gt_partial<DT, MT><<<grid, 256, 0, st>>>(ix, queries, qstride, nq, k, nchunks, part_d, part_i);
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
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
