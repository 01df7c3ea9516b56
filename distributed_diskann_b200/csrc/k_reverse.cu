// Reverse-edge kernels of the B200 Vamana hot path.
//
//   k_apply_rows  : update_neighbors of the batch (src/bsp_index.hpp:354-357)
//   k_reverse     : one warp per target: append, or robustPrune when the row
//                   would overflow R (src/bsp_index.hpp:384-407)
//   k_reverse_big : targets with more candidates than a warp's shared memory
//                   holds, one CTA each
// The grouping of (target, source) pairs by target is semisort.cu.
#include <cfloat>
#include <cstdio>

#include "dd_common.cuh"
#include "kernel_util.cuh"
#include "kernels.cuh"
#include "prune_core.cuh"
#include "search_core.cuh"
#include "sort_emul.cuh"

namespace ddk {

// row_key (may be null): the rows' distances go beside them (new_key)
__global__ void k_apply_rows(uint32_t* graph, const uint32_t* new_out, float* row_key,
                             const float* new_key, uint64_t floor, uint64_t nvec, uint32_t Rp) {
  // rows are Rp uint32 = Rp/4 uint4; batch rows are contiguous in the graph
  const uint4* src = (const uint4*)new_out;
  uint4* dst = (uint4*)(graph + floor * Rp);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvec;
       i += (uint64_t)gridDim.x * blockDim.x) {
    dst[i] = src[i];
    if (row_key) ((float4*)(row_key + floor * Rp))[i] = ((const float4*)new_key)[i];
  }
}

// per-warp shared layout of the reverse kernel
struct RevLayout {
  uint32_t tv, cid, ckey, ws, total;
};
__host__ __device__ inline RevLayout rev_layout(uint32_t d, int dtype, uint32_t Rp, bool tensor) {
  RevLayout r;
  uint32_t off = 0;
  uint32_t esz = dtype == DD_F32 ? 4 : 1;
  const uint32_t sel_bytes = greedy_sel_bytes(d, dtype, Rp, tensor);
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

// the reverse prune's greedy loads the next chunk's rows ahead (with kept
// row distances no candidate row is read before the greedy)
constexpr bool kRevPrefetch = true;

// Append the sources of segment [start, end) (already in batch order), or
// prune when the row would exceed R (one warp; s + deg <= kRevCandCap).
template <int DT, int MT, bool TC>
__device__ void reverse_one(const IndexView& ix, const RoundArgs& ra, const ReverseScratch& rs,
                            uint32_t t, uint32_t start, uint32_t s, uint32_t deg, uint8_t* tv,
                            PruneSmem Pm) {
  const uint32_t lane = lane_id();
  uint32_t* row = ix.graph + (uint64_t)t * ix.Rp;
  // the row's distances to t, kept beside the graph (fast form)
  float* rk = (ra.new_key && ra.row_key) ? ra.row_key + (uint64_t)t * ix.Rp : nullptr;
  const uint32_t* sk = rs.sv + start;
  if (s + deg <= ix.R) {
    for (uint32_t j = lane; j < s; j += 32) {
      row[deg + j] = (uint32_t)(ra.floor + sk[j] / ix.Rp);
      if (rk) rk[deg + j] = ra.new_key[sk[j]];
    }
    __syncwarp();
    return;
  }
  if (!rk) {  // otherwise no distance to t is computed here
    const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
    load_vec(tv, ix.points + (uint64_t)t * ix.stride, qb);
    __syncwarp();
  }
  // a source's distance to t is the one its own prune selected t with (the
  // distances are symmetric bit for bit: (a-b)^2 = (b-a)^2, a*b = b*a, same
  // summation order), when the insert prune kept it
  for (uint32_t j = lane; j < s; j += 32) {
    uint32_t c = (uint32_t)(ra.floor + sk[j] / ix.Rp);
    Pm.cid[j] = c;
    Pm.ckey[j] = ra.new_key ? ra.new_key[sk[j]]
                            : Dist<DT, MT>::eval(tv, ix.points + (uint64_t)c * ix.stride, ix.d);
  }
  for (uint32_t j = lane; j < deg; j += 32) {
    uint32_t c = row[j];
    Pm.cid[s + j] = c;
    Pm.ckey[s + j] = rk ? rk[j] : Dist<DT, MT>::eval(tv, ix.points + (uint64_t)c * ix.stride, ix.d);
  }
  __syncwarp();
  const uint32_t m = s + deg;
  warp_std_sort(Pm, m);
  warp_greedy_select_fast<DT, MT, kRevPrefetch, TC>(ix.points, ix.stride, ix.d, t, Pm, m, ra.alpha,
                                                    ix.R, row, ix.Rp, Pm.sel, rk);
  if (lane == 0) {
    atomicAdd(&rs.counters[2], 1u);
    atomicAdd(&rs.counters[3], m);
  }
}

template <int DT, int MT, bool TC>
__global__ void __launch_bounds__(kRevWarps * 32, 8) k_reverse(IndexView ix, RoundArgs ra, ReverseScratch rs) {
  extern __shared__ uint4 smem_raw[];
  const RevLayout L = rev_layout(ix.d, DT, ix.Rp, TC);
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
    reverse_one<DT, MT, TC>(ix, ra, rs, t, start, s, deg, base + L.tv, Pm);
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

template <int DT, int MT, bool TC>
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
    float* rk = (ra.new_key && ra.row_key) ? ra.row_key + (uint64_t)t * ix.Rp : nullptr;
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
      const uint32_t key = rs.sv[start + j];
      uint32_t c = (uint32_t)(ra.floor + key / ix.Rp);
      cid[j] = c;
      ckey[j] = ra.new_key ? ra.new_key[key]
                           : Dist<DT, MT>::eval(tv, ix.points + (uint64_t)c * ix.stride, ix.d);
    }
    for (uint32_t j = tid; j < deg; j += blockDim.x) {
      uint32_t c = row[j];
      cid[s + j] = c;
      ckey[s + j] = rk ? rk[j] : Dist<DT, MT>::eval(tv, ix.points + (uint64_t)c * ix.stride, ix.d);
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
    if (TC && DT != DD_F32 && greedy_uses_mma(ix.d, DT)) {
      // chunked greedy on one warp: every candidate row is read once, and the
      // walk stops at the R-th selection (hub lists are far longer than that)
      if (wid == 0) {
        PruneSmem Pg{};
        Pg.cid = cid;
        Pg.ckey = ckey;
        Pg.sel = (uint4*)gsel;
        warp_greedy_select_mma<DT, MT>(ix.points, ix.stride, ix.d, t, Pg, m, ra.alpha, ix.R, row,
                                       ix.Rp, Pg.sel, rk);
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
      if (tid == 0) {
        row[nsel] = ps;
        if (rk) rk[nsel] = ckey[idx - 1];
      }
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

void launch_apply_rows(const IndexView& ix, const RoundArgs& ra, cudaStream_t st) {
  uint64_t nvec = (uint64_t)ra.B * ix.Rp / 4;
  if (!nvec) return;
  int grid = (int)std::min<uint64_t>((nvec + 255) / 256, 4096);
  k_apply_rows<<<grid, 256, 0, st>>>(ix.graph, ra.new_out, ra.new_key ? ra.row_key : nullptr,
                                     ra.new_key, ra.floor, nvec, ix.Rp);
}

void launch_reverse(const IndexView& ix, const RoundArgs& ra, const ReverseScratch& rs,
                    bool tensor, cudaStream_t st, int sm_count) {
  if (!ra.B) return;
  RevLayout L = rev_layout(ix.d, ix.dtype, ix.Rp, tensor);
  size_t sm = (size_t)L.total * kRevWarps;
#define CALL2(DT, MT, TC)                                                             \
  set_smem(k_reverse<DT, MT, TC>, sm);                                                \
  k_reverse<DT, MT, TC><<<sm_count * occupancy(k_reverse<DT, MT, TC>, kRevWarps * 32, sm), \
                          kRevWarps * 32, sm, st>>>(ix, ra, rs);                      \
  k_reverse_big<DT, MT, TC><<<kBigSlots, kBigThreads, 0, st>>>(ix, ra, rs);
#define CALL(DT, MT)                                                                  \
  if (tensor) { CALL2(DT, MT, true); } else { CALL2(DT, MT, false); }
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
#undef CALL2
}

}  // namespace ddk
