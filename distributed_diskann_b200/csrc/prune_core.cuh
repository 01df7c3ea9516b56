// Warp-cooperative robustPrune (include/index.h:63-123; src/bsp_index.hpp:483-545).
//
//  1. the candidate list (ids + distances to p) is ordered exactly as the
//     reference's std::sort orders it (sort_emul.cuh): the introsort
//     partition phase is replayed with each Hoare partition done in parallel
//     by rank pairing, then every lane finishes whole leaves;
//  2. greedy selection: walk the sorted list, skip p and removed entries,
//     select p*, and remove every later p' with alpha * d(p*, p') <= d(p, p')
//     (alpha is a double in the reference, so the test is done in double).
//     The occlusion distances of one p* are spread over the 32 lanes.
#pragma once
#include "dd_common.cuh"
#include "sort_emul.cuh"

namespace ddk {

__device__ __forceinline__ uint32_t lanemask_lt_() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

struct PruneSmem {
  uint32_t* cid;      // candidate ids (DD_NONE = removed)
  float* ckey;        // distance to p
  uint32_t* leafbits; // leaf starts of the sort emulation, (capacity + 31) / 32 words
  int* stack;         // ddsort::stack_ints(capacity) ints
  int* posL;          // rank-pairing scratch, capacity ints each
  int* posR;
  uint4* sel;         // selected rows of warp_greedy_select_reg (overlays posL/posR), or null
};

// bytes of the leaf bitmap + stack + rank scratch for `cap` candidates (16-byte multiple)
__host__ __device__ inline uint32_t prune_ws_bytes(uint32_t cap) {
  uint32_t b = ((cap + 31) / 32) * 4 + 4u * (uint32_t)ddsort::stack_ints((int)cap) + 8u * cap;
  return (b + 15) & ~15u;
}

__device__ __forceinline__ PruneSmem prune_ws(uint32_t* cid, float* ckey, uint8_t* ws, uint32_t cap) {
  PruneSmem p;
  p.cid = cid;
  p.ckey = ckey;
  p.leafbits = (uint32_t*)ws;
  p.stack = (int*)(ws + ((cap + 31) / 32) * 4);
  p.posL = p.stack + ddsort::stack_ints((int)cap);
  p.posR = p.posL + cap;
  p.sel = nullptr;
  return p;
}

// One Hoare partition of [first, last) around the pivot at `pivot` (= first-1),
// done by the warp: the k-th "not less" position from the left is swapped
// with the k-th "not greater" position from the right for every k where the
// former is left of the latter (ddsort::partition_by_rank_pairing).
__device__ __forceinline__ int warp_partition_rank(const ddsort::Arr<uint32_t>& A, int first,
                                                   int last, int pivot, int* posL, int* posR) {
  const uint32_t FULL = 0xffffffffu;
  const int lane = (int)lane_id();
  const float pk = A.key[pivot];
  int nL = 0;
  for (int base = first; base < last; base += 32) {
    const int i = base + lane;
    const bool f = i < last && !(A.key[i] < pk);
    const uint32_t b = __ballot_sync(FULL, f);
    if (f) posL[nL + __popc(b & lanemask_lt_())] = i;
    nL += __popc(b);
  }
  int nR = 0;
  for (int base = last - 1; base >= pivot; base -= 32) {
    const int i = base - lane;
    const bool f = i >= pivot && !(pk < A.key[i]);
    const uint32_t b = __ballot_sync(FULL, f);
    if (f) posR[nR + __popc(b & lanemask_lt_())] = i;
    nR += __popc(b);
  }
  __syncwarp();
  const int lim = nL < nR ? nL : nR;
  int K = 0;
  for (int kb = 0; kb < lim; kb += 32) {  // posL[k] < posR[k] holds for a prefix of k
    const int k = kb + lane;
    const uint32_t b = __ballot_sync(FULL, k < lim && posL[k] < posR[k]);
    K += __popc(b);
    if (b != FULL) break;
  }
  for (int k = lane; k < K; k += 32) A.swap(posL[k], posR[k]);
  __syncwarp();
  if (K == 0) return posL[0];
  const int a = K < nL ? posL[K] : last;
  const int r = posR[K - 1];
  return a < r ? a : r;
}

// The introsort partition phase of one range [first0, last0) with the
// remaining depth budget depth0, replayed by a warp: median-of-three and the
// heap fallback on lane 0, each partition in parallel; leaf starts are marked
// in `bits` (atomically when other warps mark neighbouring ranges).  posL /
// posR need room for last0 - first0 entries; the stack for
// 3 * (depth0 + 2) ints.
__device__ __forceinline__ void warp_partition_loop(const ddsort::Arr<uint32_t>& A, int first0,
                                                    int last0, int depth0, int* stack,
                                                    uint32_t* bits, int* posL, int* posR,
                                                    bool atomic_bits) {
  const uint32_t lane = lane_id();
  if (lane == 0) {
    stack[0] = first0;
    stack[1] = last0;
    stack[2] = depth0;
  }
  int sp = 3;
  __syncwarp();
  while (sp > 0) {
    int depth = stack[sp - 1], last = stack[sp - 2], first = stack[sp - 3];
    sp -= 3;
    __syncwarp();
    while (last - first > ddsort::kThreshold) {
      if (depth == 0) {
        if (lane == 0) ddsort::heap_sort_range(A, first, last);
        __syncwarp();
        break;
      }
      --depth;
      const int mid = first + (last - first) / 2;
      if (lane == 0) ddsort::move_median_to_first(A, first, first + 1, mid, last - 1);
      __syncwarp();
      const int cut = warp_partition_rank(A, first + 1, last, first, posL, posR);
      if (lane == 0) {
        stack[sp] = cut;
        stack[sp + 1] = last;
        stack[sp + 2] = depth;
      }
      sp += 3;
      last = cut;
      __syncwarp();
    }
    if (lane == 0) {
      if (atomic_bits) atomicOr(&bits[first >> 5], 1u << (first & 31));
      else bits[first >> 5] |= 1u << (first & 31);
    }
    __syncwarp();
  }
}

// Orders cid/ckey[0, m) exactly like std::sort with the distance-only
// comparator: the warp replays the partition phase, marking leaf starts in a
// bitmap; then the lanes finish the leaves in parallel.
__device__ __forceinline__ void warp_std_sort(const PruneSmem& S, uint32_t m) {
  const uint32_t lane = lane_id();
  ddsort::Arr<uint32_t> A{S.cid, S.ckey};
  const uint32_t nw = (m + 31) / 32;
  for (uint32_t w = lane; w < nw; w += 32) S.leafbits[w] = 0;
  __syncwarp();
  if (m > 0)
    warp_partition_loop(A, 0, (int)m, 2 * ddsort::floor_log2((int)m), S.stack, S.leafbits, S.posL,
                        S.posR, false);
  for (uint32_t i = lane; i < m; i += 32)
    if (S.leafbits[i >> 5] & (1u << (i & 31)))
      ddsort::insertion_sort_range(A, (int)i, ddsort::leaf_end(S.leafbits, (int)i, (int)m));
  __syncwarp();
}

// CTA-wide sum (all threads call it; sh: 32 words)
__device__ __forceinline__ uint32_t cta_reduce_add(uint32_t v, uint32_t* sh) {
  uint32_t tot;
  cta_scan_excl(v, &tot, sh);
  return tot;
}

// One Hoare partition (rank pairing) done by the whole CTA; the pivot value
// must be in place at `pivot` (= first - 1) before the call.
__device__ __forceinline__ int cta_partition_rank(const ddsort::Arr<uint32_t>& A, int first,
                                                  int last, int pivot, int* posL, int* posR,
                                                  uint32_t* sh) {
  const int NT = (int)blockDim.x, tid = (int)threadIdx.x;
  const float pk = A.key[pivot];
  // left stops, ascending: contiguous chunks per thread
  const int n = last - first;
  const int ch = (n + NT - 1) / NT;
  const int lo = first + tid * ch, hi = min(last, lo + ch);
  uint32_t c = 0;
  for (int i = lo; i < hi; i++) c += !(A.key[i] < pk) ? 1u : 0u;
  uint32_t nL;
  uint32_t j = cta_scan_excl(c, &nL, sh);
  for (int i = lo; i < hi; i++)
    if (!(A.key[i] < pk)) posL[j++] = i;
  // right stops, descending over [pivot, last)
  const int nr = last - pivot;
  const int ch2 = (nr + NT - 1) / NT;
  const int q0 = tid * ch2, q1 = min(nr, q0 + ch2);
  c = 0;
  for (int q = q0; q < q1; q++) c += !(pk < A.key[last - 1 - q]) ? 1u : 0u;
  uint32_t nR;
  j = cta_scan_excl(c, &nR, sh);
  for (int q = q0; q < q1; q++)
    if (!(pk < A.key[last - 1 - q])) posR[j++] = last - 1 - q;
  __syncthreads();
  const int lim = (int)min(nL, nR);
  c = 0;
  for (int k = tid; k < lim; k += NT) c += posL[k] < posR[k] ? 1u : 0u;
  const int K = (int)cta_reduce_add(c, sh);  // the pairs with posL < posR form a prefix
  for (int k = tid; k < K; k += NT) A.swap(posL[k], posR[k]);
  __syncthreads();
  if (K == 0) return posL[0];
  const int a = K < (int)nL ? posL[K] : last;
  const int r = posR[K - 1];
  return a < r ? a : r;
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

// ---------------------------------------------------------------------------
// Greedy selection with register-resident candidate rows.
//
// warp_greedy_select reads a whole candidate row from global memory (L1/L2)
// per lane for every selected p*, so each selection waits on a round of
// scattered loads.  This form walks the sorted list in chunks of 32: lane j
// loads candidate c0+j's row into registers once (NVM 16-byte words), tests it
// against the rows selected in earlier chunks, then the chunk is selected in
// order.  Selected rows are kept in shared memory (`sel`, Rp rows of nv
// 16-byte words) and read by broadcast, so the inner loops make no global
// loads.  A candidate is removed iff some selected p* before it has
// alpha * d(p*, p') <= d(p, p'), which is exactly the reference's rule
// (include/index.h:100-118): removal is monotone and selection of an entry
// depends only on the earlier selections, so testing against all earlier
// selected rows in any grouping gives the same result.  Distances are the
// reference's arithmetic with p* as the first operand, like Dist::eval.
// ---------------------------------------------------------------------------
template <int DT, int MT, int NVM>
__device__ __forceinline__ float dist_reg(const uint4* a, const uint4 (&b)[NVM], uint32_t d,
                                          uint32_t nv) {
  if (DT == DD_F32) {
    float r = 0.f;
#pragma unroll
    for (int k = 0; k < NVM; k++) {
      if ((uint32_t)k >= nv) break;
      const uint4 xa = a[k];
      const float x[4] = {__uint_as_float(xa.x), __uint_as_float(xa.y), __uint_as_float(xa.z),
                          __uint_as_float(xa.w)};
      const float y[4] = {__uint_as_float(b[k].x), __uint_as_float(b[k].y),
                          __uint_as_float(b[k].z), __uint_as_float(b[k].w)};
      const uint32_t i = 4u * (uint32_t)k;
      if (MT == DD_L2) {
        if (i + 3 < d) {  // NSGDist: groups of 4 summed left to right, then added
          float d0 = __fsub_rn(x[0], y[0]), d1 = __fsub_rn(x[1], y[1]);
          float d2 = __fsub_rn(x[2], y[2]), d3 = __fsub_rn(x[3], y[3]);
          float s = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1)),
                                        __fmul_rn(d2, d2)),
                              __fmul_rn(d3, d3));
          r = __fadd_rn(r, s);
        } else {  // the 0-3 element tail, one at a time
#pragma unroll
          for (int t = 0; t < 4; t++)
            if (i + t < d) {
              float d0 = __fsub_rn(x[t], y[t]);
              r = __fadd_rn(r, __fmul_rn(d0, d0));
            }
        }
      } else {
#pragma unroll
        for (int t = 0; t < 4; t++)
          if (i + t < d) r = __fadd_rn(r, __fmul_rn(x[t], y[t]));
      }
    }
    return MT == DD_L2 ? r : -r;
  } else {
    uint32_t u = 0;
    int v = 0;
#pragma unroll
    for (int k = 0; k < NVM; k++) {
      if ((uint32_t)k >= nv) break;
      const uint4 x = a[k];
      const uint4 y = b[k];
      if (MT == DD_L2) {
        uint32_t s;
        s = absdiff4<DT>(x.x, y.x); u = __dp4a(s, s, u);
        s = absdiff4<DT>(x.y, y.y); u = __dp4a(s, s, u);
        s = absdiff4<DT>(x.z, y.z); u = __dp4a(s, s, u);
        s = absdiff4<DT>(x.w, y.w); u = __dp4a(s, s, u);
      } else if (DT == DD_U8) {
        u = __dp4a(x.x, y.x, u); u = __dp4a(x.y, y.y, u);
        u = __dp4a(x.z, y.z, u); u = __dp4a(x.w, y.w, u);
      } else {
        v = __dp4a((int)x.x, (int)y.x, v); v = __dp4a((int)x.y, (int)y.y, v);
        v = __dp4a((int)x.z, (int)y.z, v); v = __dp4a((int)x.w, (int)y.w, v);
      }
    }
    if (MT == DD_L2) return __int2float_rn((int)u);
    return DT == DD_U8 ? -__int2float_rn((int)u) : -__int2float_rn(v);
  }
}

// 16-byte words of a padded point row, and the largest row the register form
// takes (128 bytes for integer data, 256 bytes for float data)
__host__ __device__ inline uint32_t row_words16(uint32_t d, int dtype) {
  return (d * (dtype == DD_F32 ? 4u : 1u) + 15u) / 16u;
}
template <int DT>
struct RegRow { static constexpr int NVM = (DT == DD_F32) ? 16 : 8; };
__host__ __device__ inline uint32_t reg_row_max_words(int dtype) {
  return dtype == DD_F32 ? 16u : 8u;
}

template <int DT, int MT>
__device__ uint32_t warp_greedy_select_reg(const uint8_t* points, uint64_t stride, uint32_t d,
                                           uint32_t p, const PruneSmem& S, uint32_t m,
                                           double alpha, uint32_t R, uint32_t* out_row,
                                           uint32_t Rp, uint4* sel) {
  constexpr int NVM = RegRow<DT>::NVM;
  const uint32_t FULL = 0xffffffffu;
  const uint32_t lane = lane_id();
  const uint32_t nv = row_words16(d, DT);
  uint32_t nsel = 0;
  for (uint32_t c0 = 0; c0 < m && nsel < R; c0 += 32) {
    const uint32_t j = c0 + lane;
    const uint32_t cj = j < m ? S.cid[j] : DD_NONE;
    bool alive = cj != DD_NONE && cj != p;
    const double kj = alive ? (double)S.ckey[j] : 0.0;
    uint4 row[NVM];
#pragma unroll
    for (int k = 0; k < NVM; k++) row[k] = make_uint4(0, 0, 0, 0);
    if (alive) {
      const uint4* src = (const uint4*)(points + (uint64_t)cj * stride);
#pragma unroll
      for (int k = 0; k < NVM; k++)
        if ((uint32_t)k < nv) row[k] = __ldg(src + k);
    }
    // occlusion by the rows selected in earlier chunks
    for (uint32_t s = 0; s < nsel; s++) {
      if (!__any_sync(FULL, alive)) break;
      const float dsp = dist_reg<DT, MT, NVM>(sel + (uint64_t)s * nv, row, d, nv);
      if (alive && __dmul_rn(alpha, (double)dsp) <= kj) alive = false;
    }
    // this chunk, in order
    uint32_t rem = __ballot_sync(FULL, alive);
    while (rem && nsel < R) {
      const uint32_t i = (uint32_t)__ffs(rem) - 1;
      uint4* dst = sel + (uint64_t)nsel * nv;
      if (lane == i) {
        out_row[nsel] = cj;
#pragma unroll
        for (int k = 0; k < NVM; k++)
          if ((uint32_t)k < nv) dst[k] = row[k];
      }
      __syncwarp();
      nsel++;
      const bool later = alive && lane > i;
      if (__any_sync(FULL, later)) {
        const float dsp = dist_reg<DT, MT, NVM>(dst, row, d, nv);
        if (later && __dmul_rn(alpha, (double)dsp) <= kj) alive = false;
      }
      rem = __ballot_sync(FULL, alive) & ~((2u << i) - 1u);
    }
    __syncwarp();
  }
  for (uint32_t j = nsel + lane; j < Rp; j += 32) out_row[j] = DD_NONE;
  __syncwarp();
  return nsel;
}

// byte offset of the (16-byte aligned) selected-row area inside a prune
// workspace of `cap` candidates: it overlays the rank-pairing scratch, which
// is dead once the sort is done
__host__ __device__ inline uint32_t prune_sel_offset(uint32_t cap) {
  uint32_t b = ((cap + 31) / 32) * 4 + 4u * (uint32_t)ddsort::stack_ints((int)cap);
  return (b + 15) & ~15u;
}
// workspace bytes when the selected rows (sel_bytes) share it
__host__ __device__ inline uint32_t prune_ws_bytes_sel(uint32_t cap, uint32_t sel_bytes) {
  uint32_t a = prune_ws_bytes(cap);
  uint32_t b = prune_sel_offset(cap) + sel_bytes;
  b = (b + 15) & ~15u;
  return a > b ? a : b;
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
