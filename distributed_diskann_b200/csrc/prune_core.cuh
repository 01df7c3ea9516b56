// Warp-cooperative robustPrune (include/index.h:63-123; src/bsp_index.hpp:483-545).
//
//  1. the candidate list (ids + distances to p) is ordered exactly as the
//     reference's std::sort orders it (sort_emul.cuh): the introsort
//     partition phase is replayed with each Hoare partition done in parallel
//     by rank pairing, then every lane finishes whole leaves;
//  2. greedy selection: walk the sorted list, skip p and removed entries,
//     select p*, and remove every later p' with alpha * d(p*, p') <= d(p, p')
//     (alpha is a double in the reference, so the test is done in double).
//     Three exact forms: INT8 tensor-core Gram tiles (integer data), rows in
//     registers (float rows <= 256 bytes), and a per-lane form (the rest).
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
  uint4* sel;         // rows of the register / tensor-core greedy (overlays posL/posR), or null
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

// Fast path of warp_std_sort for lists without equal keys, where std::sort's
// result is the one ascending order.  Returns false (list untouched) when two
// keys are equal.  A list already in strictly ascending order is left as is
// (a sorted list with equal neighbours goes straight back to the caller);
// otherwise each element's rank (count of smaller keys) is its position, and
// the list is rewritten through the rank-pairing scratch (2 * cap ints).
constexpr uint32_t kRankSortMax = 256;

// The rank sort of a list made of one long strictly ascending run and at most
// 32 other elements: a reverse prune's list, where the target's row is the
// selection of its last prune (ascending) followed by the few sources
// appended since, and the new sources come in batch order.  A run element's
// rank is its place in the run plus the other elements below it; another
// element's rank is its lower bound in the run (binary search) plus the other
// elements below it.  Returns 1 when sorted, 0 when two keys are equal (list
// untouched), -1 when the list does not have that shape (list untouched).
__device__ __forceinline__ int warp_sort_run_plus_few(const PruneSmem& S, uint32_t m) {
  const uint32_t FULL = 0xffffffffu;
  const uint32_t lane = lane_id();
  constexpr uint32_t kMaxRuns = 48;
  // the longest run [rs, rs + rl): runs start at 0 and where a key is not
  // above its predecessor
  uint32_t nruns = 0, prev = 0, rs = 0, rl = 0;
  for (uint32_t b = 0; b < m && nruns <= kMaxRuns; b += 32) {
    const uint32_t i = b + lane;
    const bool st = i < m && i > 0 && !(S.ckey[i - 1] < S.ckey[i]);
    for (uint32_t bits = __ballot_sync(FULL, st); bits; bits &= bits - 1) {
      const uint32_t s0 = b + __ffs(bits) - 1;
      if (s0 - prev > rl) {
        rl = s0 - prev;
        rs = prev;
      }
      prev = s0;
      nruns++;
    }
  }
  if (m - prev > rl) {
    rl = m - prev;
    rs = prev;
  }
  const uint32_t u = m - rl;
  if (nruns > kMaxRuns || u > 32) return -1;
  // lane q < u holds the q-th element outside the run
  const bool qv = lane < u;
  const uint32_t qi = lane < rs ? lane : lane + rl;
  const float kq = qv ? S.ckey[qi] : 0.f;
  const uint32_t re = rs + rl;
  uint32_t rq = rs;
  bool tie = false;
  if (qv) {
    uint32_t hi = re;
    while (rq < hi) {
      const uint32_t mid = (rq + hi) >> 1;
      if (S.ckey[mid] < kq) rq = mid + 1;
      else hi = mid;
    }
    tie = rq < re && S.ckey[rq] == kq;
  }
  rq -= rs;
  for (uint32_t j = 0; j < u; j++) {
    const float kj = __shfl_sync(FULL, kq, j);
    rq += kj < kq ? 1u : 0u;
    tie |= qv && j != lane && kj == kq;
  }
  if (__any_sync(FULL, tie)) return 0;
  int* tid = S.posL;
  float* tkey = (float*)S.posR;
  if (qv) {
    tid[rq] = (int)S.cid[qi];
    tkey[rq] = kq;
  }
  for (uint32_t b = 0; b < rl; b += 32) {
    const uint32_t i = b + lane;
    const float ki = i < rl ? S.ckey[rs + i] : 0.f;
    uint32_t r = i;
    for (uint32_t j = 0; j < u; j++) r += __shfl_sync(FULL, kq, j) < ki ? 1u : 0u;
    if (i < rl) {
      tid[r] = (int)S.cid[rs + i];
      tkey[r] = ki;
    }
  }
  __syncwarp();
  for (uint32_t i = lane; i < m; i += 32) {
    S.cid[i] = (uint32_t)tid[i];
    S.ckey[i] = tkey[i];
  }
  __syncwarp();
  return 1;
}

__device__ __forceinline__ bool warp_sort_distinct(const PruneSmem& S, uint32_t m) {
  const uint32_t FULL = 0xffffffffu;
  const uint32_t lane = lane_id();
  bool strict = true, nondesc = true;
  for (uint32_t b = 1; b < m && nondesc; b += 32) {
    const uint32_t i = b + lane;
    const float k0 = i < m ? S.ckey[i - 1] : 0.f, k1 = i < m ? S.ckey[i] : 1.f;
    strict = __all_sync(FULL, !strict ? false : k0 < k1) && strict;
    nondesc = __all_sync(FULL, k0 <= k1);
  }
  if (strict && nondesc) return true;
  if (nondesc || m > kRankSortMax) return false;
  const int rp = warp_sort_run_plus_few(S, m);
  if (rp >= 0) return rp == 1;
  uint32_t rk[kRankSortMax / 32];
  bool tie = false;
#pragma unroll
  for (int t = 0; t < (int)(kRankSortMax / 32); t++) {
    const uint32_t i = lane + 32u * t;
    rk[t] = 0;
    if (i < m) {
      const float ki = S.ckey[i];
      uint32_t r = 0, eq = 0;
      for (uint32_t j = 0; j < m; j++) {
        const float kj = S.ckey[j];
        r += kj < ki ? 1u : 0u;
        eq += kj == ki ? 1u : 0u;
      }
      rk[t] = r;
      tie |= eq != 1u;
    }
  }
  if (__any_sync(FULL, tie)) return false;
  int* tid = S.posL;
  float* tkey = (float*)S.posR;
#pragma unroll
  for (int t = 0; t < (int)(kRankSortMax / 32); t++) {
    const uint32_t i = lane + 32u * t;
    if (i < m) {
      tid[rk[t]] = (int)S.cid[i];
      tkey[rk[t]] = S.ckey[i];
    }
  }
  __syncwarp();
  for (uint32_t i = lane; i < m; i += 32) {
    S.cid[i] = (uint32_t)tid[i];
    S.ckey[i] = tkey[i];
  }
  __syncwarp();
  return true;
}

// Leaf phase of the emulation: the library's final insertion sort is a
// stable sort inside each leaf.  Leaves of more than kThreshold elements are
// heap-sorted ranges (already ascending); in the others each element's place
// is its stable rank within the leaf, computed by all lanes in parallel.  The
// permuted list goes through the rank-pairing scratch (2 * cap ints).
__device__ __forceinline__ void warp_finish_leaves(const PruneSmem& S, uint32_t m) {
  const uint32_t lane = lane_id();
  int* tid = S.posL;
  float* tkey = (float*)S.posR;
  for (uint32_t i = lane; i < m; i += 32) {
    // leaf start: the last marked position <= i
    int w = (int)(i >> 5);
    uint32_t bw = S.leafbits[w] & (0xffffffffu >> (31 - (i & 31)));
    while (bw == 0 && w > 0) bw = S.leafbits[--w];
    const int lo = (w << 5) + 31 - __clz(bw);
    const int hi = ddsort::leaf_end(S.leafbits, lo, (int)m);
    const float ki = S.ckey[i];
    uint32_t dst = i;
    if (hi - lo <= ddsort::kThreshold) {
      uint32_t r = 0;
      for (int j = lo; j < hi; j++) {
        const float kj = S.ckey[j];
        r += (kj < ki || (kj == ki && j < (int)i)) ? 1u : 0u;
      }
      dst = (uint32_t)lo + r;
    }
    tid[dst] = (int)S.cid[i];
    tkey[dst] = ki;
  }
  __syncwarp();
  for (uint32_t i = lane; i < m; i += 32) {
    S.cid[i] = (uint32_t)tid[i];
    S.ckey[i] = tkey[i];
  }
  __syncwarp();
}

// Orders cid/ckey[0, m) exactly like std::sort with the distance-only
// comparator: lists without equal keys take warp_sort_distinct; otherwise
// the warp replays the partition phase, marking leaf starts in a bitmap, and
// the leaves are finished in parallel (warp_finish_leaves).
__device__ __forceinline__ void warp_std_sort(const PruneSmem& S, uint32_t m) {
  const uint32_t lane = lane_id();
  if (warp_sort_distinct(S, m)) return;
  ddsort::Arr<uint32_t> A{S.cid, S.ckey};
  const uint32_t nw = (m + 31) / 32;
  for (uint32_t w = lane; w < nw; w += 32) S.leafbits[w] = 0;
  __syncwarp();
  if (m > 0)
    warp_partition_loop(A, 0, (int)m, 2 * ddsort::floor_log2((int)m), S.stack, S.leafbits, S.posL,
                        S.posR, false);
  warp_finish_leaves(S, m);
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
// out_key (may be null): the selected entries' distances to p, beside out_row.
template <int DT, int MT>
__device__ uint32_t warp_greedy_select(const uint8_t* points, uint64_t stride, uint32_t d,
                                       uint32_t p, const PruneSmem& S, uint32_t m, double alpha,
                                       uint32_t R, uint32_t* out_row, uint32_t Rp,
                                       float* out_key = nullptr) {
  const uint32_t lane = lane_id();
  uint32_t nsel = 0, idx = 0;
  while (nsel < R && idx < m) {
    const uint32_t ps = S.cid[idx];
    idx++;
    if (ps == p || ps == DD_NONE) continue;
    if (lane == 0) {
      out_row[nsel] = ps;
      if (out_key) out_key[nsel] = S.ckey[idx - 1];
    }
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
                                           uint32_t Rp, uint4* sel, float* out_key = nullptr) {
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
        if (out_key) out_key[nsel] = S.ckey[j];
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

// ---------------------------------------------------------------------------
// Greedy selection on the tensor cores (integer data, rows of <= 128 bytes).
//
// The occlusion distances are exact integers, so they come from Gram tiles of
// the rows: d(a, b) = |a|^2 + |b|^2 - 2 a.b for L2 and -a.b for MIPS, with a.b
// from mma.sync m16n8k32 (u8 x u8 or s8 x s8, s32 accumulation: exact for
// rows of <= 128 bytes), which is the reference's int32 value bit for bit.
// The sorted list is walked in chunks of 16 candidates:
//   1. the chunk's rows are staged in shared memory (right after the rows of
//      the nsel already selected entries) with their squared norms;
//   2. cross tiles (selected rows x chunk rows) remove every chunk member
//      that some selected entry occludes;
//   3. the chunk's own 16 x 16 tile gives, for each member j, the mask of
//      members i < j with alpha * d(i, j) <= d(p, j); the chunk is then
//      selected in order with bit operations, and the selected rows are
//      compacted into the selected area.
// Shared layout (`sel`): (Rp + 16) rows of 128 bytes, 16-byte words swizzled
// by (row & 7) so the fragment loads are free of bank conflicts, then
// (Rp + 16) norms, then 16 chunk occlusion thresholds.
// ---------------------------------------------------------------------------
constexpr uint32_t kMmaChunk = 16;

__host__ __device__ inline uint32_t mma_sel_bytes(uint32_t Rp) {
  return (Rp + kMmaChunk) * 128u + (Rp + kMmaChunk) * 4u + kMmaChunk * 4u;
}
// the tensor-core form applies to integer data whose padded rows fit 128 bytes
__host__ __device__ inline bool greedy_uses_mma(uint32_t d, int dtype) {
  return dtype != DD_F32 && d <= 128;
}
// bytes the fast greedy forms need in the prune workspace (0: generic form);
// tensor = false leaves the tensor-core form out (the plain form)
__host__ __device__ inline uint32_t greedy_sel_bytes(uint32_t d, int dtype, uint32_t Rp,
                                                     bool tensor = true) {
  if (tensor && greedy_uses_mma(d, dtype)) return mma_sel_bytes(Rp);
  const uint32_t nv = row_words16(d, dtype);
  return nv <= reg_row_max_words(dtype) ? Rp * nv * 16u : 0u;
}

template <int DT>
__device__ __forceinline__ void mma_k32(int (&acc)[4], const uint32_t (&a)[4], uint32_t b0,
                                        uint32_t b1) {
  if (DT == DD_U8)
    asm("mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+r"(acc[0]), "+r"(acc[1]), "+r"(acc[2]), "+r"(acc[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
  else
    asm("mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+r"(acc[0]), "+r"(acc[1]), "+r"(acc[2]), "+r"(acc[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// 32-bit word q (0..31) of staged row r
__device__ __forceinline__ uint32_t mma_row_word(const uint32_t* rw, uint32_t r, uint32_t q) {
  return rw[r * 32u + (q ^ ((r & 7u) << 2))];
}
// 16-byte word w (0..7) of staged row r
__device__ __forceinline__ uint4* mma_row_vec(uint32_t* rw, uint32_t r, uint32_t w) {
  return (uint4*)(rw + r * 32u + ((w ^ (r & 7u)) << 2));
}

// Four 8 x 16-byte tiles of staged rows into registers (ldmatrix .x4): lane l
// names row `row` of tile l / 8 at 16-byte word `w`; register j then holds
// bytes 4 (l % 4) .. 4 (l % 4) + 3 of row l / 4 of tile j, which is the
// m16n8k32 fragment layout of 8-bit operands.
__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], uint32_t* rw, uint32_t row, uint32_t w) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(mma_row_vec(rw, row, w));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

// acc[nt] += rows [ra0, ra0+16) x rows [rb0 + 8 nt, rb0 + 8 nt + 8), nt = 0, 1 (KS k-steps)
template <int DT>
__device__ __forceinline__ void mma_tile_16x16(uint32_t* rw, uint32_t ra0, uint32_t rb0,
                                               uint32_t KS, int (&acc)[2][4]) {
  const uint32_t lane = lane_id(), mi = lane >> 3, ri = lane & 7;
#pragma unroll
  for (int nt = 0; nt < 2; nt++)
#pragma unroll
    for (int i = 0; i < 4; i++) acc[nt][i] = 0;
  for (uint32_t ks = 0; ks < KS; ks++) {
    // A: tiles (rows 0-7, k 0-15), (rows 8-15, k 0-15), (rows 0-7, k 16-31), (rows 8-15, k 16-31)
    uint32_t a[4];
    ldsm_x4(a, rw, ra0 + (mi & 1u) * 8u + ri, 2u * ks + (mi >> 1));
    if (ra0 == rb0) {
      // the chunk's own tile: B's n-tiles are A's row halves
      mma_k32<DT>(acc[0], a, a[0], a[2]);
      mma_k32<DT>(acc[1], a, a[1], a[3]);
    } else {
      // B: tiles (rows 0-7, k 0-15), (rows 0-7, k 16-31), (rows 8-15, k 0-15), (rows 8-15, k 16-31)
      uint32_t b[4];
      ldsm_x4(b, rw, rb0 + (mi >> 1) * 8u + ri, 2u * ks + (mi & 1u));
      mma_k32<DT>(acc[0], a, b[0], b[1]);
      mma_k32<DT>(acc[1], a, b[2], b[3]);
    }
  }
}

// Largest integer x with alpha * (double)x <= key in the reference's double
// arithmetic (alpha > 0).  Integer distances of rows <= 128 bytes have
// |d| < 2^24, so the float the reference compares is the integer itself, and
// the rounded product is monotone in x: "alpha * d <= key" is exactly
// "d <= occlusion_threshold".  The result is clamped to +-2^25, which keeps
// that equivalence for every |d| < 2^24; floor(key / alpha) is off by at most
// one, so two correction steps each way suffice.
// inv_alpha = 1 / alpha (the estimate may be off by one; the steps fix it).
__device__ __forceinline__ int occlusion_threshold(double alpha, double inv_alpha, float key) {
  const double k = (double)key, lim = 33554432.0;
  double x = floor(k * inv_alpha);
  x = fmin(fmax(x, -lim), lim);
  for (int it = 0; it < 2 && x < lim && __dmul_rn(alpha, x + 1.0) <= k; it++) x += 1.0;
  for (int it = 0; it < 2 && x > -lim && __dmul_rn(alpha, x) > k; it++) x -= 1.0;
  return (int)x;
}

// the row-dependent part of a Gram distance: |a|^2 - 2 a.b (L2; the column's
// |b|^2 is folded into its threshold) or -a.b (MIPS)
template <int MT>
__device__ __forceinline__ int gram_part(int na, int dot) {
  return MT == DD_L2 ? na - 2 * dot : -dot;
}


// PREFETCH: load the next chunk's rows while the current chunk's tiles run
// (worth it when the rows are not in cache yet).
template <int DT, int MT, bool PREFETCH = true>
__device__ uint32_t warp_greedy_select_mma(const uint8_t* points, uint64_t stride, uint32_t d,
                                           uint32_t p, const PruneSmem& S, uint32_t m,
                                           double alpha, uint32_t R, uint32_t* out_row,
                                           uint32_t Rp, uint4* sel, float* out_key = nullptr) {
  const uint32_t FULL = 0xffffffffu;
  const uint32_t lane = lane_id(), g = lane >> 2, t = lane & 3;
  uint32_t* rw = (uint32_t*)sel;
  int* norms = (int*)(rw + (Rp + kMmaChunk) * 32u);
  int* cthr = norms + Rp + kMmaChunk;
  const uint32_t qb = (d + 15u) & ~15u;   // padded row bytes (integer data)
  const uint32_t KS = (qb + 31u) >> 5;    // k-steps of 32 bytes
  const double inv_alpha = 1.0 / alpha;
  const uint32_t NW = 2u * KS;            // 16-byte words staged per row
  // A chunk's rows are loaded into registers (two lanes per member, 16-byte
  // words h, h+2, h+4, h+6): with PREFETCH one chunk ahead of its tiles.
  uint4 pv[4];
  uint32_t pcj = DD_NONE;
  auto load_chunk = [&](uint32_t c0) {
    const uint32_t j = lane >> 1, h = lane & 1;
    const uint32_t cnt = c0 < m ? min(kMmaChunk, m - c0) : 0u;
    pcj = j < cnt ? S.cid[c0 + j] : DD_NONE;
    const bool alive = pcj != DD_NONE && pcj != p;
    const uint4* src = (const uint4*)(points + (uint64_t)(alive ? pcj : 0u) * stride);
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const uint32_t w = h + 2u * i;
      pv[i] = (alive && w < NW) ? __ldg(src + w) : make_uint4(0, 0, 0, 0);
    }
  };
  if (PREFETCH) load_chunk(0);
  uint32_t nsel = 0;
  for (uint32_t c0 = 0; c0 < m && nsel < R; c0 += kMmaChunk) {
    if (!PREFETCH) load_chunk(c0);
    // ---- 1. stage the chunk: two lanes per member, rows nsel .. nsel + 15
    uint32_t amask;
    {
      const uint32_t j = lane >> 1, h = lane & 1;
      const uint32_t cj = pcj;
      const bool alive = cj != DD_NONE && cj != p;
      const uint32_t r = nsel + j;
      uint32_t nrm = 0;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const uint32_t w = h + 2u * i;
        const uint4 v = pv[i];
        *mma_row_vec(rw, r, w) = v;
        if (DT == DD_U8) {
          nrm = __dp4a(v.x, v.x, nrm); nrm = __dp4a(v.y, v.y, nrm);
          nrm = __dp4a(v.z, v.z, nrm); nrm = __dp4a(v.w, v.w, nrm);
        } else {
          int s = (int)nrm;
          s = __dp4a((int)v.x, (int)v.x, s); s = __dp4a((int)v.y, (int)v.y, s);
          s = __dp4a((int)v.z, (int)v.z, s); s = __dp4a((int)v.w, (int)v.w, s);
          nrm = (uint32_t)s;
        }
      }
      nrm += __shfl_xor_sync(FULL, nrm, 1);
      if (h == 0) {
        norms[r] = (int)nrm;
        // occlusion of member j: L2 |a|^2 - 2 a.b <= T_j - |b|^2, MIPS -a.b <= T_j
        const int T = alive ? occlusion_threshold(alpha, inv_alpha, S.ckey[c0 + j]) : 0;
        cthr[j] = MT == DD_L2 ? T - (int)nrm : T;
      }
      const bool a2 = __shfl_sync(FULL, alive ? 1 : 0, (2u * lane) & 31u) != 0;
      amask = __ballot_sync(FULL, lane < kMmaChunk && a2);
    }
    __syncwarp();
    if (PREFETCH) load_chunk(c0 + kMmaChunk);
    // ---- 2. occlusion by the entries selected before this chunk
    for (uint32_t r0 = 0; r0 < nsel && amask; r0 += 16) {
      int acc[2][4];
      mma_tile_16x16<DT>(rw, r0, nsel, KS, acc);
      const uint32_t sa = r0 + g, sb = r0 + g + 8;
      const int na = MT == DD_L2 ? norms[sa] : 0, nb = MT == DD_L2 ? norms[sb] : 0;
      // this lane's four columns (8 nt + 2 t + e) occluded by its rows, OR-ed
      // over the warp
      uint32_t occ = 0;
#pragma unroll
      for (int nt = 0; nt < 2; nt++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int thr = cthr[8u * nt + 2u * t + e];
          const bool oa = sa < nsel && gram_part<MT>(na, acc[nt][e]) <= thr;
          const bool ob = sb < nsel && gram_part<MT>(nb, acc[nt][2 + e]) <= thr;
          occ |= (oa || ob) ? 1u << (8u * nt + 2u * t + e) : 0u;
        }
      amask &= ~__reduce_or_sync(FULL, occ);
    }
    // ---- 3. the chunk's own tile, then in-order selection with bit masks
    uint32_t colmask[kMmaChunk];
    {
      int acc[2][4];
      mma_tile_16x16<DT>(rw, nsel, nsel, KS, acc);
      const int na = MT == DD_L2 ? norms[nsel + g] : 0;
      const int nb = MT == DD_L2 ? norms[nsel + g + 8] : 0;
#pragma unroll
      for (int nt = 0; nt < 2; nt++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const uint32_t col = 8u * nt + 2u * t + e;
          const int thr = cthr[col];
          const bool oa = g < col && gram_part<MT>(na, acc[nt][e]) <= thr;
          const bool ob = g + 8 < col && gram_part<MT>(nb, acc[nt][2 + e]) <= thr;
          // column col's occluder bits (rows g and g + 8), OR-ed over the 8
          // lanes that hold it (lane = 4 g + t); lane tt then has column
          // 8 nt + 2 tt + e, which every lane takes
          uint32_t v = (oa ? 1u << g : 0u) | (ob ? 1u << (g + 8) : 0u);
          v |= __shfl_xor_sync(FULL, v, 4);
          v |= __shfl_xor_sync(FULL, v, 8);
          v |= __shfl_xor_sync(FULL, v, 16);
#pragma unroll
          for (int tt = 0; tt < 4; tt++) colmask[8 * nt + 2 * tt + e] = __shfl_sync(FULL, v, tt);
        }
    }
    uint32_t selm = 0, ns = nsel;
#pragma unroll
    for (int j = 0; j < (int)kMmaChunk; j++)
      if (ns < R && ((amask >> j) & 1u) && (colmask[j] & selm) == 0) {
        selm |= 1u << j;
        ns++;
      }
    // ---- output ids in order; compact the selected rows (read all, then write)
    {
      const uint32_t j = lane >> 1, h = lane & 1;
      const bool s = (selm >> j) & 1u;
      const uint32_t k = __popc(selm & ((1u << j) - 1u));
      if (s && h == 0) {
        out_row[nsel + k] = S.cid[c0 + j];
        if (out_key) out_key[nsel + k] = S.ckey[c0 + j];
      }
      uint4 v[4];
      int nrm = 0;
      if (s) {
#pragma unroll
        for (int i = 0; i < 4; i++) v[i] = *mma_row_vec(rw, nsel + j, 2u * i + h);
        nrm = norms[nsel + j];
      }
      __syncwarp();
      if (s) {
#pragma unroll
        for (int i = 0; i < 4; i++) *mma_row_vec(rw, nsel + k, 2u * i + h) = v[i];
        if (h == 0) norms[nsel + k] = nrm;
      }
      __syncwarp();
    }
    nsel = ns;
  }
  for (uint32_t j = nsel + lane; j < Rp; j += 32) out_row[j] = DD_NONE;
  __syncwarp();
  return nsel;
}

// The fastest exact greedy form for the data type; `sel` holds
// greedy_sel_bytes(d, DT, Rp, TENSOR) bytes (unused by the generic form).
// TENSOR = false is the plain form: every occlusion distance on the CUDA
// cores (register rows where they fit, else the per-lane form).  PREFETCH:
// see warp_greedy_select_mma.
template <int DT, int MT, bool PREFETCH = true, bool TENSOR = true>
__device__ __forceinline__ uint32_t warp_greedy_select_fast(const uint8_t* points, uint64_t stride,
                                                            uint32_t d, uint32_t p,
                                                            const PruneSmem& S, uint32_t m,
                                                            double alpha, uint32_t R,
                                                            uint32_t* out_row, uint32_t Rp,
                                                            uint4* sel, float* out_key = nullptr) {
  if (TENSOR && DT != DD_F32 && greedy_uses_mma(d, DT))
    return warp_greedy_select_mma<DT, MT, PREFETCH>(points, stride, d, p, S, m, alpha, R,
                                                    out_row, Rp, sel, out_key);
  if (row_words16(d, DT) <= (uint32_t)RegRow<DT>::NVM) {
    return warp_greedy_select_reg<DT, MT>(points, stride, d, p, S, m, alpha, R, out_row, Rp, sel,
                                          out_key);
  }
  return warp_greedy_select<DT, MT>(points, stride, d, p, S, m, alpha, R, out_row, Rp, out_key);
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

}  // namespace ddk
