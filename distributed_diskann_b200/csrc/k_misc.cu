// Ground truth and graph-format kernels of the B200 Vamana hot path.
//
//   k_gt_*          : brute-force ground truth (FP64 for float data, exact
//                     integers otherwise)
//   k_to_ref_rows / k_from_ref_rows : device rows <-> the reference's
//                     [deg, nbr...] rows (include/utils/graph.h:126-128)
#include <cfloat>
#include <climits>
#include <cstdio>

#include <cuda_bf16.h>

#include "dd_common.cuh"
#include "kernel_util.cuh"
#include "kernels.cuh"
#include "prune_core.cuh"
#include "search_core.cuh"
#include "sort_emul.cuh"

namespace ddk {

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

// ---- integer data with rows of <= 128 bytes: the tensor cores.
// d(q, p) = |q|^2 + |p|^2 - 2 q.p (L2) or -q.p (MIPS) with q.p from
// mma.sync m16n8k32 (u8 x u8 / s8 x s8, s32 accumulation): exact integers,
// the same values the CUDA-core form computes.  A CTA of two warps takes 32
// queries (16 per warp: the A operand, kept in registers) against one chunk
// of the base, streamed in tiles of 128 rows: cp.async copies the next tile
// into shared memory (rows swizzled like the prune's Gram tiles) while the
// warps multiply the current one.  Each (query, point) value is compared with
// the query's k-th best; the few that pass are inserted, one warp-wide step
// each, into the query's top-k list in shared memory.
constexpr int kGtWarps = 2;
constexpr int kGtQueries = 16 * kGtWarps;
constexpr int kGtTile = 128;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N)); }

// squared norm (L2) of a staged row of `words` 32-bit words, exact
template <int DT>
__device__ __forceinline__ int staged_norm(const uint32_t* rw, uint32_t r, uint32_t words) {
  int acc = 0;
  for (uint32_t q = 0; q < words; q++) {
    const uint32_t v = mma_row_word(rw, r, q);
    if (DT == DD_U8) acc = (int)__dp4a(v, v, (uint32_t)acc);
    else acc = __dp4a((int)v, (int)v, acc);
  }
  return acc;
}

// (d, i) < (e, j) in the ground truth's order: distance, then id
__device__ __forceinline__ bool gt_less(int d, uint32_t i, int e, uint32_t j) {
  return d < e || (d == e && i < j);
}

// warp-wide insertion of (cd, ci) into the sorted list ld/li[0, k) (shared memory)
__device__ __forceinline__ void gt_insert(int* ld, uint32_t* li, uint32_t k, int cd, uint32_t ci) {
  const uint32_t lane = lane_id();
  if (!gt_less(cd, ci, ld[k - 1], li[k - 1])) return;  // warp-uniform (same smem values)
  const int d = lane < k ? ld[lane] : INT_MAX;
  const uint32_t i = lane < k ? li[lane] : DD_NONE;
  const bool before = lane < k && gt_less(d, i, cd, ci);
  const uint32_t pos = __popc(__ballot_sync(0xffffffffu, before));
  const int ud = __shfl_up_sync(0xffffffffu, d, 1);
  const uint32_t ui = __shfl_up_sync(0xffffffffu, i, 1);
  __syncwarp();
  if (lane == pos) {
    ld[lane] = cd;
    li[lane] = ci;
  } else if (lane > pos && lane < k) {
    ld[lane] = ud;
    li[lane] = ui;
  }
  __syncwarp();
}

template <int DT, int MT>
__global__ void __launch_bounds__(kGtWarps * 32) k_gt_mma(IndexView ix, const uint8_t* queries,
                                                          uint64_t qstride, uint64_t nq, uint32_t k,
                                                          uint32_t nchunks, double* part_d,
                                                          uint32_t* part_i) {
  __shared__ __align__(16) uint32_t qrows[kGtQueries * 32];
  __shared__ __align__(16) uint32_t tiles[2][kGtTile * 32];
  __shared__ int tnorm[2][kGtTile];
  __shared__ int top_d[kGtQueries][32];
  __shared__ uint32_t top_i[kGtQueries][32];
  const uint32_t tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  const uint32_t g = lane >> 2, t4 = lane & 3;
  const uint64_t q0 = (uint64_t)blockIdx.x * kGtQueries;
  const uint32_t words = (uint32_t)(ix.stride / 4);  // 16 or 32: rows of 64 or 128 bytes
  const uint32_t KS = words / 8;                      // k-steps of 32 bytes
  const uint64_t chunk = (ix.n + nchunks - 1) / nchunks;
  const uint64_t c0 = (uint64_t)blockIdx.y * chunk;
  const uint64_t c1 = min(ix.n, c0 + chunk);
  for (uint32_t e = tid; e < kGtQueries * (words / 4); e += blockDim.x) {
    const uint32_t r = e / (words / 4), w = e % (words / 4);
    uint4 v = make_uint4(0, 0, 0, 0);
    if (q0 + r < nq) v = __ldg((const uint4*)(queries + (q0 + r) * qstride) + w);
    *mma_row_vec(qrows, r, w) = v;
  }
  for (uint32_t e = tid; e < kGtQueries * 32; e += blockDim.x) {
    top_d[e / 32][e % 32] = INT_MAX;
    top_i[e / 32][e % 32] = DD_NONE;
  }
  auto load_tile = [&](int buf, uint64_t base) {
    for (uint32_t e = tid; e < kGtTile * (words / 4); e += blockDim.x) {
      const uint32_t r = e / (words / 4), w = e % (words / 4);
      if (base + r < c1)
        cp_async16(mma_row_vec(tiles[buf], r, w), ix.points + (base + r) * ix.stride + 16 * w);
      else
        *mma_row_vec(tiles[buf], r, w) = make_uint4(0, 0, 0, 0);
    }
    cp_async_commit();
  };
  if (c0 < c1) load_tile(0, c0);
  __syncthreads();
  // A fragments of this warp's 16 queries (all k-steps) and their norms
  const uint32_t ra = 16 * warp + g;
  uint32_t afr[4][4];
#pragma unroll
  for (int ks = 0; ks < 4; ks++) {
    const uint32_t qw = 8 * ks + t4;
    const bool on = (uint32_t)ks < KS;
    afr[ks][0] = on ? mma_row_word(qrows, ra, qw) : 0u;
    afr[ks][1] = on ? mma_row_word(qrows, ra + 8, qw) : 0u;
    afr[ks][2] = on ? mma_row_word(qrows, ra, qw + 4) : 0u;
    afr[ks][3] = on ? mma_row_word(qrows, ra + 8, qw + 4) : 0u;
  }
  const int qn_lo = MT == DD_L2 ? staged_norm<DT>(qrows, ra, words) : 0;
  const int qn_hi = MT == DD_L2 ? staged_norm<DT>(qrows, ra + 8, words) : 0;
  const bool live_lo = q0 + ra < nq, live_hi = q0 + ra + 8 < nq;
  // the k-th best of the rows g and g + 8 (refreshed after insertions)
  int th_lo = INT_MAX, th_hi = INT_MAX;
  uint32_t ti_lo = DD_NONE, ti_hi = DD_NONE;
  int buf = 0;
  for (uint64_t base = c0; base < c1; base += kGtTile, buf ^= 1) {
    if (base + kGtTile < c1) {
      load_tile(buf ^ 1, base + kGtTile);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (MT == DD_L2)
      for (uint32_t r = tid; r < kGtTile; r += blockDim.x)
        tnorm[buf][r] = staged_norm<DT>(tiles[buf], r, words);
    __syncthreads();
    const uint32_t* rw = tiles[buf];
    for (int nt = 0; nt < kGtTile / 8; nt++) {
      int acc[4] = {0, 0, 0, 0};
      const uint32_t rb = 8 * nt + g;
#pragma unroll
      for (int ks = 0; ks < 4; ks++)
        if ((uint32_t)ks < KS)
          mma_k32<DT>(acc, afr[ks], mma_row_word(rw, rb, 8 * ks + t4),
                      mma_row_word(rw, rb, 8 * ks + t4 + 4));
      // acc[0..1]: query row g, points 8 nt + 2 t4 + {0, 1}; acc[2..3]: row g + 8
      int dist[4];
      uint32_t pass = 0;
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const uint32_t col = 8 * nt + 2 * t4 + (e & 1);
        const bool lo = e < 2;
        dist[e] = MT == DD_L2 ? (lo ? qn_lo : qn_hi) + tnorm[buf][col] - 2 * acc[e] : -acc[e];
        const uint32_t pid = (uint32_t)(base + col);
        if (base + col < c1 && (lo ? live_lo : live_hi) &&
            gt_less(dist[e], pid, lo ? th_lo : th_hi, lo ? ti_lo : ti_hi))
          pass |= 1u << e;
      }
      uint32_t anyp = __ballot_sync(0xffffffffu, pass != 0);
      if (anyp) {
        while (anyp) {
          const int src = __ffs(anyp) - 1;
          anyp &= anyp - 1;
          const uint32_t m = __shfl_sync(0xffffffffu, pass, src);
          int sd[4];
#pragma unroll
          for (int e = 0; e < 4; e++) sd[e] = __shfl_sync(0xffffffffu, dist[e], src);
#pragma unroll
          for (int e = 0; e < 4; e++) {
            if (m & (1u << e)) {
              const uint32_t qr = 16 * warp + (uint32_t)(src >> 2) + (e < 2 ? 0u : 8u);
              const uint32_t col = 8 * nt + 2 * (uint32_t)(src & 3) + (e & 1);
              gt_insert(top_d[qr], top_i[qr], k, sd[e], (uint32_t)(base + col));
            }
          }
        }
        th_lo = top_d[ra][k - 1];
        ti_lo = top_i[ra][k - 1];
        th_hi = top_d[ra + 8][k - 1];
        ti_hi = top_i[ra + 8][k - 1];
      }
    }
    __syncthreads();  // the next iteration's copies overwrite this tile's buffer
  }
  for (uint32_t r = 0; r < 16; r++) {
    const uint32_t qr = 16 * warp + r;
    const uint64_t q = q0 + qr;
    if (q < nq && lane < k) {
      const uint64_t o = (q * nchunks + blockIdx.y) * k + lane;
      const uint32_t id = top_i[qr][lane];
      part_d[o] = id == DD_NONE ? INFINITY : (double)top_d[qr][lane];
      part_i[o] = id;
    }
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

// ============================================================ sharded build exchange
// The targets whose rows the reverse-edge step of this rank changed (the
// segment heads of the grouped pairs) and their new rows, for the other ranks.
__global__ void k_export_rows(const uint32_t* graph, uint32_t Rp, const uint32_t* st,
                              const uint32_t* heads, const uint32_t* counters, uint64_t cap,
                              uint32_t* ids_out, uint32_t* rows_out) {
  const uint32_t T = counters[1];
  const uint32_t lane = lane_id();
  for (uint64_t k = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < T && k < cap;
       k += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
    const uint32_t t = st[heads[k]];
    if (lane == 0) ids_out[k] = t;
    for (uint32_t j = lane; j < Rp; j += 32) rows_out[k * Rp + j] = graph[(uint64_t)t * Rp + j];
  }
}

// rows received from the other ranks; ids are checked against n
__global__ void k_set_rows(uint32_t* graph, uint64_t n, uint32_t Rp, const uint32_t* ids,
                           const uint32_t* rows, uint64_t count, uint32_t* err) {
  const uint32_t lane = lane_id();
  for (uint64_t k = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < count;
       k += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
    const uint32_t t = ids[k];
    if (t >= n) {
      if (lane == 0) dd_set_error(err, DD_EBAD_ID);
      continue;
    }
    for (uint32_t j = lane; j < Rp; j += 32) {
      uint32_t a = rows[k * Rp + j];
      if (a != DD_NONE && a >= n) {
        dd_set_error(err, DD_EBAD_ID);
        a = DD_NONE;
      }
      graph[(uint64_t)t * Rp + j] = a;
    }
  }
}

void launch_export_rows(const IndexView& ix, const uint32_t* st, const uint32_t* heads,
                        const uint32_t* counters, uint64_t cap, uint32_t* ids_out,
                        uint32_t* rows_out, cudaStream_t stream) {
  k_export_rows<<<1184, 256, 0, stream>>>(ix.graph, ix.Rp, st, heads, counters, cap, ids_out,
                                          rows_out);
}

void launch_set_rows(const IndexView& ix, const uint32_t* ids, const uint32_t* rows,
                     uint64_t count, cudaStream_t stream) {
  if (!count) return;
  const int grid = (int)std::min<uint64_t>((count * 32 + 255) / 256, 65536);
  k_set_rows<<<grid, 256, 0, stream>>>(ix.graph, ix.n, ix.Rp, ids, rows, count, ix.err);
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

bool groundtruth_uses_mma(const IndexView& ix) {
  return ix.dtype != DD_F32 && (ix.stride == 64 || ix.stride == 128);
}

void launch_groundtruth(const IndexView& ix, const uint8_t* queries, uint64_t qstride, uint64_t nq,
                        uint32_t k, uint32_t* ids, float* dists, double* part_d, uint32_t* part_i,
                        uint32_t nchunks, cudaStream_t st) {
  if (groundtruth_uses_mma(ix)) {
    // integer data of rows <= 128 bytes: tensor-core Gram tiles
    dim3 grid((unsigned)((nq + kGtQueries - 1) / kGtQueries), nchunks);
#define CALL(DT, MT)                                                                  \
  k_gt_mma<DT, MT><<<grid, kGtWarps * 32, 0, st>>>(ix, queries, qstride, nq, k, nchunks, part_d, \
                                                   part_i);
    if (ix.dtype == DD_I8 && ix.metric == DD_L2) { CALL(DD_I8, DD_L2); }
    else if (ix.dtype == DD_I8) { CALL(DD_I8, DD_MIPS); }
    else if (ix.metric == DD_L2) { CALL(DD_U8, DD_L2); }
    else { CALL(DD_U8, DD_MIPS); }
#undef CALL
  } else {
    dim3 grid((unsigned)((nq + 7) / 8), nchunks);
#define CALL(DT, MT)                                                                  \
  k_gt_partial<DT, MT><<<grid, 256, 0, st>>>(ix, queries, qstride, nq, k, nchunks, part_d, part_i);
    DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
  }
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

// ============================================================ BF16 row copies
// One warp per row: each lane converts 8 values (two float4 of the FP32 row)
// into one 16-byte word of BF16 values; values at or beyond d become zeros.
// The squared norm of the BF16 row is summed in FP32 (its rounding is far
// inside the screen's 1% slack on the bound term it enters).
__global__ void __launch_bounds__(256) k_screen_rows(const uint8_t* points, uint64_t stride,
                                                     uint64_t n, uint32_t d, uint8_t* screen,
                                                     uint64_t sstride, float* snorm) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nw = (d + 7) >> 3;
  const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t i = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n;
       i += nwarps) {
    const float* row = (const float*)(points + i * stride);
    uint4* out = (uint4*)(screen + i * sstride);
    float nrm = 0.f;
    for (uint32_t w = lane; w < nw; w += 32) {
      uint32_t h[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const uint32_t e = 8 * w + 2 * j;
        const float x0 = e < d ? __ldg(row + e) : 0.f;
        const float x1 = e + 1 < d ? __ldg(row + e + 1) : 0.f;
        const __nv_bfloat16 b0 = __float2bfloat16_rn(x0), b1 = __float2bfloat16_rn(x1);
        const float f0 = __bfloat162float(b0), f1 = __bfloat162float(b1);
        nrm = fmaf(f0, f0, nrm);
        nrm = fmaf(f1, f1, nrm);
        h[j] = (uint32_t)__bfloat16_as_ushort(b0) | ((uint32_t)__bfloat16_as_ushort(b1) << 16);
      }
      out[w] = make_uint4(h[0], h[1], h[2], h[3]);
    }
    for (uint32_t w = nw + lane; w < sstride / 16; w += 32) out[w] = make_uint4(0, 0, 0, 0);
    for (int o = 16; o; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
    if (lane == 0) snorm[i] = nrm;
  }
}

void launch_screen_rows(const IndexView& ix, uint8_t* screen, uint64_t sstride, float* snorm,
                        cudaStream_t st) {
  const int grid = (int)std::min<uint64_t>((ix.n + 7) / 8, 148 * 16);
  k_screen_rows<<<grid, 256, 0, st>>>(ix.points, ix.stride, ix.n, ix.d, screen, sstride, snorm);
}

}  // namespace ddk
