// Ground truth and graph-format kernels of the B200 Vamana hot path.
//
//   k_gt_*          : brute-force ground truth (FP64 for float data, exact
//                     integers otherwise)
//   k_to_ref_rows / k_from_ref_rows : device rows <-> the reference's
//                     [deg, nbr...] rows (include/utils/graph.h:126-128)
#include <cfloat>
#include <cstdio>

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
