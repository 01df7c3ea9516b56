// robustPrune kernels of the B200 Vamana hot path.
//
//   k_prune       : one warp per batch point: robustPrune of its visited list
//                   and its current out-list (include/index.h:279-285;
//                   src/bsp_index.hpp:269-277)
//   k_prune_tasks : robustPrune on explicit candidate lists (include/index.h:63-123)
//   k_sort_rows   : knn_index's final per-row sort (include/index.h:133-136)
#include <cfloat>
#include <cstdio>

#include "dd_common.cuh"
#include "kernel_util.cuh"
#include "kernels.cuh"
#include "prune_core.cuh"
#include "search_core.cuh"
#include "sort_emul.cuh"

namespace ddk {

// Per-warp shared memory of k_prune: p's vector | candidate ids | distances |
// sort workspace, which the fast greedy forms share after the sort.
PruneLayout make_prune_layout(uint32_t d, int dtype, uint32_t Rp, uint32_t ccap, bool tensor) {
  PruneLayout w{};
  uint32_t esz = dtype == DD_F32 ? 4 : 1;
  uint32_t off = 0;
  w.qv = off; off += r16((uint64_t)d * esz);
  w.cid = off; off += r16(4ull * ccap);
  w.ckey = off; off += r16(4ull * ccap);
  w.ws = off; off += prune_ws_bytes_sel(ccap, greedy_sel_bytes(d, dtype, Rp, tensor));
  w.ccap = ccap;
  w.total = r16(off);
  return w;
}

// k_prune: one warp per batch point runs robustPrune of its visited list plus
// its current out-list (include/index.h:279-285; src/bsp_index.hpp:269-277).
// TC: occlusion distances from tensor-core Gram tiles where they apply (the
// fast form); otherwise all on the CUDA cores (the plain form).
template <int DT, int MT, bool TC>
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
  uint64_t cur = gw;
  const uint64_t step = (uint64_t)gridDim.x * wpc;
  for (uint64_t b = warp_next_item(ra.qprune, cur, step); b < ra.B;
       b = warp_next_item(ra.qprune, cur, step)) {
    const uint32_t p = (uint32_t)(ra.floor + b);
    load_vec(qv, ix.points + (uint64_t)p * ix.stride, qb);
    // the visited list, sorted by (dist, id) like the reference's
    const uint32_t* vis = ra.vis_all + b * 2ull * vcap;
    uint32_t m = min(ra.stat_vis[b], vcap);
    const uint32_t off = ra.vis_sorted_tail ? vcap - m : 0u;
    for (uint32_t j = lane; j < m; j += 32) {
      Pm.cid[j] = vis[off + j];
      Pm.ckey[j] = __uint_as_float(vis[vcap + off + j]);
    }
    __syncwarp();
    if (!ra.vis_sorted_tail) warp_sort_pairs(Pm.cid, Pm.ckey, m);
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
    warp_greedy_select_fast<DT, MT, true, TC>(ix.points, ix.stride, ix.d, p, Pm, m, ra.alpha, ix.R,
                                    ra.new_out + b * ix.Rp, ix.Rp, Pm.sel,
                                    ra.new_key ? ra.new_key + b * ix.Rp : nullptr);
  }
}

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

LaunchPlan plan_prune(const IndexView& ix, const PruneLayout& lay, bool tensor) {
  LaunchPlan p{1, 1};
#define CALL(DT, MT)                                                                 \
  p = tensor ? plan_warp_kernel(k_prune<DT, MT, true>, lay.total)                    \
             : plan_warp_kernel(k_prune<DT, MT, false>, lay.total);
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
  return p;
}

std::vector<LaunchPlan> prune_plan_candidates(const IndexView& ix, const PruneLayout& lay,
                                              bool tensor) {
  std::vector<LaunchPlan> v;
#define CALL(DT, MT)                                                                 \
  v = tensor ? warp_kernel_candidates(k_prune<DT, MT, true>, lay.total)              \
             : warp_kernel_candidates(k_prune<DT, MT, false>, lay.total);
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
  return v;
}

void launch_prune_round(const IndexView& ix, const RoundArgs& ra, const PruneLayout& lay,
                        uint32_t vcap, const LaunchPlan& plan, int grid, bool tensor,
                        cudaStream_t st) {
  const size_t sm = (size_t)lay.total * plan.warps_per_cta;
#define CALL2(DT, MT, TC)                                                            \
  set_smem(k_prune<DT, MT, TC>, sm);                                                 \
  k_prune<DT, MT, TC><<<grid, plan.warps_per_cta * 32, sm, st>>>(ix, ra, lay, vcap);
#define CALL(DT, MT)                                                                 \
  if (tensor) { CALL2(DT, MT, true); } else { CALL2(DT, MT, false); }
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
#undef CALL2
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

}  // namespace ddk
