// Beam-search kernels of the B200 Vamana hot path.
//
//   k_search : one warp per batch point: beam_search on the round-start
//              graph; the visited list goes to the point's global slice
//              (include/index.h:274-278; src/bsp_index.hpp:259-268)
//   k_query  : searchAll (include/utils/beamSearch.h:314-346), mixed L
//   k_beam   : beam_search with the full frontier and visited outputs
#include <cfloat>
#include <cstdio>

#include "dd_common.cuh"
#include "kernel_util.cuh"
#include "kernels.cuh"
#include "prune_core.cuh"
#include "search_core.cuh"
#include "sort_emul.cuh"

namespace ddk {

// Per-warp shared memory of the search kernels:
//   build search: qv | frontier | step candidates | hash table; the visited
//     list goes to the point's slice of a global array (read by k_prune).
//   query / debug: qv | frontier | step candidates | visited | evicted | hash.
// With h24 the hash table stores 24-bit ids (3 bytes a slot instead of 4),
// which is exact whenever every id is below 0xFFFFFF.
WarpLayout make_search_layout(uint32_t d, int dtype, uint32_t L, uint32_t Rp, uint32_t vcap,
                              bool build, bool h24, bool keep_vis, bool fastf, bool hash_global) {
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
  w.fastf = (build && fastf) ? 1u : 0u;
  w.hbits = w.fastf ? fast_hash_bits(L) : hash_bits_for(L);
  w.h24 = h24 ? 1u : 0u;
  const uint32_t hash_bytes =
      r16(w.fastf ? fast_table_bytes(w.hbits) : hash_table_bytes(w.hbits, h24));
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
    w.ws = off; off += 128;  // filter of the evicted ids
    if (keep_vis) {          // the debug search keeps its evicted list here too
      w.ev = off; off += r16(4ull * vcap);
    }
    w.hash_global = hash_global ? 1u : 0u;
    w.hash_words = hash_bytes / 4;
    if (!hash_global) off += hash_bytes;
  }
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
  S.ev_bloom = nullptr;
  S.hash = (uint32_t*)(base + w.ws);
  S.h24 = (int)w.h24;
  return S;
}

// query / debug layout: everything in shared memory
// global_hash / global_ev: this warp's global slices (hash_global layouts; the
// evicted list of layouts without keep_vis)
__device__ __forceinline__ SearchSmem carve_query(uint8_t* base, const WarpLayout& w,
                                                  uint32_t* global_hash = nullptr,
                                                  uint32_t* global_ev = nullptr) {
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
  S.ev_bloom = (uint32_t*)(base + w.ws);
  S.ev_id = w.keep_vis ? (uint32_t*)(base + w.ev) : global_ev;
  S.hash = w.hash_global ? global_hash
                         : (uint32_t*)(base + w.ws + 128 + (w.keep_vis ? r16(4ull * w.vcap) : 0));
  S.h24 = (int)w.h24;
  return S;
}

// ============================================================ build round
// k_search: one warp per batch point runs beam_search on the round-start graph
// and leaves its visited list in the point's global slice
// (include/index.h:274-278; src/bsp_index.hpp:259-268).
// FASTF: the fast form's seen filter, with registers capped at 64 (L <= 128)
// so that four CTAs of up to 8 warps fit an SM; at L = 128 a search takes
// 6.2 KB of shared memory with that filter's 4 KB table, and the autotuner
// settles on four 7-warp CTAs (28 searches per SM).
template <int DT, int MT, int FPL, int CPL, bool FASTF>
__global__ void __launch_bounds__((FASTF && FPL == 4) ? 256 : 512, (FASTF && FPL == 4) ? 4 : 1)
    k_search(IndexView ix, RoundArgs ra, WarpLayout lay) {
  extern __shared__ uint4 smem_raw[];
  const uint32_t wpc = blockDim.x >> 5;
  const uint32_t wic = threadIdx.x >> 5;
  const uint64_t gw = (uint64_t)blockIdx.x * wpc + wic;
  uint8_t* base = (uint8_t*)smem_raw + (size_t)wic * lay.total;
  SearchParams P;
  P.points = ix.points; P.stride = ix.stride; P.graph = ix.graph; P.Rp = ix.Rp; P.n = ix.n;
  P.d = ix.d; P.start = ra.start; P.L = ra.L; P.k = 0; P.cut = 0.0; P.limit = ix.n;
  P.degree_limit = ix.R; P.hbits = lay.hbits; P.vcap = lay.vcap; P.ecap = 0; P.query_mode = 0;
  P.keep_visited = 1; P.err = ix.err;
  P.screen = ix.screen; P.sstride = ix.sstride; P.snorm = ix.snorm; P.fgroup_lg = ix.fgroup_lg;
  const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
  uint64_t cur = gw;
  const uint64_t step = (uint64_t)gridDim.x * wpc;
  for (uint64_t b = warp_next_item(ra.qsearch, cur, step); b < ra.B;
       b = warp_next_item(ra.qsearch, cur, step)) {
    const uint32_t p = (uint32_t)(ra.floor + b);
    const SearchSmem S = carve_build(base, lay, ra.vis_all + b * 2ull * lay.vcap);
    load_vec(S.qv, ix.points + (uint64_t)p * ix.stride, qb);
    __syncwarp();
    const SearchOut o = warp_beam_search<DT, MT, FPL, CPL, FASTF>(P, S, p);
    if (lane_id() == 0) {
      ra.stat_vis[b] = o.vis_n;
      if (ra.stat_cmps) ra.stat_cmps[b] = o.cmps;
    }
    __syncwarp();
  }
}

// ============================================================ queries
template <int DT, int MT, int FPL, int CPL>
__global__ void __launch_bounds__(512) k_query(IndexView ix, QueryArgs qa, WarpLayout lay) {
  extern __shared__ uint4 smem_raw[];
  const uint32_t wpc = blockDim.x >> 5, wic = threadIdx.x >> 5, lane = lane_id();
  const uint64_t gw = (uint64_t)blockIdx.x * wpc + wic;
  // large seen tables (beam widths above 128) live in this warp's global slice
  const SearchSmem S =
      carve_query((uint8_t*)smem_raw + (size_t)wic * lay.total, lay,
                  lay.hash_global ? qa.hash_scratch + gw * (uint64_t)lay.hash_words : nullptr,
                  qa.ev_scratch + gw * (uint64_t)qa.ev_cap);
  const uint32_t qb = r16((uint64_t)ix.d * ElemSize<DT>::v);
  const uint64_t nitems = qa.cls_items ? (uint64_t)*qa.cls_count : qa.nq;
  uint64_t cur = gw;
  const uint64_t step = (uint64_t)gridDim.x * wpc;
  for (uint64_t it = warp_next_item(qa.cls_queue, cur, step); it < nitems;
       it = warp_next_item(qa.cls_queue, cur, step)) {
    const uint64_t q = qa.cls_items ? qa.cls_items[it] : it;
    SearchParams P;
    uint32_t Lq = qa.Ls[q];
    if (Lq == 0 || Lq > qa.Lvalid || Lq < qa.k) {
      if (lane == 0) dd_set_error(ix.err, DD_ECAND_CAP);
      Lq = qa.Lvalid;
    }
    P.points = ix.points; P.stride = ix.stride; P.graph = ix.graph; P.Rp = ix.Rp; P.n = ix.n;
    P.d = ix.d; P.start = qa.start; P.L = Lq; P.k = qa.k; P.cut = qa.cut; P.limit = qa.limit;
    P.degree_limit = qa.degree_limit; P.hbits = hash_bits_for(P.L); P.vcap = 0;
    P.ecap = qa.ev_cap; P.query_mode = 1; P.keep_visited = 0; P.err = ix.err;
    P.screen = ix.screen; P.sstride = ix.sstride; P.snorm = ix.snorm;
    P.fgroup_lg = ix.fgroup_lg;
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

__global__ void k_bin_queries(const uint32_t* Ls, uint64_t nq, uint32_t k, uint32_t Lvalid,
                              uint32_t* items, uint32_t* counts) {
  for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nq;
       q += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t L = Ls[q];
    if (L == 0 || L > Lvalid || L < k) L = Lvalid;
    const int c = query_class(L);
    items[(uint64_t)c * nq + atomicAdd(&counts[c], 1u)] = (uint32_t)q;
  }
}

void launch_bin_queries(const uint32_t* Ls, uint64_t nq, uint32_t k, uint32_t Lvalid,
                        uint32_t* items, uint32_t* counts, cudaStream_t st) {
  const int grid = (int)std::min<uint64_t>((nq + 255) / 256, 1024);
  k_bin_queries<<<grid, 256, 0, st>>>(Ls, nq, k, Lvalid, items, counts);
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
    P.degree_limit = ba.degree_limit; P.hbits = lay.hbits; P.vcap = lay.vcap; P.ecap = lay.vcap;
    P.query_mode = ba.k > 0; P.keep_visited = 1; P.err = ix.err;
    P.screen = nullptr; P.sstride = 0; P.snorm = nullptr; P.fgroup_lg = 0;  // the plain form
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
#define CALL4(DT, MT, F, C)                                                          \
  p = lay.fastf ? plan_warp_kernel(k_search<DT, MT, F, C, true>, lay.total)          \
                : plan_warp_kernel(k_search<DT, MT, F, C, false>, lay.total);
#define CALL(DT, MT) DD_DISPATCH_FC(L, ix.Rp, DT, MT, CALL4)
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
#undef CALL4
  return p;
}

std::vector<LaunchPlan> search_plan_candidates(const IndexView& ix, const WarpLayout& lay,
                                               uint32_t L) {
  std::vector<LaunchPlan> v;
#define CALL4(DT, MT, F, C)                                                          \
  v = lay.fastf ? warp_kernel_candidates(k_search<DT, MT, F, C, true>, lay.total)    \
                : warp_kernel_candidates(k_search<DT, MT, F, C, false>, lay.total);
#define CALL(DT, MT) DD_DISPATCH_FC(L, ix.Rp, DT, MT, CALL4)
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
#undef CALL4
  return v;
}

void launch_search(const IndexView& ix, const RoundArgs& ra, const WarpLayout& lay,
                   const LaunchPlan& plan, int grid, cudaStream_t st) {
  const size_t sm = (size_t)lay.total * plan.warps_per_cta;
#define CALL5(DT, MT, F, C, X)                                                       \
  set_smem(k_search<DT, MT, F, C, X>, sm);                                           \
  k_search<DT, MT, F, C, X><<<grid, plan.warps_per_cta * 32, sm, st>>>(ix, ra, lay);
#define CALL4(DT, MT, F, C)                                                          \
  if (lay.fastf) { CALL5(DT, MT, F, C, true); } else { CALL5(DT, MT, F, C, false); }
#define CALL(DT, MT) DD_DISPATCH_FC(ra.L, ix.Rp, DT, MT, CALL4)
  DD_DISPATCH_DM(ix.dtype, ix.metric, CALL);
#undef CALL
#undef CALL5
#undef CALL4
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

}  // namespace ddk
