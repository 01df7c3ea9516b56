// dd_robust_prune_noalloc: robustPrune on explicit candidate lists with no
// device allocation at all.
//
// Some callers cannot call cudaMalloc while they run this step: a host that
// has reserved all device memory up front and forbids allocation afterwards
// (a serving process with a fixed budget: cudaMalloc may also synchronize the
// device and stall its other streams), or a caller whose memory belongs to
// another allocator that must not be bypassed.  For them this entry point
// takes device pointers for every input and output and keeps its candidate
// workspace in the fixed-size device array below, which every GPU that loads
// the library holds until the process exits.
//
// The workspace is shared by all calls on a device and keeps the last call's
// contents.  Every call rewrites each part of it before reading it (the leaf
// bitmap of the sort emulation is cleared by the kernel), so nothing has to
// start at zero; calls whose kernels overlap on the GPU (different streams or
// handles on the same device) race on it and must be serialized by the caller.
#include <cstdio>
#include <mutex>

#include "../../include/dd_gpu.h"
#include "dd_common.cuh"
#include "internal.h"
#include "kernels.cuh"
#include "prune_core.cuh"

namespace {

using namespace ddk;

// Capacity of the workspace: sum over tasks of (candidates + Rp) slots, and tasks.
constexpr uint64_t kNoAllocMaxSlots = 1u << 16;
constexpr uint32_t kNoAllocMaxTasks = 2048;
// ids (slots) | distances (slots) | bitmap + stack + rank scratch (3*slots + tasks*stack)
constexpr uint64_t kNoAllocWords =
    5 * kNoAllocMaxSlots + (uint64_t)kNoAllocMaxTasks * kGlobalStackInts;

static __device__ __align__(256) uint32_t g_prune_workspace[kNoAllocWords];

// per-device address of g_prune_workspace (the host-side symbol is only a
// stand-in: kernels must be given the device address)
std::mutex g_mu;
void* g_workspace_addr[256] = {nullptr};

// k_prune_tasks with the workspace slices carved from the fixed array and with
// the device-side inputs validated (the host cannot read them).  Task slices
// are disjoint only when the offsets never decrease, so every warp first checks
// the whole offsets array (at most kNoAllocMaxTasks + 1 words): offsets that
// decrease or do not end at `total` invalidate the call and every row is
// padded.  An id >= n (p or a candidate) pads only its own task's row.
template <int DT, int MT>
__global__ void k_prune_tasks_fixed(IndexView ix, PruneArgs pa, uint64_t total) {
  const uint32_t lane = lane_id();
  bool offsets_ok = pa.offsets[pa.ntasks] == total;
  for (uint32_t t = lane; t < pa.ntasks; t += 32)
    if (pa.offsets[t] > pa.offsets[t + 1]) offsets_ok = false;
  offsets_ok = __all_sync(0xffffffffu, offsets_ok);
  for (uint32_t t = blockIdx.x; t < pa.ntasks; t += gridDim.x) {
    uint32_t* out_row = pa.out + (uint64_t)t * ix.Rp;
    const uint32_t p = pa.p[t];
    const uint64_t o0 = pa.offsets[t], o1 = pa.offsets[t + 1];
    bool ok = offsets_ok && p < ix.n;
    if (ok) {
      for (uint64_t j = o0 + lane; j < o1; j += 32)
        if (pa.cand_ids[j] >= ix.n) ok = false;
      ok = __all_sync(0xffffffffu, ok);
    }
    if (!ok) {
      if (lane == 0) dd_set_error(ix.err, DD_EBAD_ID);
      for (uint32_t j = lane; j < ix.Rp; j += 32) out_row[j] = DD_NONE;
      continue;
    }
    const uint64_t wbase = o0 + (uint64_t)t * ix.Rp;
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
        uint32_t pos = m + __popc(vb & lanemask_lt_());
        cid[pos] = a;
        ckey[pos] = Dist<DT, MT>::eval(pv, ix.points + (uint64_t)a * ix.stride, ix.d);
      }
      m += __popc(vb);
    }
    __syncwarp();
    PruneSmem Pm = prune_ws(cid, ckey, ws, (uint32_t)cap);
    warp_std_sort(Pm, m);
    warp_greedy_select<DT, MT>(ix.points, ix.stride, ix.d, p, Pm, m, pa.alpha, ix.R, out_row,
                               ix.Rp);
  }
}

}  // namespace

extern "C" int dd_robust_prune_noalloc(dd_index* h, uint32_t ntasks, const uint32_t* p,
                                       const uint64_t* offsets, uint64_t total_cands,
                                       const uint32_t* cand_ids, const float* cand_dists,
                                       double alpha, uint32_t* out, int synchronize) {
  if (!h) return DD_ERR_ARG;
  if (ntasks == 0) return DD_OK;
  if (!p || !offsets || !out || (total_cands && (!cand_ids || !cand_dists)))
    return internal_fail(h, DD_ERR_ARG, "dd_robust_prune_noalloc: null device pointer");
  IndexView ix = internal_view(h);
  const uint64_t slots = total_cands + (uint64_t)ntasks * ix.Rp;
  if (ntasks > kNoAllocMaxTasks || slots > kNoAllocMaxSlots) {
    char msg[256];
    snprintf(msg, sizeof msg,
             "dd_robust_prune_noalloc: %u tasks / %llu workspace slots (candidates + %u per "
             "task) exceed the fixed workspace (%u tasks, %llu slots); split the call or use "
             "dd_robust_prune",
             ntasks, (unsigned long long)slots, ix.Rp, kNoAllocMaxTasks,
             (unsigned long long)kNoAllocMaxSlots);
    return internal_fail(h, DD_ERR_UNSUPPORTED, msg);
  }
  const int dev = internal_device(h);
  if (dev < 0 || dev >= 256) return internal_fail(h, DD_ERR_ARG, "device index out of range");
  cudaError_t e = cudaSetDevice(dev);
  if (e != cudaSuccess) return internal_fail(h, DD_ERR_CUDA, cudaGetErrorString(e));
  void* ws = nullptr;
  {
    // first call on this device: look up the array's device address (with the
    // device current).  Make this first call before any stream capture.
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_workspace_addr[dev]) {
      e = cudaGetSymbolAddress(&g_workspace_addr[dev], g_prune_workspace);
      if (e != cudaSuccess) {
        g_workspace_addr[dev] = nullptr;
        return internal_fail(h, DD_ERR_CUDA, cudaGetErrorString(e));
      }
    }
    ws = g_workspace_addr[dev];
  }
  uint32_t* base = (uint32_t*)ws;
  PruneArgs pa;
  pa.ntasks = ntasks;
  pa.p = p;
  pa.offsets = offsets;
  pa.cand_ids = cand_ids;
  pa.cand_d = cand_dists;
  pa.alpha = alpha;
  pa.out = out;
  pa.gcand = base;
  pa.gkey = (float*)(base + kNoAllocMaxSlots);
  pa.gws = (int*)(base + 2 * kNoAllocMaxSlots);
  const int grid = (int)(ntasks < 4096 ? ntasks : 4096);
  cudaStream_t st = internal_stream(h);
#define CALL(DT, MT) k_prune_tasks_fixed<DT, MT><<<grid, 32, 0, st>>>(ix, pa, total_cands);
  if (ix.dtype == DD_F32 && ix.metric == DD_L2) { CALL(DD_F32, DD_L2); }
  else if (ix.dtype == DD_F32) { CALL(DD_F32, DD_MIPS); }
  else if (ix.dtype == DD_I8 && ix.metric == DD_L2) { CALL(DD_I8, DD_L2); }
  else if (ix.dtype == DD_I8) { CALL(DD_I8, DD_MIPS); }
  else if (ix.metric == DD_L2) { CALL(DD_U8, DD_L2); }
  else { CALL(DD_U8, DD_MIPS); }
#undef CALL
  e = cudaGetLastError();
  if (e != cudaSuccess) return internal_fail(h, DD_ERR_CUDA, cudaGetErrorString(e));
  if (synchronize) return internal_check_error_word(h);
  return DD_OK;
}
